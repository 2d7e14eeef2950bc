// launch.h -- host-side declarations of the kernel launchers (implemented in
// the k_*.cu files) used by the prover schedule in prover.cu.
#pragma once
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime_api.h>

namespace wg {

typedef uint64_t u64;
typedef unsigned int u32;
struct TxState;
struct ProofScalars;
struct E3;

// Twiddle tables: w_{2^TW_LOG}^E = tw_hi[E >> TW_HALF] * tw_lo[E & (2^TW_HALF - 1)],
// and stage twiddles tw_stage[u] = w_{2^TW_STAGE_LOG}^u, u < 2^(TW_STAGE_LOG-1).
constexpr u32 TW_LOG = 26, TW_HALF = 13, TW_STAGE_LOG = 11;

// ---- Reed-Solomon encoder -------------------------------------------------
// A pass plan: npass passes of radix 2^logR[s] (sum = logN, each <= 2^11),
// pass s staging 2^logW[s] columns per CTA (LDE_W_AUTO: the built-in choice).
// minb: CTAs per SM the kernel's registers are sized for (2, 3 or 4; 0 = default).
// pipe: run the passes as persistent CTAs that copy the next tile in while
// transforming the current one (two tile buffers); the coset-form last pass
// always runs one tile per CTA.
constexpr u32 LDE_W_AUTO = 0xFF, LDE_MINB_DEFAULT = 3;
struct LdePlan {
    u32 logN, npass;
    u32 logR[3];
    u32 logW[3];
    u32 minb;
    u32 pipe;
};
struct NttPassArgs {
    const u64* src[3];
    u64 m;
    u64* tmp;
    u64* out;
    u32 depth, logN, logR, logS, logW, npass, pass, logR0, logR1, logE;
    u32 twist;  // last pass of two whose first is a pure broadcast (m <= columns): reads the message itself
    u32 cs;     // shared-memory words per tile column
    u32 tiles_per_plane, planes;  // pipelined kernel: tiles of one plane, planes
    const u64* tw_stage;
    const u64* tw_hi;
    const u64* tw_lo;
    const u64* tw_pass;  // this pass boundary's LdeTables entry, or null
    u32 vec2;            // every plane base and the message length allow 16-byte word pairs
};
struct LdeArgs {
    const u64* src[3];  // component planes of the message vector (block b at src[c] + b*m)
    u64 m;              // message length per block
    u32 depth;          // interleaving depth (blocks per component)
    u32 planes;         // depth * components
    u32 logN;           // codeword length
    u64* tmp;           // scratch, planes * N words
    u64* out;           // codeword planes, planes * N words
    const u64* tw_stage;
    const u64* tw_hi;
    const u64* tw_lo;
    const struct LdeTables* tables;  // inter-pass factors of the context, or null
};
// Inter-pass twiddle tables of one context.  The pass boundary of a
// 2^logNs-point (sub-)transform split as 2^logR rows x 2^logS columns
// (logS = logNs - logR) multiplies element (row i, column col) by
// w_{2^logNs}^(i col); its table holds those factors row by row,
// tab[i 2^logS + col], so the storing threads read them coalesced and the pass
// pays one multiply per element instead of two (the factor and its advance).
// Tables are built before a proof that uses the split is enqueued
// (lde_tables_prepare, outside any graph capture) and live as long as the
// context; a pass whose table is missing computes its factors by multiplying.
struct LdeTables {
    static constexpr u32 MAX_LOG = 24;  // largest table: 2^24 words (128 MiB)
    std::atomic<u64*> tab[(TW_LOG + 1) * (TW_STAGE_LOG + 1)];
    LdeTables() {
        for (auto& t : tab) t.store(nullptr);
    }
    const u64* get(u32 logNs, u32 logR) const {
        return logNs <= TW_LOG && logR <= TW_STAGE_LOG ? tab[logNs * (TW_STAGE_LOG + 1) + logR].load() : nullptr;
    }
};
// The plan launch_lde uses for a 2^logN codeword of a 2^logN / 2^logX message:
// an installed (autotuned) plan for (logN, logX) if there is one, else the
// built-in split.
LdePlan plan_lde(u32 logN, u32 logX);
LdePlan default_plan_lde(u32 logN);
bool lde_plan_valid(const LdePlan& p);
void lde_install_plan(u32 logX, const LdePlan& p);  // p.npass == 0 removes
void lde_clear_plans();
// Incremented by every plan install or clear (captured graphs hold the plans
// of their capture and are re-captured after a change).
u32 lde_plan_epoch();
size_t lde_installed_plans(u32* keys, LdePlan* plans, size_t cap);  // keys: logN << 8 | logX
// Launches one LDE with an explicit plan (autotuner).
int launch_lde_plan(const LdeArgs& a, const LdePlan& pl, cudaStream_t st);
int launch_lde(const LdeArgs& a, cudaStream_t st);
int lde_prepare();
// Builds the missing inter-pass tables of `pl` (or of plan_lde(logN, logX))
// whose size fits `room` bytes, on `st`, and waits for them before publishing
// them.  Returns the bytes allocated, or -1 after a CUDA error (the tables
// stay missing; the LDE still runs).
long long lde_tables_prepare_plan(LdeTables& t, const LdePlan& pl, const u64* tw_hi, const u64* tw_lo,
                                  cudaStream_t st, u64 room);
long long lde_tables_prepare(LdeTables& t, u32 logN, u32 logX, const u64* tw_hi, const u64* tw_lo, cudaStream_t st,
                             u64 room);
void lde_tables_free(LdeTables& t);
// Resident-CTA counts of the sumcheck round kernels on the current device
// (their grids never leave a partial wave); called once per context.
int sumcheck_prepare();

// ---- Merkle commitment ------------------------------------------------------
// Leaf i = BLAKE3 of row i (LE bytes of `depth` elements of `ncomp` words),
// written to nodes[i].  Rows are gathered from the codeword planes.
// hash: 0 = BLAKE3, 1 = SHA-256 (the engine a configuration's hash_id selects).
// perm_log_e > 0: coset-major rows -- leaf k hashes natural row
// (k >> (logN - perm_log_e)) + ((k mod 2^(logN - perm_log_e)) << perm_log_e).
int launch_leaves(const u64* planes, u64 N, u32 depth, u32 ncomp, u32* nodes, int hash, cudaStream_t st,
                  u32 perm_log_e = 0);
// `count` independent matrices: planes and node arrays `plane_stride` /
// `node_stride` words apart.
int launch_leaves_batch(const u64* planes, u64 N, u32 depth, u32 ncomp, u32* nodes, u32 count, u64 plane_stride,
                        u64 node_stride, int hash, cudaStream_t st, u32 perm_log_e = 0);
// Builds all Merkle levels above the leaves of a 2^logN-leaf tree in `nodes`
// ([leaves | level 1 | ... | root], 8 words per node).  The CTA that computes
// the root also performs the transcript step of irs_commit::commit
// (irs_commit.hpp:433-478): prover_message(root), then squeezes `n_ood`
// Ext3 out-of-domain points into sc->ood_pts[commit_idx].
int launch_merkle(u32* nodes, u32 logN, TxState* tx, ProofScalars* sc, int commit_idx, int n_ood, int hash,
                  cudaStream_t st);
// Tree levels only (no transcript) of `count` trees `node_stride` words apart.
int launch_merkle_batch(u32* nodes, u32 logN, u32 count, u64 node_stride, cudaStream_t st);

// ---- Out-of-domain evaluation ----------------------------------------------
// value_(j,v) = sum_i x_v[i] z_j^i for the points z_j = pts[j] and the vectors
// x_v, v < nvec (base vectors vec_stride words apart, or one Ext3 vector in
// three planes).  Vectors in [skip_lo, skip_hi) are skipped.  The last CTA
// stores value_(j,v) at out[j * out_stride + v] and sends the values as prover
// messages, point-major.
struct OodArgs {
    const u64* v[3];
    int ext3;
    u64 size;                 // coefficients per vector
    u32 nvec;
    u64 vec_stride;
    u32 skip_lo, skip_hi;
    const E3* pts;
    int n_ood;
    E3* out;
    u32 out_stride;
    TxState* tx;
    void* scratch;
    u32 scratch_values;       // n_ood * nvec capacity of the scratch
    int ext2;                 // target field GoldilocksExt2 (vectors and points (c0, c1, 0))
};
int launch_ood(const OodArgs& a, cudaStream_t st);
size_t ood_scratch_bytes(u64 max_size, u32 max_values);

// ---- Transcript / protocol steps (single-thread kernels) ---------------------
// deg: degree of the target field (3 Ext3, 1 Goldilocks): field elements cross
// the transcript as 3 or 1 words.
int launch_tx_init(TxState* tx, const unsigned char* ds, u32 ds_len, unsigned char* narg, u64 narg_cap,
                   unsigned char* hints, u64 hints_cap, ProofScalars* sc, unsigned deg, cudaStream_t st);
// Vector RLC, constraint RLC + initial sum (whir_prover.hpp:122-197) over
// nvec vectors and nwit initial commitments of `ood` OOD points each.
int launch_constraint_rlc(TxState* tx, ProofScalars* sc, int n_forms, int nwit, int ood, int nvec, cudaStream_t st);
// PoW: squeeze the 32-byte challenge, grind the minimum nonce, send it.
int launch_pow(TxState* tx, ProofScalars* sc, u64 threshold, int slot, int hash, cudaStream_t st);
// `count` Ext3 challenges into sc->sc_r[slot ..] (verifier_message_vec).
int launch_squeeze_challenges(TxState* tx, ProofScalars* sc, int slot, int count, cudaStream_t st);
// Sends every coefficient of the final folded vector (whir_prover.hpp:360-362).
int launch_send_vector(TxState* tx, const u64* c0, const u64* c1, const u64* c2, u64 size, cudaStream_t st);

// ---- Opening ------------------------------------------------------------------
struct OpenArgs {
    TxState* tx;
    ProofScalars* sc;
    const u64* planes;  // codeword planes of the first opened commitment
    const u32* nodes;   // its Merkle nodes
    u32 nwit;           // commitments opened at the same rows (initial commitments)
    u64 planes_stride;  // words from one commitment's planes to the next
    u64 nodes_stride;   // u32 words from one commitment's nodes to the next
    u64 N;              // codeword length
    u32 logN;
    u32 depth, ncomp;   // row = depth elements of ncomp words (vectors x 2^fold)
    u32 q;              // in-domain samples
    u64 gen;            // w_N (evaluation-domain generator)
    int stir;           // also fill sc->stir_pts/stir_vals[ood_offset + i]
    int use_vrlc;       // weigh vector v's columns by sc->vrlc[v] (first round)
    int ood_offset;
    int r_offset;       // sc->sc_r[r_offset .. r_offset + fold) are the folding randomness
    u32 fold;           // number of folding variables (2^fold columns per vector)
    u32 perm_log_e;     // coset-major rows (see launch_leaves); 0 = natural order
};
int launch_open(const OpenArgs& a, cudaStream_t st);
// STIR combination (whir_prover.hpp:283-336): copy the new commitment's OOD
// points/values into the STIR arrays, squeeze the geometric RLC, update the sum.
int launch_stir_rlc(TxState* tx, ProofScalars* sc, int commit_idx, int n_ood, int q, cudaStream_t st);

// ---- Covector / sumcheck ---------------------------------------------------------
// cov[i] = sum_f crlc_f eq(p_f, i) + sum_j crlc_{F+j} z_j^i over 2^logS entries
// (z_j = sc->init_ood_pts[j]).  With nvec > 1 the same pass writes the vector
// RLC vec[i] = sum_v vrlc_v x_v[i] of the committed base vectors
// (whir_prover.hpp:131-140).
struct CovInitArgs {
    u64* cov[3];
    u32 logS;
    const u64* points;  // n_forms * logS * 3 words (Ext3 coordinates)
    int n_forms, n_ood;
    ProofScalars* sc;
    void* scratch;
    u32 nvec;           // committed vectors (1: no vector RLC)
    bool write_vec;     // write vec_out (several vectors, or the lifted vector when no round reads the base one)
    const u64* vecs;    // nvec base vectors, 2^logS words each, back to back
    u64* vec_out[3];    // Ext3 planes of the combined vector
    u32 dense_mask;     // forms f with bit f set are dense covectors (their points slot is unused):
    const u64* dense[8];  // cov[i] += crlc_f * dense[f][i] (Ext3, AoS), crlc_0 = 1
    int ext2;           // target field GoldilocksExt2 (values (c0, c1, 0), X^2 = 7)
    TxState* tx;        // with ext2: a form value outside (c0, c1) sets TX_ERR_FIELD in tx->err
};
int launch_cov_init(const CovInitArgs& a, cudaStream_t st);
size_t cov_init_scratch_bytes(u32 logS, int n_forms, int n_ood);
// cov[i] += sum_j stir_rlc_j stir_pts_j^i (Ext3 OOD points first, then base points).
struct CovAccArgs {
    u64* cov[3];
    u64 size;
    int n_ext, n_base;
    ProofScalars* sc;
    void* scratch;
    int ext2;
};
int launch_cov_accumulate(const CovAccArgs& a, cudaStream_t st);
size_t cov_acc_scratch_bytes(u64 size, int n_points);

struct SumcheckArgs {
    const u64* a_base;  // non-null: the (unfolded) vector is in the base field
    u64* a_in[3];
    u64* a_out[3];
    u64* b[3];
    u64 size;           // vector size of this round (after the optional fold)
    int fold;           // fold from 2*size with sc->sc_r[fold_r] first
    int fold_r;
    int r_slot;         // this round's challenge goes to sc->sc_r[r_slot]
    u64 pow_threshold;
    int hash;           // PoW engine (0 BLAKE3, 1 SHA-256)
    TxState* tx;
    ProofScalars* sc;
    void* scratch;
    int ext2;           // target field GoldilocksExt2
};
// One sumcheck round (sumcheck_protocol.hpp:99-135) with the previous round's
// fold fused in.  PoW (if any) and the challenge squeeze happen in-stream.
int launch_sumcheck_round(const SumcheckArgs& a, cudaStream_t st);
// All `rounds` rounds of a small sumcheck (and the fold after the last one when
// fold_after) in one single-CTA kernel: round t's challenge goes to
// sc_r[r_slot + t].  Returns 1 (nothing launched) when the sumcheck is too
// large or has round PoW.
int launch_sumcheck_small(const SumcheckArgs& a, int rounds, int fold_after, cudaStream_t st);
// Fold only: a_out[i] = a_in[i] + r (a_in[i+size] - a_in[i]), same for b.
int launch_fold(const SumcheckArgs& a, cudaStream_t st);
size_t sumcheck_scratch_bytes();
// The initial sumcheck of one base-field vector against a covector of MLE
// forms and OOD points, by block evaluation (k_sc_tensor.cu): the k rounds'
// messages and challenges (sc_r[r_slot ..]), and the vector and covector folded
// to size 2^(n - k) in a_out / cov_out -- the state the round kernels reach,
// without writing the 2^n covector.  Target field Ext3 or the base field.
struct TscArgs {
    const u64* coeffs;  // 2^n base coefficients
    u32 n, k;           // variables, initial-sumcheck rounds (no round PoW)
    const u64* points;  // n_forms MLE points, n Ext3 coordinates each
    int n_forms, n_ood; // terms: the forms, then sc->init_ood_pts[0 .. n_ood)
    ProofScalars* sc;
    TxState* tx;
    int r_slot;
    u64* a_out[3];
    u64* cov_out[3];
    void* scratch;      // tsc_scratch_bytes
    size_t scratch_bytes;
};
bool tsc_applicable(u32 n, u32 k, int n_terms);
size_t tsc_scratch_bytes(u32 n, u32 k, int n_terms);
int launch_tsc(const TscArgs& a, cudaStream_t st);

// ---- Twiddle tables ----------------------------------------------------------------
void host_twiddles(u64* stage /*1024*/, u64* hi /*8192*/, u64* lo /*8192*/);

}  // namespace wg

namespace wg {
// Multilinear extension of base coefficients at one Ext3 point; the result
// (3 words) is written to `out` in device memory.
int launch_mle_eval(const u64* coeffs, u32 logS, const u64* point, void* scratch, u64* out, cudaStream_t st);
size_t mle_eval_scratch_bytes(u32 logS);

// Streaming multiprocessors of the current device (cudaDevAttrMultiProcessorCount,
// looked up once per device); grid-stride kernels size their grids from it.
u32 device_sms();

// Process-wide count of kernel launches issued by the launchers.
void count_launches(u64 k);
u64 launch_count();

// Kernel-family timing hooks used by the schedule (null timer = off).
enum Family { FAM_NTT = 0, FAM_LEAF, FAM_MERKLE, FAM_OOD, FAM_SUMCHECK, FAM_COV, FAM_POW, FAM_OPEN, FAM_TX, FAM_COUNT };
struct Timer {
    virtual ~Timer() {}
    virtual void begin(int fam, cudaStream_t st) = 0;
    virtual void end(int fam, cudaStream_t st) = 0;
};
}  // namespace wg
