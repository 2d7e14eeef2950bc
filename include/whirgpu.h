/* whirgpu.h -- C ABI of the B200-native WHIR prover (whirplonk_b200/libwhirgpu.so).
 *
 * Drop-in boundary for the reference C++ prover of hxd77/WhirPlonk
 * (cpp/include/whir/protocols/whir/whir.hpp, whir_prover.hpp): the same
 * ProtocolParameters, the same SHAKE128 Fiat-Shamir transcript and the same
 * proof byte layout ({narg_string, hints}), for
 *   M = Basefield<GoldilocksExt3> (Goldilocks vectors, Ext3 challenges),
 *   hash = BLAKE3 or SHA-2, one or more witnesses of batch_size vectors,
 *   statements of MultilinearExtension and dense Covector forms;
 * also M = Identity<Goldilocks>, Configs given field by field, and the
 * zero-knowledge prover ZkConfig<Goldilocks> (protocols/whir_zk).
 * Everything below is plain C: opaque handles, pointers, sizes and status
 * codes; no C++ types or exceptions cross this boundary.
 *
 * Threading: a context is used by one host thread at a time (the reference's
 * NttEngine singletons and GpuPool are single-threaded too,
 * cpp/include/whir/algebra/ntt/cooley_tukey_goldilocks.hpp:6-9).
 */
#ifndef WHIRGPU_H
#define WHIRGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    WHIRGPU_OK = 0,
    WHIRGPU_E_INVALID = 1,     /* bad argument or parameters the reference asserts on */
    WHIRGPU_E_UNSUPPORTED = 2, /* valid for the reference but not on this path (e.g. more than 64 vectors) */
    WHIRGPU_E_OOM = 3,         /* device or pinned memory exhausted, or above the HBM budget */
    WHIRGPU_E_CUDA = 4,        /* CUDA runtime error (text in whirgpu_last_error) */
    WHIRGPU_E_DEVICE = 5,      /* a kernel reported an error word (overflow, PoW exhausted) */
    WHIRGPU_E_TIMEOUT = 6,     /* a bounded device wait expired */
    WHIRGPU_E_TOO_LARGE = 7    /* size above the fixed capacity of an allocation-free entry point */
} whirgpu_status;

/* Byte-for-byte the fields of whir::ProtocolParameters
 * (cpp/include/whir/parameters.hpp:25-34), in the same order. */
typedef struct {
    uint8_t unique_decoding;
    uint64_t starting_log_inv_rate;
    uint64_t initial_folding_factor;
    uint64_t folding_factor;
    uint64_t security_level;
    uint64_t pow_bits;
    uint64_t batch_size;
    uint8_t hash_id[32]; /* EngineId: BLAKE3 (03e01749...5b4c) or SHA-2 (018eaa24...b076) */
} whirgpu_params;

typedef struct whirgpu_ctx whirgpu_ctx;
typedef struct whirgpu_transcript whirgpu_transcript;
typedef struct whirgpu_witness whirgpu_witness;

/* Coefficient pointers may be host or device memory. */
#define WHIRGPU_INPUT_HOST 0
#define WHIRGPU_INPUT_DEVICE 1

/* ---- context ---------------------------------------------------------------
 * One CUDA device, one stream, a workspace cache bounded by hbm_budget bytes
 * (0 = no bound).  Twiddle tables sit outside the bound: a few KiB of root
 * powers, plus one table of the inter-pass NTT factors per LDE split in use
 * (2^logN words, at most 128 MiB each, built on the first proof of a shape
 * and only while it fits under a nonzero bound).  Replaces the reference's
 * GpuPool singleton (cpp/cuda/cuda_integration.hpp:142-282). */
whirgpu_status whirgpu_ctx_create(int device, uint64_t hbm_budget, whirgpu_ctx** out);
void whirgpu_ctx_destroy(whirgpu_ctx* ctx);
const char* whirgpu_last_error(const whirgpu_ctx* ctx);
/* cudaStream_t of the context, for callers that time or order work around it. */
void* whirgpu_stream(whirgpu_ctx* ctx);
/* Codeword row order of the commitments this context makes from now on.
 * WHIRGPU_ORDER_NATURAL (the default): row i is the evaluation at w_N^i, as
 * the C++ reference commits (cpp/include/whir/algebra/ntt/mod_ntt.hpp:49-130).
 * WHIRGPU_ORDER_COSET_MAJOR: the Rust crate's order without its rs_in_order
 * feature (rust/src/algebra/ntt/cooley_tukey.rs:375-480): with message length
 * m and e = N / m cosets, committed row k is the evaluation at
 * w_N^(k / m + (k mod m) e) (transpose_permute, rust/src/algebra/ntt/
 * transpose.rs:10-15); the opened rows and their evaluation points follow.
 * Zero-knowledge commitments accept the natural order only (the Rust ZK
 * prover requires rs_in_order). */
#define WHIRGPU_ORDER_NATURAL 0
#define WHIRGPU_ORDER_COSET_MAJOR 1
whirgpu_status whirgpu_set_codeword_order(whirgpu_ctx* ctx, int order);

/* ---- parameters ------------------------------------------------------------
 * Round schedule of Config::from_params (whir.hpp:118-224) as a flat array:
 *   [n_rounds, init_N, init_q, init_ood, init_sumcheck_pow_thr, skip_pow_thr,
 *    per round: vector_size, N, q, ood, pow_thr, sumcheck_pow_thr,
 *    final_size, final_rounds, final_pow_thr, final_sumcheck_pow_thr]
 * Returns the number of words (0 on invalid parameters). */
size_t whirgpu_schedule(const whirgpu_params* params, uint64_t num_variables, uint64_t* out, size_t cap);

/* Device workspace bytes one proof of this shape occupies (0 when invalid):
 * what HBM-budget admission counts. */
uint64_t whirgpu_workspace_bytes(const whirgpu_params* params, uint64_t num_variables);

/* Domain separator of the reference CLI (cpp/main.cpp:174-215):
 * out[0..64) = SHA3-512(CBOR(params)), out[64..96) = SHA3-256(CBOR(session)). */
whirgpu_status whirgpu_cli_domain_separator(const whirgpu_params* params, uint8_t out[96]);

/* ---- transcript (ProverState, transcript.hpp:595-662) ------------------------ */
whirgpu_status whirgpu_transcript_create(whirgpu_ctx* ctx, const uint8_t protocol_id[64], const uint8_t session_id[32],
                                         const uint8_t* instance, size_t instance_len, whirgpu_transcript** out);
void whirgpu_transcript_destroy(whirgpu_transcript* tx);
/* Proof bytes after whirgpu_prove: pointers stay valid until the transcript is destroyed. */
whirgpu_status whirgpu_proof_get(const whirgpu_transcript* tx, const uint8_t** narg, size_t* narg_len,
                                 const uint8_t** hints, size_t* hints_len);

/* ---- commit (Config::commit, whir.hpp:303-309) ---------------------------------
 * Encodes, hashes and commits params->batch_size vectors of 2^num_variables
 * canonical Goldilocks words each, back to back in `coeffs`
 * (irs_commit::Config::commit with num_vectors = batch_size,
 * irs_commit.hpp:344-561); the codeword matrix and Merkle tree stay in HBM in
 * the witness.  Work is queued on the context stream; the call returns without
 * waiting for it.  The commit's kernels are captured into a CUDA graph on the
 * first call of a workspace (a proof shape) and replayed by later calls; an
 * NTT plan install or clear, or the family timer (whirgpu_set_timing), makes
 * the next call capture anew or launch directly. */
whirgpu_status whirgpu_commit(whirgpu_ctx* ctx, const whirgpu_params* params, const uint64_t* coeffs,
                              uint64_t num_variables, int coeffs_location, whirgpu_transcript* tx,
                              whirgpu_witness** out);
/* num_witnesses commits in a row on the same transcript, the reference caller's
 * `for (...) witnesses.push_back(config.commit(ps, vectors_w))` before one
 * Config::prove over all of them (whir_prover.hpp:56-120): coeffs holds
 * num_witnesses * batch_size vectors, witness w's first.  The handle stands
 * for all of them; whirgpu_prove then proves every vector.  At most
 * WHIRGPU_MAX_WITNESSES witnesses and WHIRGPU_MAX_VECTORS vectors in all. */
#define WHIRGPU_MAX_WITNESSES 8
#define WHIRGPU_MAX_VECTORS 64
whirgpu_status whirgpu_commit_witnesses(whirgpu_ctx* ctx, const whirgpu_params* params, const uint64_t* coeffs,
                                        uint64_t num_witnesses, uint64_t num_variables, int coeffs_location,
                                        whirgpu_transcript* tx, whirgpu_witness** out);
void whirgpu_witness_destroy(whirgpu_witness* w);

/* ---- a Config given field by field -----------------------------------------------
 * Config<M> (whir.hpp:104-116) as the reference's callers can also build it
 * by hand (cpp/tests/dump_whir.cpp:121-148), and the embedding M: the CLI's
 * --field Goldilocks3 (Basefield<GoldilocksExt3>, the default), Goldilocks2
 * (Basefield<GoldilocksExt2>, Fp[X]/(X^2 - 7)) or Goldilocks1
 * (Identity<Goldilocks>: challenges, sums and messages in the base field).
 * Target-field values cross this ABI as three words c0 c1 c2 (c2 = 0 for
 * Ext2, c1 = c2 = 0 for the base field).
 * Each committer's interleaving depth is 2^(rounds of the sumcheck after it) and
 * sizes chain from round to round (checked; WHIRGPU_E_INVALID otherwise). */
#define WHIRGPU_FIELD_GOLDILOCKS1 1
#define WHIRGPU_FIELD_GOLDILOCKS2 2
#define WHIRGPU_FIELD_GOLDILOCKS3 3
#define WHIRGPU_MAX_ROUNDS 24
typedef struct {
    uint64_t vector_size, codeword_length, interleaving_depth, in_domain_samples, out_domain_samples;
} whirgpu_irs_config;
typedef struct {
    uint64_t num_rounds;
    uint64_t pow_threshold; /* UINT64_MAX: no PoW */
} whirgpu_sumcheck_config;
typedef struct {
    whirgpu_irs_config irs_committer;
    uint64_t pow_threshold;
    whirgpu_sumcheck_config sumcheck;
} whirgpu_round_config;
typedef struct {
    uint32_t field;         /* WHIRGPU_FIELD_GOLDILOCKS3 / _GOLDILOCKS2 / _GOLDILOCKS1 */
    uint64_t batch_size;    /* vectors per commitment (initial_committer.num_vectors) */
    uint8_t hash_id[32];    /* engine of every Merkle layer and PoW */
    whirgpu_irs_config initial_committer;
    whirgpu_sumcheck_config initial_sumcheck;
    uint64_t initial_skip_pow;
    uint64_t num_rounds;
    whirgpu_round_config round_configs[WHIRGPU_MAX_ROUNDS];
    whirgpu_sumcheck_config final_sumcheck;
    uint64_t final_pow;
} whirgpu_config;
/* Config::from_params (whir.hpp:118-224) for the given field. */
whirgpu_status whirgpu_config_from_params(const whirgpu_params* params, uint64_t num_variables, uint32_t field,
                                          whirgpu_config* out);
/* whirgpu_commit_witnesses for a Config given field by field;
 * num_variables = log2(initial_committer.vector_size). */
whirgpu_status whirgpu_commit_config(whirgpu_ctx* ctx, const whirgpu_config* config, const uint64_t* coeffs,
                                     uint64_t num_witnesses, int coeffs_location, whirgpu_transcript* tx,
                                     whirgpu_witness** out);

/* ---- prove (Config::prove, whir_prover.hpp:56-407) ---------------------------
 * Statement: num_points MultilinearExtension forms; points are
 * num_points * num_variables Ext3 coordinates (3 words each, c0 c1 c2),
 * evaluations are num_points * V Ext3 values, form-major (the claimed MLE value
 * of form f on vector v at f * V + v), V = the witness's committed vectors.
 * On return the proof is complete and readable with whirgpu_proof_get.  Like
 * the commit, the prove replays a graph captured on the workspace's first call
 * with the same statement count (dense covector statements launch directly).
 * evaluation_point (optional) receives num_variables Ext3 values (the
 * FinalClaim evaluation point), rlc (optional) num_points Ext3 values. */
whirgpu_status whirgpu_prove(whirgpu_ctx* ctx, whirgpu_witness* witness, const uint64_t* points, size_t num_points,
                             const uint64_t* evaluations, whirgpu_transcript* tx, uint64_t* evaluation_point,
                             uint64_t* rlc);

/* The statement's linear forms as the reference builds them (linear_form.hpp:54-138):
 * a MultilinearExtension at a point, or a dense Covector -- the two LinearForm
 * kinds callers construct.  Forms are combined in the order given. */
#define WHIRGPU_FORM_MLE 0      /* data: num_variables Ext3 coordinates (host memory) */
#define WHIRGPU_FORM_COVECTOR 1 /* data: 2^num_variables Ext3 values, c0 c1 c2 each (host or device) */
typedef struct {
    uint32_t kind;
    int location;           /* WHIRGPU_INPUT_HOST / WHIRGPU_INPUT_DEVICE, for covector data */
    const uint64_t* data;
} whirgpu_linear_form;
/* Config::prove with num_forms (<= 8) forms of either kind; evaluations as in
 * whirgpu_prove (num_forms * V values, form-major).  Host covectors are copied
 * to a temporary device buffer freed before the call returns. */
whirgpu_status whirgpu_prove_forms(whirgpu_ctx* ctx, whirgpu_witness* witness, const whirgpu_linear_form* forms,
                                   size_t num_forms, const uint64_t* evaluations, whirgpu_transcript* tx,
                                   uint64_t* evaluation_point, uint64_t* rlc);

/* Bytes the last commit + prove pair moved host->device and device->host. */
void whirgpu_last_io_bytes(const whirgpu_ctx* ctx, uint64_t* h2d, uint64_t* d2h);

/* ---- zero-knowledge WHIR (ZkConfig<Goldilocks>, protocols/whir_zk) ------------------
 * ZkConfig::from_params / from_params_with_policy (whir_zk.hpp:95-105, 270-289):
 * `blinded` is the Config<Identity<Goldilocks>> of each f_hat = f + mask (one
 * vector per commitment), `blinding` the Config of the num_polynomials *
 * (num_variables + 1) blinding vectors of 2^(num_blinding_variables + 1)
 * entries.  policy NULL: BlindingSizePolicy::from_whir_params
 * (whir_zk.hpp:48-62).  WHIRGPU_E_INVALID where the reference asserts
 * (num_blinding_variables + 1 >= num_variables). */
typedef struct {
    uint64_t q_delta_1, q_delta_2, t1, t2, sumcheck_round_degree;
} whirgpu_zk_policy;
typedef struct {
    whirgpu_config blinded, blinding;
    uint64_t num_polynomials, num_witness_variables, num_blinding_variables;
} whirgpu_zk_config;
whirgpu_status whirgpu_zk_config_from_params(const whirgpu_params* params, uint64_t num_variables,
                                             uint64_t num_polynomials, const whirgpu_zk_policy* policy,
                                             whirgpu_zk_config* out);
/* The canonical ZK configuration bytes and domain separator
 * (canonical_config.hpp:38-87, whir_zk_domain_separator): config_bytes
 * (optional, WHIRGPU_ZK_CONFIG_BYTES bytes) = "WHIR_ZK_CONFIG_V1" || sizes,
 * parameters and policy as LE u64 words; out = SHA3-512(config_bytes) ||
 * SHA3-256(CBOR text session).  policy NULL: the derived policy.  Host only. */
#define WHIRGPU_ZK_CONFIG_BYTES 154
whirgpu_status whirgpu_zk_domain_separator(const whirgpu_params* params, uint64_t vector_size, uint64_t num_polynomials,
                                          const whirgpu_zk_policy* policy, const char* session, size_t session_len,
                                          uint8_t* config_bytes, uint8_t out[96]);
typedef struct whirgpu_zk_witness whirgpu_zk_witness;
/* ZkConfig::commit (whir_zk_impl.hpp:42-95) with the masks drawn from
 * DeterministicRng(seed, rng_domain) (deterministic_rng.hpp) starting at
 * counter 0: coeffs holds num_polynomials * 2^num_variables base-field
 * coefficients, polynomial i's first.  The num_polynomials blinded
 * commitments and the blinding commitment go to tx in that order.  Up to
 * WHIRGPU_MAX_WITNESSES polynomials and WHIRGPU_MAX_VECTORS blinding vectors;
 * rng_domain up to 128 bytes. */
whirgpu_status whirgpu_zk_commit(whirgpu_ctx* ctx, const whirgpu_zk_config* config, const uint64_t* coeffs,
                                 int coeffs_location, const uint8_t seed[32], const char* rng_domain,
                                 size_t rng_domain_len, whirgpu_transcript* tx, whirgpu_zk_witness** out);
/* ZkConfig::prove (whir_zk_impl.hpp:150-330): up to 7 linear forms as in
 * whirgpu_prove_forms, over the base field (every Ext3 value (x, 0, 0)), and
 * num_forms * num_polynomials claimed evaluations (Ext3 layout, form-major).
 * On return the proof is complete and readable with whirgpu_proof_get.  The
 * FinalClaim it returns is the blinded inner proof's (whir_zk_impl.hpp:305-310):
 * evaluation_point (optional) receives num_variables Ext3 values, rlc
 * (optional) num_forms Ext3 values, as in whirgpu_prove_forms. */
whirgpu_status whirgpu_zk_prove(whirgpu_ctx* ctx, whirgpu_zk_witness* witness, const whirgpu_linear_form* forms,
                                size_t num_forms, const uint64_t* evaluations, whirgpu_transcript* tx,
                                uint64_t* evaluation_point, uint64_t* rlc);
void whirgpu_zk_witness_destroy(whirgpu_zk_witness* witness);
/* The DeterministicRng byte stream (deterministic_rng.hpp:16-98) as 64-bit LE
 * words first_word .. first_word + count - 1, computed on the device. */
whirgpu_status whirgpu_deterministic_rng(whirgpu_ctx* ctx, const uint8_t seed[32], const char* domain,
                                         size_t domain_len, uint64_t first_word, uint64_t* out, size_t count);

/* ---- many proofs at once --------------------------------------------------------
 * A request is one complete commit + prove (with its own domain separator).
 * Proofs are independent: the bytes of each are the same alone or in a batch. */
typedef struct {
    uint64_t num_variables;
    whirgpu_params params;
    const uint64_t* coeffs;      /* params.batch_size vectors of 2^num_variables canonical words */
    int coeffs_location;         /* WHIRGPU_INPUT_HOST / WHIRGPU_INPUT_DEVICE */
    const uint64_t* points;      /* num_points * num_variables Ext3 coordinates */
    const uint64_t* evaluations; /* num_points * batch_size Ext3 values, form-major */
    uint64_t num_points;
    uint8_t protocol_id[64];
    uint8_t session_id[32];
} whirgpu_request;

typedef struct whirgpu_batch whirgpu_batch;
/* mode 0: the whole batch captured into one CUDA graph (one branch per proof,
 *         launched with a single cudaGraphLaunch per run);
 * mode 1: the same schedule issued stream by stream without a graph;
 * mode 2: plain -- one proof at a time, each waited for before the next.
 * Inputs are read again at every run (host inputs through pinned staging). */
whirgpu_status whirgpu_batch_create(whirgpu_ctx* ctx, const whirgpu_request* reqs, size_t count, int mode,
                                    whirgpu_batch** out);
whirgpu_status whirgpu_batch_run(whirgpu_batch* b);
whirgpu_status whirgpu_batch_proof(const whirgpu_batch* b, size_t i, const uint8_t** narg, size_t* narg_len,
                                   const uint8_t** hints, size_t* hints_len);
void whirgpu_batch_destroy(whirgpu_batch* b);

/* Serving: a worker thread admits submitted requests (their host buffers are
 * borrowed until poll has returned the result, and copied once into pinned
 * staging at admission) as
 * HBM budget and one of max_inflight streams free up -- continuous batching:
 * requests arriving while others run join them on the device.  Each
 * workspace keeps a captured CUDA graph of its proof program.  While a server
 * runs it owns the context.  poll waits up to timeout_ms (WHIRGPU_E_TIMEOUT
 * if not done); result pointers stay valid until whirgpu_server_release. */
typedef struct whirgpu_server whirgpu_server;
typedef struct {
    whirgpu_status status;
    const uint8_t* narg;
    size_t narg_len;
    const uint8_t* hints;
    size_t hints_len;
    double queue_ms; /* submit -> admission */
    double total_ms; /* submit -> proof complete */
} whirgpu_result;
whirgpu_status whirgpu_server_create(whirgpu_ctx* ctx, uint64_t hbm_budget, uint32_t max_inflight,
                                     whirgpu_server** out);
whirgpu_status whirgpu_server_submit(whirgpu_server* s, const whirgpu_request* req, uint64_t* ticket);
whirgpu_status whirgpu_server_poll(whirgpu_server* s, uint64_t ticket, uint32_t timeout_ms, whirgpu_result* out);
void whirgpu_server_release(whirgpu_server* s, uint64_t ticket);
void whirgpu_server_stats(whirgpu_server* s, uint64_t* admitted, uint64_t* peak_inflight, uint64_t* peak_bytes,
                          uint64_t* queued);
void whirgpu_server_destroy(whirgpu_server* s);

/* ---- kernel level: Reed-Solomon encoding and matrix commitment ----------------- */
/* RS-encode `count` vectors of 2^log_len canonical base-field words each, as
 * irs_commit::commit encodes one vector (irs_commit.hpp:402-411 -> mod_ntt.hpp:49-130):
 * interleaving depth 2^log_depth, block b = words [b m, (b+1) m) with
 * m = 2^(log_len - log_depth), codeword X_b[i] = sum_j v[b m + j] w_N^(i j) for
 * i < N = 2^log_expansion m, w_N = 7^((p-1)/N).  Device pointers only: the
 * vectors back to back; d_tmp and d_planes hold count * 2^log_depth * N words
 * each; plane (vector k, block b) = d_planes + (k 2^log_depth + b) N.
 * Enqueued on the context stream (whirgpu_stream); returns without waiting. */
whirgpu_status whirgpu_rs_encode(whirgpu_ctx* ctx, const uint64_t* d_vectors, size_t count, uint32_t log_len,
                                 uint32_t log_expansion, uint32_t log_depth, uint64_t* d_tmp, uint64_t* d_planes);
/* RS-encode and Merkle-commit `count` vectors (host or device memory, see
 * WHIRGPU_INPUT_*): per vector the root of irs_commit::commit's matrix
 * commitment (rows of 2^log_depth elements, leaf = BLAKE3 of the row's LE bytes,
 * matrix_commit.hpp:169-195; tree merkle_tree.hpp:104-147), written to
 * roots[32 k ..].  Synchronous.  Replaces the commitment half of
 * Config::commit (irs_commit.hpp:433-470) for many vectors at once, without the
 * transcript. */
whirgpu_status whirgpu_rs_commit_batch(whirgpu_ctx* ctx, const uint64_t* vectors, int location, size_t count,
                                       uint32_t log_len, uint32_t log_expansion, uint32_t log_depth, uint8_t* roots);

/* ---- NTT pass plans (autotuned) ------------------------------------------------- */
/* The LDE of a 2^log_n codeword from a 2^(log_n - log_expansion) message runs in
 * npass passes of radix 2^log_radix[s] (sum = log_n, each <= 11); pass s stages
 * 2^log_cols[s] columns per CTA (255 = built-in choice); the kernel variant's
 * registers are sized for min_blocks CTAs per SM (2..4, 0 = built-in);
 * pipelined = 1 runs the passes as persistent CTAs that copy the next tile in
 * while transforming the current one.  No counterpart in the reference (its
 * NTT engine picks fixed radices, cooley_tukey.hpp:200-259). */
typedef struct {
    uint32_t log_n, log_expansion, npass;
    uint32_t log_radix[3];
    uint32_t log_cols[3];
    uint32_t min_blocks;
    uint32_t pipelined;
} whirgpu_ntt_plan;
/* Times every valid plan for the shape on `planes` synthetic planes (median of
 * `reps` runs each), checks each plan's codeword against the built-in plan's,
 * installs the fastest agreeing plan for (log_n, log_expansion) and returns it.
 * Returns WHIRGPU_E_DEVICE (after installing) if any plan disagreed. */
whirgpu_status whirgpu_ntt_autotune(whirgpu_ctx* ctx, uint32_t log_n, uint32_t log_expansion, uint32_t planes,
                                    uint32_t reps, whirgpu_ntt_plan* best, double* best_us, uint32_t* tried);
/* Installs a plan (npass = 0 removes the shape's plan); process-wide. */
whirgpu_status whirgpu_ntt_set_plan(const whirgpu_ntt_plan* plan);
/* The plan the encoder uses for a shape (installed, else built-in). */
whirgpu_status whirgpu_ntt_get_plan(uint32_t log_n, uint32_t log_expansion, whirgpu_ntt_plan* out);
void whirgpu_ntt_clear_plans(void);
/* Installed plans (returns the count; writes at most cap). */
size_t whirgpu_ntt_list_plans(whirgpu_ntt_plan* out, size_t cap);
/* JSON plan files: {"plans": [{"log_n": .., "log_expansion": .., "npass": ..,
 * "log_radix": [..], "log_cols": [..], "min_blocks": .., "pipelined": ..}, ..]}
 * (min_blocks and pipelined optional). */
whirgpu_status whirgpu_ntt_load_plans(const char* path, size_t* loaded);
whirgpu_status whirgpu_ntt_save_plans(const char* path);
/* Installs, once per process, the plans in $WHIRGPU_NTT_PLANS or else in
 * ntt_plans.json beside the library (called by whirgpu_ctx_create). */
void whirgpu_ntt_load_default_plans(void);

/* ---- helpers ------------------------------------------------------------------- */
/* Multilinear extension of 2^num_variables base coefficients at an Ext3 point
 * (MultilinearExtension::evaluate, linear_form.hpp:119-126), on the device. */
whirgpu_status whirgpu_mle_evaluate(whirgpu_ctx* ctx, const uint64_t* coeffs, uint64_t num_variables,
                                    int coeffs_location, const uint64_t* point, uint64_t out[3]);
/* Allocation-free variant of whirgpu_mle_evaluate.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc where they need the
 * value (host callbacks and driver hooks, callers whose device memory comes
 * from their own pool or arena, latency-critical loops): it allocates nothing
 * and needs no context.  Inputs and output are device buffers the caller owns:
 * d_coeffs (2^num_variables words), d_point (num_variables Ext3 coordinates,
 * 3 words each), d_out (3 words); the work is queued on `stream`
 * (a cudaStream_t, NULL = legacy stream) of the current device and the call
 * returns without waiting.  Working memory is a fixed file-scope device array
 * of under 0.5 MiB, held on every GPU that loads the library until the process
 * exits; num_variables above WHIRGPU_NOALLOC_MLE_MAX_VARS is rejected with
 * WHIRGPU_E_TOO_LARGE.  Every call looks the array's device address up
 * (cudaGetSymbolAddress, which allocates nothing); the first lookup on a device
 * may load the library's module there, so make the first call on each device
 * before any stream capture.  A CUDA error already pending on the calling
 * thread is left for its owner: the call then returns WHIRGPU_E_CUDA and
 * queues nothing.  All calls on a device share the array: calls whose kernels
 * overlap on the GPU race and give wrong results, so order them on one
 * stream. */
#define WHIRGPU_NOALLOC_MLE_MAX_VARS 24
whirgpu_status whirgpu_mle_evaluate_noalloc(const uint64_t* d_coeffs, uint64_t num_variables, const uint64_t* d_point,
                                            uint64_t* d_out, void* stream);
/* Diagnostics: runs the device field arithmetic on n host operand pairs
 * (op 0: a+b, 1: a-b, 2: a*b in Goldilocks; 3: a*b in Ext3, three words per
 * element) and copies the results back.  Operands must be canonical. */
whirgpu_status whirgpu_debug_field_ops(const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t n, int op);
/* Seeded uniform Goldilocks words: ChaCha20 block function (RFC 8439),
 * key = seed as 8 LE bytes then 24 zero bytes, nonce 0, counter from 0;
 * each 64-bit LE keystream word below p is taken, others are skipped. */
void whirgpu_sample_goldilocks(uint64_t seed, uint64_t* out, size_t count);
/* Raw ChaCha20 block (for known-answer tests). */
void whirgpu_chacha20_block(const uint8_t key[32], uint32_t counter, const uint8_t nonce[12], uint8_t out[64]);
/* Page-locked host memory for fast host<->device copies. */
void* whirgpu_host_alloc(size_t bytes);
void whirgpu_host_free(void* p);

/* Integer-pipe peaks of `device`, measured (no reference counterpart): the
 * roofline denominators of the families bound by integer arithmetic.  Each
 * rate is operations per second of a register-only kernel over a full grid:
 * out[0] Goldilocks radix-2 butterflies (one multiply, add, subtract),
 * out[1] BLAKE3 compressions, out[2] 64x64-bit products accumulated into
 * 192 bits, then PTX instruction rates: out[3] mad.lo.u32, out[4]
 * mad.wide.u32, out[5] add.u32 (counted once per two-add pair a + b + c),
 * out[6] lop3.b32, out[7] shf.l.wrap.b32.  Takes well under a second. */
#define WHIRGPU_NUM_INT_PEAKS 8
whirgpu_status whirgpu_measure_int_peaks(int device, double out[WHIRGPU_NUM_INT_PEAKS]);

/* ---- timing of the hot kernels (for roofline reporting) --------------------------
 * When enabled, every kernel family is bracketed by CUDA events on the context
 * stream; whirgpu_kernel_stats returns, per family, launches and total ms
 * accumulated since the last reset.  Families: 0 NTT/LDE, 1 leaf hash,
 * 2 Merkle, 3 OOD, 4 sumcheck, 5 covector, 6 PoW, 7 opening, 8 transcript. */
#define WHIRGPU_NUM_FAMILIES 9
whirgpu_status whirgpu_set_timing(whirgpu_ctx* ctx, int enabled);
/* Number of kernels this library has launched in the process so far. */
uint64_t whirgpu_launch_count(void);
/* Workspace cache of the context: bytes of device memory its workspaces hold
 * now, workspaces allocated so far, and idle workspaces freed to make room
 * under an HBM budget (each such free synchronises the device). */
whirgpu_status whirgpu_workspace_stats(whirgpu_ctx* ctx, uint64_t* cached_bytes, uint64_t* allocations,
                                       uint64_t* evictions);
whirgpu_status whirgpu_kernel_stats(whirgpu_ctx* ctx, uint64_t launches[WHIRGPU_NUM_FAMILIES],
                                    double ms[WHIRGPU_NUM_FAMILIES], int reset);

#ifdef __cplusplus
}
#endif
#endif /* WHIRGPU_H */
