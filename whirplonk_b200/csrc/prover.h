// prover.h -- the device-resident WHIR prover schedule.
//
// A ProofPlan is a pure function of (num_variables, ProtocolParameters,
// number of statement forms): every buffer offset and every kernel launch of
// commit + prove is fixed by it.  All data-dependent values (challenges,
// indices, nonces, hint lengths) stay on the device, so a plan is enqueued
// without a single host synchronisation and can be captured into a CUDA graph.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime_api.h>

#include "params.h"

namespace wg {

struct TxState;
struct ProofScalars;

struct CommitBuffers {
    uint64_t N = 0;
    uint32_t logN = 0, depth = 0, ncomp = 0;
    uint32_t logX = 0;        // log2(N / message length per plane): the LDE's expansion
    uint32_t perm_log_e = 0;  // coset-major rows: log2(N / message length); 0 = natural order
    size_t planes = 0, nodes = 0;  // byte offsets in the workspace
};

struct ProofPlan {
    WhirSchedule sch;
    ProtocolParams params;
    uint32_t n = 0;          // num_variables
    int n_forms = 0;
    uint32_t dense_mask = 0;                 // statement forms that are dense covectors (bit f)
    const uint64_t* dense[8] = {};           // their device data: 2^n Ext3 values each, AoS (c0 c1 c2)
    uint32_t nwit = 1;       // initial commitments (witnesses), each of params.batch_size vectors
    uint32_t nvec = 1;       // committed vectors: nwit * batch_size
    size_t init_planes_stride = 0, init_nodes_stride = 0;  // bytes between the initial commitments' buffers
    // byte offsets in the workspace
    size_t off_coeffs = 0, off_a = 0, off_cov = 0, off_tmp = 0;
    size_t off_sc_scratch = 0, off_ood_scratch = 0, off_cov_scratch = 0;
    size_t off_tx = 0, off_scalars = 0, off_narg = 0, off_hints = 0, off_ds = 0, off_points = 0;
    std::vector<CommitBuffers> commits;  // [initial 0 .. initial nwit-1, round 0, round 1, ...]
    size_t a_plane_words = 0, cov_plane_words = 0;
    bool full_vector = false;  // the covector pass writes the lifted / combined vector (no base-field first round)
    uint32_t ood_values = 0;   // OOD scratch capacity in values (points x vectors)
    size_t narg_len = 0;       // exact narg length (every message has a fixed size)
    size_t narg_len_constrained = 0, narg_len_free = 0;  // with / without any constraint
    size_t hints_cap = 0;      // upper bound of the hint stream
    size_t ds_cap = 0;
    size_t total_bytes = 0;
    size_t total_sumcheck_rounds = 0;
    // When set, the transcript state lives here instead of in the workspace:
    // several plans then share one sponge and one proof stream (the two inner
    // proofs of the zero-knowledge prover).
    TxState* tx_ext = nullptr;
};

// Sets the statement's form count; a proof with no form and no OOD sample has
// no constraint (no initial sumcheck), which changes the narg length.
void plan_set_forms(ProofPlan& p, int n_forms);

// Throws std::invalid_argument on unsupported parameters.  The plan covers
// num_witnesses initial commitments of p.batch_size vectors each.
ProofPlan make_plan(uint32_t num_variables, const ProtocolParams& p, int n_forms, size_t ds_len,
                    uint32_t num_witnesses = 1);
// The same for a schedule given field by field (checked by validate_schedule);
// p supplies the hash engine, batch_size and field degree.
ProofPlan make_plan(const WhirSchedule& sched, const ProtocolParams& p, int n_forms, size_t ds_len,
                    uint32_t num_witnesses = 1);

struct LdeTables;
struct DeviceTables {
    uint64_t* tw_stage = nullptr;
    uint64_t* tw_hi = nullptr;
    uint64_t* tw_lo = nullptr;
    const LdeTables* lde = nullptr;  // the context's inter-pass twiddle tables
};

// Enqueue the whole commit (Config::commit, once per initial commitment) on
// `st`.  The workspace must hold the nvec coefficient vectors at off_coeffs and
// the domain-separator bytes at off_ds.  Without init_tx the commit continues
// the transcript already in plan_tx(p, ws).
struct Timer;
int enqueue_commit(const ProofPlan& p, char* ws, uint32_t ds_len, const DeviceTables& tw, cudaStream_t st,
                   Timer* timer = nullptr, bool init_tx = true);
// Enqueue Config::prove for MLE-point statements (points at off_points,
// claimed evaluations already in ProofScalars::forms_eval, form-major over
// the nvec vectors).
int enqueue_prove(const ProofPlan& p, char* ws, const DeviceTables& tw, cudaStream_t st, Timer* timer = nullptr);

TxState* plan_tx(const ProofPlan& p, char* ws);
ProofScalars* plan_scalars(const ProofPlan& p, char* ws);

}  // namespace wg
