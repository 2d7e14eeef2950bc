// state.cuh -- per-proof device state shared by all kernels of one proof.
//
// Everything the reference prover keeps in host variables between transcript
// interactions (whir_prover.hpp:56-407: the running sum, folding randomness,
// OOD points/values, constraint and STIR combination coefficients, opened
// indices, PoW nonces) lives here in HBM, so the whole commit+prove is one
// stream of kernels with no host round trip.
#pragma once
#include "gl.cuh"
#include "transcript.cuh"

namespace wg {

constexpr int MAX_OOD = 8;          // out-of-domain samples per commitment
constexpr int MAX_FORMS = 8;        // statement linear forms
constexpr int MAX_QUERIES = 1024;   // in-domain samples per opening
constexpr int MAX_SC_ROUNDS = 64;   // total sumcheck rounds (= num_variables)
constexpr int MAX_WITNESSES = 8;    // initial commitments proven together
constexpr int MAX_VECTORS = 64;     // committed vectors over all initial commitments
constexpr int MAX_COMMITS = 32;     // initial + round commitments
constexpr int MAX_DEPTH = 64;       // interleaving depth 2^k
constexpr int MAX_INIT_OOD = MAX_WITNESSES * MAX_OOD;

// Natural row of committed row k: k itself, or with coset-major rows of
// message length 2^log_m and 2^log_e cosets, k / 2^log_m + (k mod 2^log_m) 2^log_e
// (transpose_permute, rust/src/algebra/ntt/transpose.rs:10-15).
__host__ __device__ __forceinline__ u64 codeword_row(u64 k, u32 logN, u32 log_e) {
    if (!log_e) return k;
    const u32 log_m = logN - log_e;
    return (k >> log_m) + ((k & ((1ull << log_m) - 1)) << log_e);
}

struct ProofScalars {
    E3 sum;                                  // claimed <vector, covector>
    E3 c0, c2;                               // current sumcheck round polynomial
    E3 sc_r[MAX_SC_ROUNDS];                  // folding randomness, in order (= evaluation point)
    E3 ood_pts[MAX_COMMITS][MAX_OOD];        // commitment c's OOD points (initial commitments first)
    E3 ood_vals[MAX_COMMITS][MAX_OOD];       // round commitments' OOD values
    // The initial commitments' OOD points in order, and the values of every
    // committed vector at each of them: init_ood_mat[i * V + v].
    E3 init_ood_pts[MAX_INIT_OOD];
    E3 init_ood_mat[MAX_INIT_OOD * MAX_VECTORS];
    E3 vrlc[MAX_VECTORS];                    // vector RLC coefficients
    E3 crlc[MAX_FORMS + MAX_INIT_OOD];       // constraint RLC coefficients
    E3 forms_eval[MAX_FORMS * MAX_VECTORS];  // claimed evaluations (input), form-major [f * V + v]
    E3 stir_rlc[MAX_QUERIES + MAX_OOD];      // STIR combination coefficients of the current round
    E3 stir_pts[MAX_QUERIES + MAX_OOD];      // OOD points then in-domain points (base, lifted)
    E3 stir_vals[MAX_QUERIES + MAX_OOD];
    u64 indices[MAX_QUERIES];                // opened rows of the current opening
    u64 pow_best;                            // minimum valid nonce (atomicMin target)
    u64 pow_next;                            // next unclaimed nonce chunk of the search
    u64 pow_nonces[MAX_COMMITS + 4];         // recorded nonces (diagnostics)
    unsigned char pow_ch[32];
    unsigned counters[64];                   // self-resetting last-block tickets
};
// ProofScalars::counters slots.
constexpr int CTR_MERKLE_TAIL = 0;  // k_merkle_tail: subtree CTAs finished

}  // namespace wg
