// zk.cu -- zero-knowledge WHIR (ZkConfig<Goldilocks>) on the device.
//
// The reference (cpp/include/whir/protocols/whir_zk/whir_zk_impl.hpp:42-330,
// whir_zk_utils.hpp) wraps two WHIR instances over Identity<Goldilocks>:
//   commit  per polynomial: sample the blinding polynomials from the RNG
//           (m_poly = g0_hat and msk interleaved, g_hat_0 .. g_hat_{mu-1}) and
//           commit f_hat = f + m_poly (applied with period |m_poly|); then
//           commit the blinding vectors [m_poly, embed(g_hat_j) ...] of every
//           polynomial as one batch;
//   prove   beta; every form folded to the mask period and its value on every
//           blinding vector (messages); rho; the in-domain opening of the f_hat
//           commitments; tau1, tau2; at each point gamma of the opened rows'
//           cosets the blinding values (messages) and their tau2-batched
//           claims; the inner proof of the f_hat commitments for the masked
//           claims; the inner proof of the blinding commitment for
//           [beq covector, folded forms].
// Both inner proofs run on the device schedule of prover.cu, in two workspaces
// of one allocation that share ONE transcript state and ONE proof stream
// (ProofPlan::tx_ext); the steps between the inner proofs are the kernels
// below, except the absorption of the per-gamma messages (tens of thousands
// of words), which the host CPU runs on a copy of the sponge between two
// device phases: a sequential Keccak is faster on one CPU core than on one warp.
// All arithmetic is in the base field (rho, beta, tau1, tau2 and every message
// are Goldilocks elements).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/whirgpu.h"
#include "blake3.cuh"
#include "ctx.h"
#include "host_keccak.h"
#include "launch.h"
#include "prover.h"
#include "state.cuh"
#include "wtx.cuh"

using namespace wg;

namespace wg {
namespace {

constexpr u32 ZK_MAX_LOG_HALF = 14;  // eq weights of one gamma in shared memory: 2^14 words
constexpr u32 ZK_RNG_MAX_DOMAIN = 128;
constexpr int ZK_MAX_DOTS = MAX_VECTORS + 2 * MAX_WITNESSES;

struct ZkScalars {
    u64 beta, rho, tau1, tau2;
};

__device__ __forceinline__ u64 gl_canon(u64 v) { return v >= GL_P ? v - GL_P : v; }  // Goldilocks::from_u64

__device__ __forceinline__ u64 warp_sum_gl(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = gl_add(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}

// ---- DeterministicRng (deterministic_rng.hpp:16-98) ---------------------------
// Block c of the stream = BLAKE3("WHIR_DETERMINISTIC_RNG_V1" || u32 |domain| ||
// domain || seed || u64 c), all LE; u64() reads the next 8 bytes LE.  The
// message (with c = 0) is built on the host; a thread hashes one block.
struct RngMsg {
    u32 w[64];  // message bytes, LE words, zero past len
    u32 len;    // 69 + |domain| <= 197: one chunk of at most 4 blocks
};

__global__ void k_zk_rng(RngMsg msg, u64 first_word, u64 count, u64* out) {
    const u64 c0 = first_word >> 2, c1 = (first_word + count + 3) >> 2;
    for (u64 c = c0 + (u64)blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += (u64)gridDim.x * blockDim.x) {
        u32 m[64];
#pragma unroll
        for (int i = 0; i < 64; ++i) m[i] = msg.w[i];
        const u32 off = msg.len - 8;
        for (u32 b = 0; b < 8; ++b) {
            const u32 p = off + b, sh = 8 * (p & 3);
            m[p >> 2] = (m[p >> 2] & ~(0xFFu << sh)) | ((u32)((c >> (8 * b)) & 0xFF) << sh);
        }
        const int nb = (int)((msg.len + 63) / 64);
        unsigned cv[8];
        b3_init(cv);
        for (int t = 0; t < nb; ++t) {
            const unsigned bl = t == nb - 1 ? msg.len - 64 * t : 64;
            b3_compress(cv, m + 16 * t, b3_flags(t, nb), bl, 0);
        }
        for (int k = 0; k < 4; ++k) {
            const u64 wi = 4 * c + k;
            if (wi >= first_word && wi < first_word + count)
                out[wi - first_word] = (u64)cv[2 * k] | ((u64)cv[2 * k + 1] << 32);
        }
    }
}

RngMsg rng_message(const uint8_t seed[32], const char* domain, size_t dlen) {
    static const char kPers[] = "WHIR_DETERMINISTIC_RNG_V1";
    uint8_t b[256] = {};
    size_t p = 0;
    std::memcpy(b, kPers, sizeof(kPers) - 1);
    p += sizeof(kPers) - 1;
    for (int i = 0; i < 4; ++i) b[p++] = (uint8_t)(dlen >> (8 * i));
    if (dlen) std::memcpy(b + p, domain, dlen);
    p += dlen;
    std::memcpy(b + p, seed, 32);
    p += 32 + 8;  // counter, patched per block
    RngMsg m{};
    std::memcpy(m.w, b, sizeof(m.w));
    m.len = (u32)p;
    return m;
}

// ---- commit: masks and blinding vectors ----------------------------------------
// Stream words of polynomial i start at i * (mu + 2) * half (sample order of
// BlindingPolynomials::sample, whir_zk_utils.hpp:112-140): msk[k], g0_hat[k]
// alternately for k < half, then g_hat_0 .. g_hat_{mu-1}.  So m_poly[j] (g0_hat
// at even j, msk at odd j) is stream word j ^ 1.

// f_hat = f + m_poly[i mod P] (whir_zk_impl.hpp:62-66), in place.
__global__ void k_zk_mask(u64* coeffs, const u64* R, u32 n, u32 logP, u32 npolys, u64 per_poly) {
    const u64 total = (u64)npolys << n, P = 1ull << logP;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u64 pi = e >> n, j = e & (P - 1);
        coeffs[e] = gl_add(coeffs[e], gl_canon(R[pi * per_poly + (j ^ 1)]));
    }
}

// Blinding vector v = i * (mu + 1) + t of P words (layout_vectors,
// whir_zk_utils.hpp:151-176): t = 0: m_poly; t >= 1: g_hat_{t-1} at even
// positions, zero at odd ones (embed_to_ell_plus_one).
__global__ void k_zk_layout(u64* out, const u64* R, u32 logP, u32 npolys, u32 mu, u64 per_poly) {
    const u64 P = 1ull << logP, half = P >> 1;
    const u64 total = (u64)npolys * (mu + 1) << logP;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u64 v = e >> logP, j = e & (P - 1);
        const u64 pi = v / (mu + 1), t = v % (mu + 1);
        const u64* r = R + pi * per_poly;
        u64 x;
        if (t == 0) x = gl_canon(r[j ^ 1]);
        else x = (j & 1) ? 0 : gl_canon(r[P + (t - 1) * half + (j >> 1)]);
        out[e] = x;
    }
}

// ---- prove ------------------------------------------------------------------
// fold_weight_to_mask_size (whir_zk_utils.hpp:283-303): W_f[j] = sum over
// i = j (mod P) of the form's covector.  For a MultilinearExtension (point[0]
// = most significant variable) the sum over the high variables of eq is 1, so
// W_f = eq(point[n - logP ..], j) over the low logP variables.
struct ZkFoldArgs {
    const E3* mle[MAX_FORMS];
    const E3* dense[MAX_FORMS];
    int nforms;
    u32 n, logP;
    E3* out;  // form f at out + f * P (AoS, the dense-covector layout)
};
__global__ void k_zk_fold(ZkFoldArgs a) {
    const u64 P = 1ull << a.logP;
    const u64 total = (u64)a.nforms * P;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const int f = (int)(e >> a.logP);
        const u64 j = e & (P - 1);
        E3 acc;
        if (a.mle[f]) {
            acc = e3_one();
            for (u32 b = 0; b < a.logP; ++b) {
                const E3 z = a.mle[f][a.n - 1 - b];
                acc = e3_mul(acc, ((j >> b) & 1) ? z : e3_sub(e3_one(), z));
            }
        } else {
            acc = e3_zero();
            const u64 reps = 1ull << (a.n - a.logP);
            for (u64 h = 0; h < reps; ++h) acc = e3_add(acc, a.dense[f][(h << a.logP) + j]);
        }
        a.out[e] = acc;
    }
}

// E[f * V + v] = <W_f, blinding vector v> (Covector::evaluate): one CTA per pair.
__global__ void k_zk_dots(const E3* W, const u64* vecs, u32 logP, u32 V, E3* out) {
    __shared__ E3 red[32];
    const u32 f = blockIdx.x / V, v = blockIdx.x % V;
    const u64 P = 1ull << logP;
    const E3* w = W + (u64)f * P;
    const u64* x = vecs + (u64)v * P;
    E3 acc = e3_zero();
    for (u64 j = threadIdx.x; j < P; j += blockDim.x) {
        const E3 c = w[j];
        const u64 s = x[j];
        acc = e3_add(acc, E3{gl_mul(c.c0, s), gl_mul(c.c1, s), gl_mul(c.c2, s)});
    }
    acc = e3_warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        E3 r = e3_zero();
        for (u32 k = 0; k < (blockDim.x >> 5); ++k) r = e3_add(r, red[k]);
        out[blockIdx.x] = r;
    }
}

// Steps 1-4 (whir_zk_impl.hpp:176-236): beta; the folded values as messages,
// form-major then polynomial then blinding vector; rho (non-zero); the masked
// claims of the f_hat proof (+ the forms' values on m_poly) and the claims of
// forms 1.. of the blinding proof.
__global__ void k_zk_tx_a(TxState* tx, ZkScalars* zs, const E3* E, int nforms, u32 V, u32 npolys, u32 mu,
                          ProofScalars* scb, ProofScalars* scg) {
    if (threadIdx.x >= 32) return;
    const u32 l = threadIdx.x;
    WarpTx t;
    wtx_load(t, tx);
    const u64 beta = wtx_challenge_base(t);
    for (u32 i = 0; i < (u32)nforms * V; ++i) wtx_message_t(t, E[i]);
    const u64 rho = wtx_challenge_base(t);
    if (rho == 0) t.err |= TX_ERR_FIELD;  // the reference asserts masking_challenge != 0
    wtx_store(t, tx);
    if (l == 0) {
        zs->beta = beta;
        zs->rho = rho;
    }
    for (u32 i = l; i < (u32)nforms * npolys; i += 32) {
        const u32 f = i / npolys, pi = i % npolys;
        scb->forms_eval[f * npolys + pi] = e3_add(scb->forms_eval[f * npolys + pi], E[f * V + pi * (mu + 1)]);
    }
    for (u32 i = l; i < (u32)nforms * V; i += 32) scg->forms_eval[V + i] = E[i];
}

// Step 6: tau1, tau2.
__global__ void k_zk_taus(TxState* tx, ZkScalars* zs) {
    if (threadIdx.x >= 32) return;
    WarpTx t;
    wtx_load(t, tx);
    const u64 tau1 = wtx_challenge_base(t);
    const u64 tau2 = wtx_challenge_base(t);
    wtx_store(t, tx);
    if (threadIdx.x == 0) {
        zs->tau1 = tau1;
        zs->tau2 = tau2;
    }
}

// Step 7 (all_gammas, whir_zk.hpp:158-173; evaluate_gamma_block,
// whir_zk_utils.hpp:333-440), one CTA per gamma: opened row idx_i, coset
// member j: gamma = omega_full^(idx_i + j N) (omega_full of order N * depth,
// zeta = omega_full^N).  With eq = the eq weights of (gamma, gamma^2, ...,
// gamma^(2^(ell-1))), gamma^1 the most significant bit, and each polynomial's
// blinding vectors:
//   m_eval = (1 + rho) <eq, m_even> - rho <eq, m_odd>,
//   g_t    = (1 + rho) <eq, g_hat_t>,
//   h      = m_eval + sum_t beta^(t+1) gamma^(2^t) g_t,
// stored as res[(g * npolys + i) * (mu + 2) + (0 | 1 + t | mu + 1)].
struct ZkGammaArgs {
    const ProofScalars* scb;
    const ZkScalars* zs;
    const u64* vecs;
    u64 omega_full, N;
    u32 depth, ell, npolys, mu;
    u64* res;
    u64* gx;    // [g * ell + b] = gamma_g^(2^b)
    u64* tpow;  // [g] = tau2^g
};
__global__ void k_zk_gamma(ZkGammaArgs a) {
    extern __shared__ u64 eq[];
    __shared__ u64 xs[32];
    __shared__ u64 dots[ZK_MAX_DOTS];
    const u32 g = blockIdx.x;
    const u32 i = g / a.depth, j = g % a.depth;
    const u64 half = 1ull << a.ell, P = half << 1;
    if (threadIdx.x == 0) {
        u64 x = gl_pow(a.omega_full, a.scb->indices[i] + (u64)j * a.N);
        for (u32 b = 0; b <= a.ell && b < 32; ++b) {
            xs[b] = x;
            if (b < a.ell) a.gx[(u64)g * a.ell + b] = x;
            x = gl_mul(x, x);
        }
        a.tpow[g] = gl_pow(a.zs->tau2, g);
    }
    __syncthreads();
    for (u64 jj = threadIdx.x; jj < half; jj += blockDim.x) {
        u64 e = 1;
        for (u32 b = 0; b < a.ell; ++b) {
            const u64 x = xs[b];
            e = gl_mul(e, ((jj >> (a.ell - 1 - b)) & 1) ? x : gl_sub(1, x));
        }
        eq[jj] = e;
    }
    __syncthreads();
    const u32 ndots = a.npolys * (a.mu + 2);
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (u32 d = warp; d < ndots; d += nwarps) {
        const u32 pi = d / (a.mu + 2), s = d % (a.mu + 2);
        const u64* vec = a.vecs + (u64)(pi * (a.mu + 1) + (s < 2 ? 0 : s - 1)) * P;
        const u32 odd = s == 1 ? 1 : 0;
        u64 acc = 0;
        for (u64 jj = lane; jj < half; jj += 32) acc = gl_add(acc, gl_mul(eq[jj], vec[2 * jj + odd]));
        acc = warp_sum_gl(acc);
        if (lane == 0) dots[d] = acc;
    }
    __syncthreads();
    if (threadIdx.x < a.npolys) {
        const u32 pi = threadIdx.x;
        const u64 rho = a.zs->rho, beta = a.zs->beta;
        const u64 onep = gl_add(1, rho);
        const u64* dd = dots + pi * (a.mu + 2);
        u64* out = a.res + ((u64)g * a.npolys + pi) * (a.mu + 2);
        const u64 m = gl_sub(gl_mul(onep, dd[0]), gl_mul(rho, dd[1]));
        out[0] = m;
        u64 h = m, bp = beta, gp = xs[0];
        for (u32 t = 0; t < a.mu; ++t) {
            const u64 gt = gl_mul(onep, dd[2 + t]);
            out[1 + t] = gt;
            h = gl_add(h, gl_mul(gl_mul(bp, gp), gt));
            bp = gl_mul(bp, beta);
            gp = gl_mul(gp, gp);
        }
        out[1 + a.mu] = h;
    }
}

// Batched beq covector (beq_weight_accum of evaluate_gamma_block): half
// entries acc[jj] = sum_g tau2^g eq_g[jj], split over gamma ranges (partials),
// then entries 2jj = (1 + rho) acc[jj] and 2jj + 1 = -rho acc[jj].
__global__ void k_zk_beq_partial(const u64* gx, const u64* tpow, u32 G, u32 ell, u32 chunk, u64* part) {
    const u64 half = 1ull << ell;
    const u64 jj = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= half) return;
    const u32 g0 = blockIdx.y * chunk, g1 = min(G, g0 + chunk);
    u64 acc = 0;
    for (u32 g = g0; g < g1; ++g) {
        const u64* x = gx + (u64)g * ell;
        u64 e = tpow[g];
        for (u32 b = 0; b < ell; ++b) e = gl_mul(e, ((jj >> (ell - 1 - b)) & 1) ? x[b] : gl_sub(1, x[b]));
        acc = gl_add(acc, e);
    }
    part[(u64)blockIdx.y * half + jj] = acc;
}
__global__ void k_zk_beq_final(const u64* part, u32 parts, u32 ell, const ZkScalars* zs, E3* out) {
    const u64 half = 1ull << ell;
    const u64 jj = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= half) return;
    u64 acc = 0;
    for (u32 k = 0; k < parts; ++k) acc = gl_add(acc, part[(u64)k * half + jj]);
    const u64 rho = zs->rho;
    out[2 * jj] = e3_base(gl_mul(gl_add(1, rho), acc));
    out[2 * jj + 1] = e3_base(gl_mul(gl_neg(rho), acc));
}

// Step 8 claims: claims[i * (mu + 2) + s] = sum_g tau2^g res[g][i][s], one
// CTA per claim (exact field sums: any order).
__global__ void k_zk_claims(const u64* res, const u64* tpow, u32 G, u32 ndots, u64* claims) {
    __shared__ u64 red[32];
    const u32 d = blockIdx.x;
    u64 acc = 0;
    for (u32 g = threadIdx.x; g < G; g += blockDim.x) acc = gl_add(acc, gl_mul(tpow[g], res[(u64)g * ndots + d]));
    acc = warp_sum_gl(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        u64 r = 0;
        for (u32 k = 0; k < (blockDim.x >> 5); ++k) r = gl_add(r, red[k]);
        claims[d] = r;
    }
}

// Step 9 (combine_claim_from_components, build_combined_and_subproof_claims,
// whir_zk_utils.hpp:455-520): tail = [m + 2 tau1 sum_t tau1^t g_t per
// polynomial, then the batched h claims]; the blinding proof's claims for its
// beq form (form 0) are [m, g_hat_0 .. g_hat_{mu-1}] per polynomial, one per
// blinding vector.  One warp.
__global__ void k_zk_combine(const ZkScalars* zs, const u64* claims, u32 npolys, u32 mu, ProofScalars* scg,
                             u64* tail) {
    if (threadIdx.x >= 32) return;
    const u32 l = threadIdx.x, stride = mu + 2;
    const u64 tau1 = zs->tau1;
    for (u32 pi = l; pi < npolys; pi += 32) {
        const u64* c = claims + pi * stride;
        u64 gs = 0, tp = 1;
        for (u32 s = 0; s < mu; ++s) {
            gs = gl_add(gs, gl_mul(tp, c[1 + s]));
            tp = gl_mul(tp, tau1);
        }
        tail[pi] = gl_add(c[0], gl_mul(gl_add(tau1, tau1), gs));
        tail[npolys + pi] = c[mu + 1];
    }
    for (u32 i = l; i < npolys * (mu + 1); i += 32) {
        const u32 pi = i / (mu + 1), s = i % (mu + 1);
        scg->forms_eval[i] = e3_base(claims[pi * stride + s]);
    }
}

u32 grid_for(u64 work, u32 threads) {
    return (u32)std::max<u64>(1, std::min<u64>((work + threads - 1) / threads, (u64)device_sms() * 16));
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// num_in_domain_queries (irs_commit.hpp:806-816).
double in_domain_queries(bool unique, double security, double rate) {
    const double slack = unique ? 0.0 : std::sqrt(rate) / 20.0;
    const double per = unique ? (1.0 + rate) / 2.0 : std::sqrt(rate) + slack;
    return std::ceil(security / (-std::log2(per)));
}

}  // namespace
}  // namespace wg

struct whirgpu_zk_witness {
    whirgpu_ctx* ctx = nullptr;
    whirgpu_transcript* tx = nullptr;
    whirgpu_zk_config cfg{};
    ProofPlan pb, pg;  // blinded (f_hat) and blinding inner proofs
    char* dev = nullptr;
    size_t off_b = 0, off_g = 0, off_tx = 0, off_zs = 0, off_narg = 0, off_hints = 0, off_rng = 0;
    size_t off_w = 0, off_e = 0, off_res = 0, off_gx = 0, off_tpow = 0, off_claims = 0, off_part = 0;
    size_t narg_cap = 0, hints_cap = 0, total = 0;
    u32 n = 0, ell = 0, npolys = 0, G = 0, parts = 0, chunk = 0;
    bool proved = false;
};

namespace wg {
whirgpu_zk_policy zk_default_policy(const whirgpu_params* p) {
    const double rate = std::pow(0.5, (double)p->starting_log_inv_rate);
    const bool ud = p->unique_decoding != 0;
    const uint64_t q1 = (uint64_t)in_domain_queries(ud, (double)(p->security_level - p->pow_bits), rate);
    const uint64_t q2 = (uint64_t)in_domain_queries(ud, (double)p->security_level, rate);
    return {q1, q2, q1, q2, 3};
}

void zk_detach_all(whirgpu_ctx* c) {
    std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
    for (whirgpu_zk_witness* w : c->live_zk) {
        if (w->dev) cudaFree(w->dev);
        w->dev = nullptr;
        w->ctx = nullptr;
    }
    c->live_zk.clear();
    for (auto& kv : c->zk_pool)
        for (char* p : kv.second) cudaFree(p);
    c->zk_pool.clear();
}
}  // namespace wg

namespace {
whirgpu_status zk_fail(whirgpu_ctx* c, whirgpu_status s, const std::string& m) { return wg::fail(c, s, m); }
#define ZK_CUDA(c, x, what)                                   \
    do {                                                      \
        cudaError_t _e = (x);                                 \
        if (_e != cudaSuccess) return wg::cuda_fail(c, _e, what); \
    } while (0)
}  // namespace

extern "C" {

whirgpu_status whirgpu_zk_config_from_params(const whirgpu_params* params, uint64_t n, uint64_t num_polynomials,
                                             const whirgpu_zk_policy* policy, whirgpu_zk_config* out) {
    if (!params || !out || num_polynomials == 0 || n >= 40 || params->batch_size != 1) return WHIRGPU_E_INVALID;
    std::memset(out, 0, sizeof(*out));
    whirgpu_status s = whirgpu_config_from_params(params, n, WHIRGPU_FIELD_GOLDILOCKS1, &out->blinded);
    if (s != WHIRGPU_OK) return s;
    const whirgpu_zk_policy pol = policy ? *policy : zk_default_policy(params);
    // from_params_with_policy (whir_zk.hpp:270-289)
    if (out->blinded.initial_sumcheck.num_rounds >= 40 || params->initial_folding_factor >= 40) return WHIRGPU_E_INVALID;
    const uint64_t k1 = 1ull << out->blinded.initial_sumcheck.num_rounds;
    const uint64_t k2 = 1ull << params->initial_folding_factor;
    const uint64_t leak = (pol.sumcheck_round_degree + 1) * n;
    const uint64_t q_ub = k1 * pol.q_delta_1 + k2 * pol.q_delta_2 + pol.t1 + pol.t2 + leak;
    uint64_t nbv = 0;
    while (nbv < 63 && (1ull << nbv) <= q_ub) ++nbv;
    if (nbv >= n || nbv == 0) return WHIRGPU_E_INVALID;  // the reference asserts num_blinding_vars < num_witness_vars
    whirgpu_params bp = *params;
    bp.batch_size = num_polynomials * (n + 1);
    s = whirgpu_config_from_params(&bp, nbv, WHIRGPU_FIELD_GOLDILOCKS1, &out->blinding);
    if (s != WHIRGPU_OK) return s;
    out->num_polynomials = num_polynomials;
    out->num_witness_variables = n;
    out->num_blinding_variables = nbv - 1;
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_deterministic_rng(whirgpu_ctx* c, const uint8_t seed[32], const char* domain, size_t domain_len,
                                         uint64_t first_word, uint64_t* out, size_t count) {
    if (!c || !seed || !out || (domain_len && !domain) || domain_len > ZK_RNG_MAX_DOMAIN)
        return zk_fail(c, WHIRGPU_E_INVALID, "bad argument");
    if (count == 0) return WHIRGPU_OK;
    const RngMsg msg = rng_message(seed, domain, domain_len);
    u64* d = nullptr;
    ZK_CUDA(c, cudaMalloc(&d, count * 8), "cudaMalloc");
    const u64 blocks = ((first_word + count + 3) >> 2) - (first_word >> 2);
    k_zk_rng<<<grid_for(blocks, 128), 128, 0, c->stream>>>(msg, first_word, count, d);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, count * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    if (e != cudaSuccess) return wg::cuda_fail(c, e, "deterministic rng");
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_zk_commit(whirgpu_ctx* c, const whirgpu_zk_config* cfg, const uint64_t* coeffs, int where,
                                 const uint8_t seed[32], const char* rng_domain, size_t rng_domain_len,
                                 whirgpu_transcript* tx, whirgpu_zk_witness** out) {
    if (!c || !cfg || !coeffs || !seed || !tx || !out || tx->ctx != c || (rng_domain_len && !rng_domain))
        return zk_fail(c, WHIRGPU_E_INVALID, "null argument");
    *out = nullptr;
    if (rng_domain_len > ZK_RNG_MAX_DOMAIN) return zk_fail(c, WHIRGPU_E_INVALID, "rng domain above 128 bytes");
    if (c->codeword_order != WHIRGPU_ORDER_NATURAL)
        return zk_fail(c, WHIRGPU_E_UNSUPPORTED, "zero-knowledge commitments use the natural codeword order");
    const uint64_t npolys = cfg->num_polynomials, n = cfg->num_witness_variables, ell = cfg->num_blinding_variables;
    if (cfg->blinded.field != WHIRGPU_FIELD_GOLDILOCKS1 || cfg->blinding.field != WHIRGPU_FIELD_GOLDILOCKS1)
        return zk_fail(c, WHIRGPU_E_INVALID, "zero-knowledge configs are over Identity<Goldilocks>");
    if (npolys == 0 || n == 0 || n >= 40 || ell + 1 >= n) return zk_fail(c, WHIRGPU_E_INVALID, "bad sizes");
    if (cfg->blinded.batch_size != 1 || cfg->blinding.batch_size != npolys * (n + 1))
        return zk_fail(c, WHIRGPU_E_INVALID, "batch sizes do not match the polynomial count");
    if (cfg->blinded.initial_committer.vector_size != (1ull << n) ||
        cfg->blinding.initial_committer.vector_size != (2ull << ell))
        return zk_fail(c, WHIRGPU_E_INVALID, "config sizes do not match the variable counts");
    if (npolys > (uint64_t)MAX_WITNESSES || npolys * (n + 1) > (uint64_t)MAX_VECTORS)
        return zk_fail(c, WHIRGPU_E_UNSUPPORTED, "more polynomials or blinding vectors than this path holds");
    if (ell > ZK_MAX_LOG_HALF) return zk_fail(c, WHIRGPU_E_UNSUPPORTED, "more than 2^15 blinding entries");
    if (cfg->blinded.num_rounds > WHIRGPU_MAX_ROUNDS || cfg->blinding.num_rounds > WHIRGPU_MAX_ROUNDS)
        return zk_fail(c, WHIRGPU_E_INVALID, "too many rounds");
    whirgpu_params hb{}, hg{};
    std::memcpy(hb.hash_id, cfg->blinded.hash_id, 32);
    std::memcpy(hg.hash_id, cfg->blinding.hash_id, 32);
    if (!engine_supported(&hb) || !engine_supported(&hg))
        return zk_fail(c, WHIRGPU_E_UNSUPPORTED, "only the BLAKE3 and SHA-2 engines are on this path");

    auto w = std::make_unique<whirgpu_zk_witness>();
    w->ctx = c;
    w->tx = tx;
    w->cfg = *cfg;
    w->n = (u32)n;
    w->ell = (u32)ell;
    w->npolys = (u32)npolys;
    const size_t ds_len = tx->ds.size();
    try {
        ProtocolParams ppb, ppg;
        ppb.batch_size = 1;
        ppb.hash = is_sha2(&hb) ? 1 : 0;
        ppb.field_degree = 1;
        ppg.batch_size = npolys * (n + 1);
        ppg.hash = is_sha2(&hg) ? 1 : 0;
        ppg.field_degree = 1;
        w->pb = make_plan(schedule_from_config(&cfg->blinded), ppb, MAX_FORMS, std::max<size_t>(ds_len, 96),
                          (uint32_t)npolys);
        w->pg = make_plan(schedule_from_config(&cfg->blinding), ppg, MAX_FORMS, 96, 1);
    } catch (const std::exception& e) {
        return zk_fail(c, WHIRGPU_E_INVALID, e.what());
    }
    const IrsSchedule& init = w->pb.sch.initial;
    if (init.in_domain * init.depth > (1ull << 20) || init.codeword_length * init.depth > (1ull << 32))
        return zk_fail(c, WHIRGPU_E_UNSUPPORTED, "coset domain too large");
    w->G = (u32)(init.in_domain * init.depth);
    const u64 half = 1ull << ell, P = half << 1, mu = n;
    const u32 bx = (u32)((half + 255) / 256);
    w->parts = std::max<u32>(1, std::min<u32>(w->G, 4 * device_sms() / bx));
    w->chunk = (w->G + w->parts - 1) / w->parts;
    w->parts = (w->G + w->chunk - 1) / w->chunk;
    const u64 V = npolys * (mu + 1);
    w->narg_cap = w->pb.narg_len + w->pg.narg_len + 8 * ((MAX_FORMS - 1) * V + (u64)w->G * npolys * (mu + 1) + 2 * npolys) + 64;
    w->hints_cap = 2 * w->pb.hints_cap + w->pg.hints_cap + 256;
    size_t cur = 0;
    auto take = [&cur](size_t bytes) {
        const size_t o = cur;
        cur = align_up(cur + bytes, 256);
        return o;
    };
    w->off_b = take(w->pb.total_bytes);
    w->off_g = take(w->pg.total_bytes);
    w->off_tx = take(sizeof(TxState));
    w->off_zs = take(sizeof(ZkScalars));
    w->off_narg = take(w->narg_cap + 64);
    w->off_hints = take(w->hints_cap + 64);
    const u64 per_poly = (mu + 2) * half;
    w->off_rng = take(npolys * per_poly * 8);
    w->off_w = take((size_t)MAX_FORMS * P * sizeof(E3));
    w->off_e = take((size_t)MAX_FORMS * MAX_VECTORS * sizeof(E3));
    w->off_res = take((size_t)w->G * npolys * (mu + 2) * 8);
    w->off_gx = take((size_t)w->G * ell * 8 + 8);
    w->off_tpow = take((size_t)w->G * 8);
    w->off_claims = take((size_t)(ZK_MAX_DOTS + 2 * MAX_WITNESSES) * 8);  // claims, then the combined / h tail
    w->off_part = take((size_t)w->parts * half * 8);
    const size_t total = cur;
    w->total = total;
    bool fresh = false;
    {  // a pooled allocation of this size, else a new one within the budget
        std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
        prepare_lde_tables(c, w->pb);
        prepare_lde_tables(c, w->pg);
        auto it = c->zk_pool.find(total);
        if (it != c->zk_pool.end() && !it->second.empty()) {
            w->dev = it->second.back();
            it->second.pop_back();
        } else {
            if (c->budget && c->allocated + total > c->budget) {
                for (auto& kv : c->zk_pool)
                    for (char* p : kv.second) {
                        cudaFree(p);
                        c->allocated -= std::min<uint64_t>(c->allocated, kv.first);
                    }
                c->zk_pool.clear();
            }
            if (c->budget && c->allocated + total > c->budget)
                return zk_fail(c, WHIRGPU_E_OOM, "zero-knowledge witness above the HBM budget");
            fresh = true;
        }
    }
    if (fresh) {
        ZK_CUDA(c, cudaMalloc(&w->dev, total), "cudaMalloc zero-knowledge witness");
        std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
        c->allocated += total;
    }
    char* dev = w->dev;
    auto fail_free = [&](whirgpu_status s, const std::string& m) {
        std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
        c->zk_pool[total].push_back(w->dev);
        w->dev = nullptr;
        return zk_fail(c, s, m);
    };
    // Counters and tickets of both workspaces start at zero (they reset
    // themselves after use, as in the workspace cache).
    cudaError_t e = cudaMemsetAsync(dev + w->off_b + w->pb.off_sc_scratch, 0, w->pb.off_tx - w->pb.off_sc_scratch,
                                    c->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(dev + w->off_g + w->pg.off_sc_scratch, 0, w->pg.off_tx - w->pg.off_sc_scratch, c->stream);
    TxState* txs = reinterpret_cast<TxState*>(dev + w->off_tx);
    w->pb.tx_ext = txs;
    w->pg.tx_ext = txs;
    char* wsb = dev + w->off_b;
    char* wsg = dev + w->off_g;
    const size_t coeff_bytes = (size_t)npolys << (n + 3);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(wsb + w->pb.off_coeffs, coeffs, coeff_bytes,
                            where == WHIRGPU_INPUT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(wsb + w->pb.off_ds, tx->ds.data(), ds_len, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return fail_free(WHIRGPU_E_CUDA, std::string("input copy: ") + cudaGetErrorString(e));
    c->io_h2d = (where == WHIRGPU_INPUT_DEVICE ? 0 : coeff_bytes) + ds_len;
    c->io_d2h = 0;
    u64* R = reinterpret_cast<u64*>(dev + w->off_rng);
    const RngMsg msg = rng_message(seed, rng_domain, rng_domain_len);
    const u64 words = npolys * per_poly;
    k_zk_rng<<<grid_for((words + 3) / 4, 128), 128, 0, c->stream>>>(msg, 0, words, R);
    k_zk_mask<<<grid_for(npolys << n, 256), 256, 0, c->stream>>>(reinterpret_cast<u64*>(wsb + w->pb.off_coeffs), R,
                                                                   (u32)n, (u32)(ell + 1), (u32)npolys, per_poly);
    k_zk_layout<<<grid_for(V * P, 256), 256, 0, c->stream>>>(reinterpret_cast<u64*>(wsg + w->pg.off_coeffs), R,
                                                             (u32)(ell + 1), (u32)npolys, (u32)mu, per_poly);
    count_launches(3);
    if (launch_tx_init(txs, reinterpret_cast<const unsigned char*>(wsb + w->pb.off_ds), (u32)ds_len,
                       reinterpret_cast<unsigned char*>(dev + w->off_narg), w->narg_cap,
                       reinterpret_cast<unsigned char*>(dev + w->off_hints), w->hints_cap, plan_scalars(w->pb, wsb), 1,
                       c->stream) != 0 ||
        enqueue_commit(w->pb, wsb, (u32)ds_len, c->tw, c->stream, c->timer.get(), false) != 0 ||
        enqueue_commit(w->pg, wsg, (u32)ds_len, c->tw, c->stream, c->timer.get(), false) != 0) {
        cudaStreamSynchronize(c->stream);
        return fail_free(WHIRGPU_E_INVALID, "commit launch failed");
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaStreamSynchronize(c->stream);
        return fail_free(WHIRGPU_E_CUDA, std::string("commit kernels: ") + cudaGetErrorString(e));
    }
    {
        std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
        c->live_zk.insert(w.get());
    }
    tx->complete = false;
    *out = w.release();
    return WHIRGPU_OK;
}

whirgpu_status whirgpu_zk_prove(whirgpu_ctx* c, whirgpu_zk_witness* w, const whirgpu_linear_form* forms,
                                size_t num_forms, const uint64_t* evaluations, whirgpu_transcript* tx,
                                uint64_t* evaluation_point, uint64_t* rlc) {
    if (!c || !w || !tx || w->ctx != c || w->tx != tx || !w->dev) return zk_fail(c, WHIRGPU_E_INVALID, "bad handles");
    if (w->proved) return zk_fail(c, WHIRGPU_E_INVALID, "a zero-knowledge witness proves once");
    if (num_forms > (size_t)MAX_FORMS - 1 || (num_forms && (!forms || !evaluations)))
        return zk_fail(c, WHIRGPU_E_INVALID, "bad statement (at most 7 forms)");
    for (size_t f = 0; f < num_forms; ++f)
        if (!forms[f].data || forms[f].kind > WHIRGPU_FORM_COVECTOR) return zk_fail(c, WHIRGPU_E_INVALID, "bad linear form");
    const u32 n = w->n, ell = w->ell, npolys = w->npolys, mu = n;
    const u64 half = 1ull << ell, P = half << 1;
    const u32 V = npolys * (mu + 1);
    ProofPlan pb = w->pb, pg = w->pg;
    plan_set_forms(pb, (int)num_forms);
    plan_set_forms(pg, (int)num_forms + 1);
    char* dev = w->dev;
    char* wsb = dev + w->off_b;
    char* wsg = dev + w->off_g;
    ProofScalars* scb = plan_scalars(pb, wsb);
    ProofScalars* scg = plan_scalars(pg, wsg);
    TxState* txs = pb.tx_ext;
    ZkScalars* zs = reinterpret_cast<ZkScalars*>(dev + w->off_zs);
    E3* W = reinterpret_cast<E3*>(dev + w->off_w);
    E3* E = reinterpret_cast<E3*>(dev + w->off_e);
    const size_t cov_bytes = (size_t)24 << n;
    size_t host_dense = 0;
    for (size_t f = 0; f < num_forms; ++f)
        if (forms[f].kind == WHIRGPU_FORM_COVECTOR && forms[f].location != WHIRGPU_INPUT_DEVICE) ++host_dense;
    struct Tmp {
        void* p = nullptr;
        ~Tmp() { if (p) cudaFree(p); }
    } tmp;
    if (host_dense) ZK_CUDA(c, cudaMalloc(&tmp.p, host_dense * cov_bytes), "cudaMalloc covectors");
    ZkFoldArgs fa{};
    fa.nforms = (int)num_forms;
    fa.n = n;
    fa.logP = ell + 1;
    fa.out = W + P;  // form slot 0 holds the beq covector
    cudaError_t e = cudaSuccess;
    size_t slot = 0;  // io_h2d continues the commit's count
    for (size_t f = 0; f < num_forms && e == cudaSuccess; ++f) {
        if (forms[f].kind == WHIRGPU_FORM_MLE) {
            char* dst = wsb + pb.off_points + f * n * 24;
            e = cudaMemcpyAsync(dst, forms[f].data, n * 24, cudaMemcpyHostToDevice, c->stream);
            fa.mle[f] = reinterpret_cast<const E3*>(dst);
            c->io_h2d += n * 24;
            continue;
        }
        pb.dense_mask |= 1u << f;
        if (forms[f].location == WHIRGPU_INPUT_DEVICE) {
            pb.dense[f] = forms[f].data;
        } else {
            uint64_t* dst = reinterpret_cast<uint64_t*>(static_cast<char*>(tmp.p) + slot++ * cov_bytes);
            e = cudaMemcpyAsync(dst, forms[f].data, cov_bytes, cudaMemcpyHostToDevice, c->stream);
            pb.dense[f] = dst;
            c->io_h2d += cov_bytes;
        }
        fa.dense[f] = reinterpret_cast<const E3*>(pb.dense[f]);
    }
    if (e == cudaSuccess && num_forms) {
        e = cudaMemcpyAsync(&scb->forms_eval[0], evaluations, num_forms * npolys * 24, cudaMemcpyHostToDevice, c->stream);
        c->io_h2d += num_forms * npolys * 24;
    }
    if (e != cudaSuccess) return wg::cuda_fail(c, e, "statement upload");
    pg.dense_mask = (1u << (num_forms + 1)) - 1;
    for (size_t f = 0; f <= num_forms; ++f) pg.dense[f] = reinterpret_cast<const uint64_t*>(W + f * P);

    const u64* vecs = reinterpret_cast<const u64*>(wsg + pg.off_coeffs);
    const cudaStream_t st = c->stream;
    u32 launched = 0;
    if (num_forms) {
        k_zk_fold<<<grid_for(num_forms * P, 256), 256, 0, st>>>(fa);
        k_zk_dots<<<(u32)(num_forms * V), 256, 0, st>>>(W + P, vecs, ell + 1, V, E);
        launched += 2;
    }
    k_zk_tx_a<<<1, 32, 0, st>>>(txs, zs, E, (int)num_forms, V, npolys, mu, scb, scg);
    ++launched;
    {  // step 5: IrsConfig::open of the f_hat commitments (irs_commit.hpp:637-713)
        const IrsSchedule& init = pb.sch.initial;
        const CommitBuffers& cb = pb.commits[0];
        OpenArgs oa{};
        oa.tx = txs;
        oa.sc = scb;
        oa.planes = reinterpret_cast<const u64*>(wsb + cb.planes);
        oa.nodes = reinterpret_cast<const u32*>(wsb + cb.nodes);
        oa.nwit = npolys;
        oa.planes_stride = pb.init_planes_stride / 8;
        oa.nodes_stride = pb.init_nodes_stride / 4;
        oa.N = cb.N;
        oa.logN = cb.logN;
        oa.depth = cb.depth;
        oa.ncomp = cb.ncomp;
        oa.q = (u32)init.in_domain;
        oa.gen = 1;
        oa.stir = 0;
        if (launch_open(oa, st) != 0) return zk_fail(c, WHIRGPU_E_INVALID, "opening launch failed");
    }
    k_zk_taus<<<1, 32, 0, st>>>(txs, zs);
    ++launched;
    {
        const IrsSchedule& init = pb.sch.initial;
        ZkGammaArgs ga{};
        ga.scb = scb;
        ga.zs = zs;
        ga.vecs = vecs;
        ga.N = init.codeword_length;
        ga.depth = (u32)init.depth;
        ga.omega_full = gl_pow_host(7, (GL_P - 1) / (init.codeword_length * init.depth));
        ga.ell = ell;
        ga.npolys = npolys;
        ga.mu = mu;
        ga.res = reinterpret_cast<u64*>(dev + w->off_res);
        ga.gx = reinterpret_cast<u64*>(dev + w->off_gx);
        ga.tpow = reinterpret_cast<u64*>(dev + w->off_tpow);
        const size_t smem = half * 8;
        if (smem > 48 * 1024) ZK_CUDA(c, cudaFuncSetAttribute(k_zk_gamma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                      "shared memory");
        k_zk_gamma<<<w->G, 256, smem, st>>>(ga);
        const u32 bx = (u32)((half + 255) / 256);
        u64* part = reinterpret_cast<u64*>(dev + w->off_part);
        k_zk_beq_partial<<<dim3(bx, w->parts), 256, 0, st>>>(ga.gx, ga.tpow, w->G, ell, w->chunk, part);
        k_zk_beq_final<<<bx, 256, 0, st>>>(part, w->parts, ell, zs, W);
        const u32 ndots = npolys * (mu + 2);
        u64* claims = reinterpret_cast<u64*>(dev + w->off_claims);
        u64* tail = claims + ZK_MAX_DOTS;
        k_zk_claims<<<ndots, 256, 0, st>>>(ga.res, ga.tpow, w->G, ndots, claims);
        k_zk_combine<<<1, 32, 0, st>>>(zs, claims, npolys, mu, scg, tail);
        launched += 5;
        count_launches(launched);
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            cudaStreamSynchronize(st);
            return wg::cuda_fail(c, e, "zero-knowledge kernels");
        }
        // Steps 8-9 messages (whir_zk_impl.hpp:262-300): per gamma and
        // polynomial m_eval and the g_hat values, then the tail -- G * npolys *
        // (mu + 1) + 2 npolys words.  The sponge is sequential; the host CPU
        // absorbs this run several times faster than one GPU warp.
        const size_t rows = (size_t)w->G * npolys, stride = mu + 2;
        const size_t add = 8 * (rows * (mu + 1) + 2 * npolys);
        const size_t need = sizeof(TxState) + rows * stride * 8 + 2 * npolys * 8 + add + 64;
        whirgpu_status ps = ensure_pinned(c, need);
        if (ps != WHIRGPU_OK) {
            cudaStreamSynchronize(st);
            return ps;
        }
        uint8_t* h = c->pinned;
        TxState* ht = reinterpret_cast<TxState*>(h);
        u64* hres = reinterpret_cast<u64*>(h + sizeof(TxState));
        u64* htail = hres + rows * stride;
        uint8_t* hbytes = reinterpret_cast<uint8_t*>(htail + 2 * npolys);
        ZK_CUDA(c, cudaMemcpyAsync(ht, txs, sizeof(TxState), cudaMemcpyDeviceToHost, st), "read-back");
        ZK_CUDA(c, cudaMemcpyAsync(hres, ga.res, rows * stride * 8, cudaMemcpyDeviceToHost, st), "read-back");
        ZK_CUDA(c, cudaMemcpyAsync(htail, tail, 2 * npolys * 8, cudaMemcpyDeviceToHost, st), "read-back");
        ZK_CUDA(c, cudaStreamSynchronize(st), "zero-knowledge steps");
        if (ht->err) {
            char buf[96];
            std::snprintf(buf, sizeof buf, "device error word 0x%x", ht->err);
            return zk_fail(c, WHIRGPU_E_DEVICE, buf);
        }
        if (ht->narg_len + add > ht->narg_cap) return zk_fail(c, WHIRGPU_E_DEVICE, "proof stream overflow");
        size_t pos = 0;
        ht->has_reader = 0;  // an absorb drops the pending squeeze reader
        for (size_t r = 0; r < rows; ++r)
            host_absorb_message_words(ht->hasher, ht->hpos, hres + r * stride, mu + 1, hbytes, pos);
        host_absorb_message_words(ht->hasher, ht->hpos, htail, 2 * npolys, hbytes, pos);
        ZK_CUDA(c, cudaMemcpyAsync(dev + w->off_narg + ht->narg_len, hbytes, add, cudaMemcpyHostToDevice, st),
                "transcript upload");
        ht->narg_len += add;
        ZK_CUDA(c, cudaMemcpyAsync(txs, ht, sizeof(TxState), cudaMemcpyHostToDevice, st), "transcript upload");
        c->io_d2h += sizeof(TxState) + rows * stride * 8 + 2 * npolys * 8;
        c->io_h2d += sizeof(TxState) + add;
    }
    if (enqueue_prove(pb, wsb, c->tw, st, c->timer.get()) != 0 || enqueue_prove(pg, wsg, c->tw, st, c->timer.get()) != 0) {
        cudaStreamSynchronize(st);
        return zk_fail(c, WHIRGPU_E_INVALID, "prove launch failed");
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        return wg::cuda_fail(c, e, "prove kernels");
    }
    w->proved = true;
    TxState htx;
    ZK_CUDA(c, cudaMemcpyAsync(&htx, txs, sizeof(TxState), cudaMemcpyDeviceToHost, st), "read-back");
    ZK_CUDA(c, cudaStreamSynchronize(st), "prove");
    if (c->timer) c->timer->harvest();
    if (htx.err) {
        char buf[96];
        std::snprintf(buf, sizeof buf, "device error word 0x%x", htx.err);
        return zk_fail(c, WHIRGPU_E_DEVICE, buf);
    }
    if (htx.narg_len > w->narg_cap || htx.hints_len > w->hints_cap)
        return zk_fail(c, WHIRGPU_E_DEVICE, "proof stream length mismatch");
    tx->narg.resize(htx.narg_len);
    tx->hints.resize(htx.hints_len);
    if (htx.narg_len)
        ZK_CUDA(c, cudaMemcpyAsync(tx->narg.data(), dev + w->off_narg, htx.narg_len, cudaMemcpyDeviceToHost, st), "read-back");
    if (htx.hints_len)
        ZK_CUDA(c, cudaMemcpyAsync(tx->hints.data(), dev + w->off_hints, htx.hints_len, cudaMemcpyDeviceToHost, st),
                "read-back");
    // FinalClaim of the blinded proof: its folding randomness and constraint RLC
    if (evaluation_point)
        ZK_CUDA(c, cudaMemcpyAsync(evaluation_point, &scb->sc_r[0], pb.total_sumcheck_rounds * 24,
                                   cudaMemcpyDeviceToHost, st), "read-back");
    if (rlc && num_forms)
        ZK_CUDA(c, cudaMemcpyAsync(rlc, &scb->crlc[0], num_forms * 24, cudaMemcpyDeviceToHost, st), "read-back");
    ZK_CUDA(c, cudaStreamSynchronize(st), "read-back");
    c->io_d2h += sizeof(TxState) + htx.narg_len + htx.hints_len;
    tx->complete = true;
    return WHIRGPU_OK;
}

void whirgpu_zk_witness_destroy(whirgpu_zk_witness* w) {
    if (!w) return;
    if (w->ctx) {
        whirgpu_ctx* c = w->ctx;
        cudaStreamSynchronize(c->stream);
        std::lock_guard<std::recursive_mutex> lk(c->cache_mu);
        if (w->dev) c->zk_pool[w->total].push_back(w->dev);  // kept for the next witness of this shape
        c->live_zk.erase(w);
    }
    delete w;
}

}  // extern "C"
