// k_ntt.cu -- Reed-Solomon encoder: batched Goldilocks NTT / low-degree extension.
//
// Computes, for every interleaved block b (and every Ext3 component c) of the
// committed vector, the codeword
//     X_{c,b}[i] = sum_{j < m} x_c[b*m + j] * w_N^(i*j),   i = 0 .. N-1,
// in natural order -- the reference's zero-pad + NTT of
// cpp/include/whir/algebra/ntt/mod_ntt.hpp:49-130 with the roots of
// cooley_tukey_goldilocks.hpp:24-47 (w_N = 7^((p-1)/N)).
//
// B200 design: an N-point transform is split four-step style into at most three
// passes of radix <= 2^11.  Each pass is one kernel over all planes
// (blockIdx.y = plane): a CTA stages a tile of W columns x R rows in shared
// memory, runs W independent R-point radix-2 DIT transforms there, applies
// the inter-pass twiddle and writes the tile back.  The first pass reads the
// *compact* message (the zero padding is never materialised, so an expansion-e
// LDE reads m = N/e words per plane), the last pass writes the codeword planes
// M[plane][i] that the leaf hasher and the opener read.
#include <algorithm>
#include <map>
#include <mutex>

#include "launch.h"
#include "gl.cuh"

namespace wg {

__device__ __forceinline__ u32 bitrev(u32 j, u32 bits) { return bits ? (__brev(j) >> (32 - bits)) : 0; }

// Shared-memory word of column element e: one pad word every 32 words keeps
// strided group accesses off a single bank; the extra word per column puts the
// W columns of a tile on different banks (the transposed store phase reads
// one element of each column per step).
__device__ __forceinline__ u32 pidx(u32 e) { return e + (e >> 5); }
__host__ __device__ __forceinline__ u32 col_stride(u32 logR) { return (1u << logR) + ((1u << logR) >> 5) + 1; }

// Stages s0+1 .. s0+RR of a radix-2 DIT on W bit-reversed columns of 2^L
// words, done as independent radix-2^RR groups in registers: a group is the
// 2^RR elements base + j 2^s0 (j < 2^RR) of one column, and the butterflies of
// stage s pair j with j + 2^(t-1) (t = s - s0) under the twiddle
// w_{2^s}^(lo + (j mod 2^(t-1)) 2^s0), lo = base mod 2^s0.
// S0ZERO: the group starts at stage 1 (s0 = 0), so lo = 0 and the butterflies
// with j mod 2^(t-1) = 0 have the twiddle w^0 = 1: their multiply is skipped
// (all of stage 1, half of stage 2, ...).
template <int RR, bool S0ZERO>
__device__ __forceinline__ void dit_group_pass(u64* sm, u32 W, u32 L, u32 s0, const u64* tws) {
    constexpr int G = 1 << RR;
    const u32 gpc_log = L - RR;  // groups per column (log2)
    const u32 total = W << gpc_log;
    const u32 cs = col_stride(L);
    for (u32 g = threadIdx.x; g < total; g += blockDim.x) {
        const u32 w = g >> gpc_log;
        const u32 gb = g & ((1u << gpc_log) - 1);
        const u32 lo = S0ZERO ? 0u : (gb & ((1u << s0) - 1));
        const u32 base = S0ZERO ? (gb << RR) : lo + ((gb >> s0) << (s0 + RR));
        u64* col = sm + w * cs;
        u64 x[G];
#pragma unroll
        for (int j = 0; j < G; ++j) x[j] = col[pidx(base + ((u32)j << s0))];
#pragma unroll
        for (int t = 1; t <= RR; ++t) {
            const int half = 1 << (t - 1);
            const u32 sh = L - (s0 + t);
#pragma unroll
            for (int j = 0; j < G; ++j) {
                if (j & half) continue;
                const u64 u = x[j];
                u64 v;
                if (S0ZERO && (j & (half - 1)) == 0) {
                    v = x[j + half];
                } else {
                    const u64 tw = tws[(lo + ((u32)(j & (half - 1)) << s0)) << sh];
                    v = gl_mul(x[j + half], tw);
                }
                x[j] = gl_add(u, v);
                x[j + half] = gl_sub(u, v);
            }
        }
#pragma unroll
        for (int j = 0; j < G; ++j) col[pidx(base + ((u32)j << s0))] = x[j];
    }
}

// w_{2^logM}^e via the two-level table of w_{2^TW_LOG} powers.
__device__ __forceinline__ u64 twiddle(u64 e, u32 logM, const u64* hi, const u64* lo) {
    u64 E = (e & ((1ull << logM) - 1)) << (TW_LOG - logM);
    return gl_mul(hi[E >> TW_HALF], lo[E & ((1ull << TW_HALF) - 1)]);
}

// One pass over all planes (blockIdx.y = plane).  MINB = CTAs per SM the
// register allocation is sized for (the pass plan picks the variant).
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_ntt_pass(NttPassArgs a) {
    extern __shared__ u64 sm[];
    const u32 logR = a.logR, R = 1u << logR, W = 1u << a.logW, halfR = R >> 1;
    const u32 tileN = W << logR;
    const u32 cs = col_stride(logR);
    u64* tws = sm + W * cs;
    const u32 plane = blockIdx.y;
    const u64 N = 1ull << a.logN;
    const bool first = a.pass == 0, last = a.pass + 1 == a.npass;
    const u32 comp = plane / a.depth, blk = plane % a.depth;
    const u64* src0 = comp == 0 ? a.src[0] : (comp == 1 ? a.src[1] : a.src[2]);  // no dynamic param indexing
    const u64* src = first ? src0 + (u64)blk * a.m : nullptr;
    u64* tmp = a.tmp + (u64)plane * N;

    for (u32 u = threadIdx.x; u < halfR; u += blockDim.x) tws[u] = a.tw_stage[u << (TW_STAGE_LOG - logR)];

    // Tile geometry.
    u64 S = 0, P = 0, col0 = 0;
    u64 i0base = 0;  // last pass: output index of (w = 0, i = 0)
    u32 i1 = 0;
    if (!last) {
        S = 1ull << a.logS;
        const u64 ngroups = S >> a.logW;
        P = blockIdx.x / ngroups;
        col0 = (blockIdx.x % ngroups) << a.logW;
    } else if (a.npass == 2) {
        i0base = (u64)blockIdx.x << a.logW;
    } else if (a.npass == 3) {
        const u32 groups = (1u << a.logR0) >> a.logW;
        i1 = blockIdx.x / groups;
        i0base = (u64)(blockIdx.x % groups) << a.logW;
    }

    // Load (bit-reversed within each column).  Only the first R >> logE rows of
    // a column can be nonzero (zero padding of the message); in bit-reversed
    // order they land on multiples of E, and the first logE DIT stages would
    // merely copy each of them over its block of E words -- done here as a
    // broadcast, the butterflies then start at stage logE.
    const u32 logE = a.logE, E = 1u << logE;
    const u32 mrows_log = logR - logE;
    if (!last) {
        // Thread t always serves column w = t mod W; its rows advance by J.
        const u32 w = threadIdx.x & (W - 1), J = blockDim.x >> a.logW;
        const u32 nrows = 1u << mrows_log;
        u64* col = sm + w * cs;
        if (first) {
            const u64 stride = (u64)J * S;
            u64 idx = (u64)(threadIdx.x >> a.logW) * S + col0 + w;
#pragma unroll 4
            for (u32 j = threadIdx.x >> a.logW; j < nrows; j += J, idx += stride)
                col[pidx(bitrev(j, logR))] = idx < a.m ? src[idx] : 0;
        } else {
            const u64 stride = (u64)J * S;
            const u64* p = tmp + (P * R + (threadIdx.x >> a.logW)) * S + col0 + w;
#pragma unroll 4
            for (u32 j = threadIdx.x >> a.logW; j < nrows; j += J, p += stride) col[pidx(bitrev(j, logR))] = *p;
        }
    } else {
        const u32 n = W << mrows_log;
#pragma unroll 4
        for (u32 e = threadIdx.x; e < n; e += blockDim.x) {
            const u32 w = e >> mrows_log, j = e & ((1u << mrows_log) - 1);
            u64 v;
            if (first) {
                v = j < a.m ? src[j] : 0;
            } else {
                const u64 i0 = i0base + w;
                const u64 row = a.npass == 2 ? i0 : (i0 << a.logR1) + i1;
                v = tmp[(row << logR) + j];
            }
            sm[w * cs + pidx(bitrev(j, logR))] = v;
        }
    }
    __syncthreads();
    if (logE) {
        const u32 nblk = W << mrows_log;  // blocks of E words, head at a multiple of E
        if (E >= 8 && nblk >= blockDim.x) {
            for (u32 b = threadIdx.x; b < nblk; b += blockDim.x) {
                u64* col = sm + (b >> mrows_log) * cs;
                const u32 p0 = (b & ((1u << mrows_log) - 1)) << logE;
                const u64 v = col[pidx(p0)];
                for (u32 k = 1; k < E; ++k) col[pidx(p0 + k)] = v;
            }
        } else {
            for (u32 e = threadIdx.x; e < tileN; e += blockDim.x) {
                const u32 w = e >> logR, p = e & (R - 1);
                if (p & (E - 1)) sm[w * cs + pidx(p)] = sm[w * cs + pidx(p & ~(E - 1))];
            }
        }
        __syncthreads();
    }

    // Decimation-in-time stages in register groups of up to 16, natural-order output.
    for (u32 s0 = logE; s0 < logR;) {
        const u32 left = logR - s0;
        const u32 rr = left >= 8 ? 4 : (left > 4 ? (left + 1) / 2 : left);
        if (s0 == 0) {
            if (rr == 4) dit_group_pass<4, true>(sm, W, logR, s0, tws);
            else if (rr == 3) dit_group_pass<3, true>(sm, W, logR, s0, tws);
            else if (rr == 2) dit_group_pass<2, true>(sm, W, logR, s0, tws);
            else dit_group_pass<1, true>(sm, W, logR, s0, tws);
        } else {
            if (rr == 4) dit_group_pass<4, false>(sm, W, logR, s0, tws);
            else if (rr == 3) dit_group_pass<3, false>(sm, W, logR, s0, tws);
            else if (rr == 2) dit_group_pass<2, false>(sm, W, logR, s0, tws);
            else dit_group_pass<1, false>(sm, W, logR, s0, tws);
        }
        s0 += rr;
        __syncthreads();
    }

    // Store.
    if (!last) {
        // Inter-pass twiddle w_{Ns}^(col i): thread t keeps col fixed and steps i
        // by J, so the twiddle advances by the constant factor w_{Ns}^(col J).
        const u32 logNs = logR + a.logS;  // size of the sub-transform this pass belongs to
        const u32 w = threadIdx.x & (W - 1), J = blockDim.x >> a.logW;
        const u64 col = col0 + w;
        u32 i = threadIdx.x >> a.logW;
        u64 tw = twiddle(col * i, logNs, a.tw_hi, a.tw_lo);
        const u64 step = twiddle(col * J, logNs, a.tw_hi, a.tw_lo);
        const u64 stride = (u64)J * S;
        u64* dst = tmp + (P * R + i) * S + col;
        const u64* scol = sm + w * cs;
#pragma unroll 2
        for (; i < R; i += J, dst += stride) {
            *dst = gl_mul(scol[pidx(i)], tw);
            tw = gl_mul(tw, step);
        }
    } else {
        u64* out = a.out + (u64)plane * N;
        const u64 outer = N >> logR;
        const u64 obase = a.npass == 3 ? i0base + ((u64)i1 << a.logR0) : i0base;
        const u32 w = threadIdx.x & (W - 1), J = blockDim.x >> a.logW;
        const u64* scol = sm + w * cs;
        u32 i = threadIdx.x >> a.logW;
        u64* dst = out + obase + w + outer * i;
        const u64 stride = outer * J;
#pragma unroll 4
        for (; i < R; i += J, dst += stride) *dst = scol[pidx(i)];
    }
}

// ---------------------------------------------------------------------------
// Host side: pass planning and launch.
// ---------------------------------------------------------------------------
static u32 pick_w(u32 logR, u64 limit_log) {
    // Tile <= 8192 elements (64 KiB), at most 16 columns, never more than the
    // dimension being grouped.
    u32 lw = logR >= 13 ? 0 : 13 - logR;
    if (lw > 4) lw = 4;
    if (lw > limit_log) lw = (u32)limit_log;
    return lw;
}

LdePlan default_plan_lde(u32 logN) {
    LdePlan p{};
    p.logN = logN;
    p.logW[0] = p.logW[1] = p.logW[2] = LDE_W_AUTO;
    if (logN <= 11) {
        p.npass = 1;
        p.logR[0] = logN;
    } else if (logN <= 22) {
        p.npass = 2;
        p.logR[0] = logN - logN / 2;
        p.logR[1] = logN / 2;
    } else {
        p.npass = 3;
        u32 a = (logN + 2) / 3, b = (logN - a + 1) / 2;
        p.logR[0] = a;
        p.logR[1] = b;
        p.logR[2] = logN - a - b;
    }
    return p;
}

size_t lde_smem_bytes(u32 logR, u32 logW) {
    return ((size_t)(1u << logW) * col_stride(logR)) * 8 + ((size_t)1 << logR) / 2 * 8 + 16;
}
constexpr size_t LDE_SMEM_MAX = 100 * 1024;

// Columns per CTA of pass s: the plan's choice, or tile <= 8192 words with at
// most 16 columns; never more than the dimension being grouped.
static u32 pass_logW(const LdePlan& pl, u32 s, u32 logS) {
    if (pl.npass == 1) return 0;
    const u32 limit = s + 1 < pl.npass ? logS : pl.logR[0];
    const u32 w = pl.logW[s] == LDE_W_AUTO ? pick_w(pl.logR[s], limit) : pl.logW[s];
    return w > limit ? limit : w;
}

bool lde_plan_valid(const LdePlan& p) {
    if (p.npass < 1 || p.npass > 3 || p.logN > TW_LOG) return false;
    if (p.minb != 0 && (p.minb < 2 || p.minb > 4)) return false;
    u32 sum = 0;
    for (u32 s = 0; s < p.npass; ++s) {
        if (p.logR[s] < 1 || p.logR[s] > TW_STAGE_LOG) return false;
        sum += p.logR[s];
    }
    if (sum != p.logN) return false;
    u32 rest = p.logN;
    for (u32 s = 0; s < p.npass; ++s) {
        rest -= p.logR[s];
        if (p.logW[s] != LDE_W_AUTO && p.logW[s] > 6) return false;  // blockDim (256) must be a multiple of W
        if (lde_smem_bytes(p.logR[s], pass_logW(p, s, rest)) > LDE_SMEM_MAX) return false;
    }
    return true;
}

static std::mutex g_plan_mu;
static std::map<u32, LdePlan> g_plans;  // key logN << 8 | logX

void lde_install_plan(u32 logX, const LdePlan& p) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    const u32 key = p.logN << 8 | logX;
    if (p.npass == 0) g_plans.erase(key);
    else g_plans[key] = p;
}
void lde_clear_plans() {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plans.clear();
}
size_t lde_installed_plans(u32* keys, LdePlan* plans, size_t cap) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    size_t i = 0;
    for (const auto& kv : g_plans) {
        if (i < cap) {
            if (keys) keys[i] = kv.first;
            if (plans) plans[i] = kv.second;
        }
        ++i;
    }
    return i;
}

LdePlan plan_lde(u32 logN, u32 logX) {
    {
        std::lock_guard<std::mutex> lk(g_plan_mu);
        auto it = g_plans.find(logN << 8 | logX);
        if (it != g_plans.end()) return it->second;
    }
    return default_plan_lde(logN);
}

int launch_lde_plan(const LdeArgs& L, const LdePlan& pl, cudaStream_t st) {
    if (L.logN > TW_LOG || L.planes == 0 || pl.logN != L.logN || !lde_plan_valid(pl)) return -1;
    NttPassArgs a{};
    for (int c = 0; c < 3; ++c) a.src[c] = L.src[c];
    a.m = L.m;
    a.tmp = L.tmp;
    a.out = L.out;
    a.depth = L.depth;
    a.logN = L.logN;
    a.npass = pl.npass;
    a.logR0 = pl.logR[0];
    a.logR1 = pl.logR[1];
    a.tw_stage = L.tw_stage;
    a.tw_hi = L.tw_hi;
    a.tw_lo = L.tw_lo;
    u32 logrest = L.logN;
    for (u32 s = 0; s < pl.npass; ++s) {
        a.pass = s;
        a.logR = pl.logR[s];
        logrest -= a.logR;
        a.logS = logrest;
        a.logW = pass_logW(pl, s, a.logS);
        dim3 grid;
        if (s + 1 < pl.npass) {
            u64 prefixes = s == 0 ? 1 : (1ull << pl.logR[0]);
            grid = dim3((unsigned)(prefixes << (a.logS - a.logW)), L.planes);
        } else if (pl.npass == 1) {
            grid = dim3(1, L.planes);
        } else {
            u64 groups = (1ull << pl.logR[0]) >> a.logW;
            if (pl.npass == 3) groups <<= pl.logR[1];
            grid = dim3((unsigned)groups, L.planes);
        }
        // Nonzero rows of this pass: the input index is (..., j_s, rest) with
        // rest < S_s; the data can be nonzero only where the index is below
        // min(m, S_{s-1}) (pass 0: below m).
        {
            const u64 bound = s == 0 ? L.m : std::min<u64>(L.m, 1ull << (logrest + a.logR));
            const u64 S_s = 1ull << a.logS;
            u64 rows = (bound + S_s - 1) / S_s;
            if (rows < 1) rows = 1;
            u32 lr = 0;
            while ((1ull << lr) < rows) ++lr;
            a.logE = a.logR > lr ? a.logR - lr : 0;
        }
        size_t smem = lde_smem_bytes(a.logR, a.logW);
        const u32 mb = pl.minb ? pl.minb : LDE_MINB_DEFAULT;
        if (mb == 2) k_ntt_pass<2><<<grid, 256, smem, st>>>(a);
        else if (mb == 4) k_ntt_pass<4><<<grid, 256, smem, st>>>(a);
        else k_ntt_pass<3><<<grid, 256, smem, st>>>(a);
        count_launches(1);
    }
    return 0;
}

int launch_lde(const LdeArgs& L, cudaStream_t st) {
    u32 lm = 0;
    while ((1ull << lm) < L.m) ++lm;
    const u32 logX = L.logN > lm ? L.logN - lm : 0;
    return launch_lde_plan(L, plan_lde(L.logN, logX), st);
}

int lde_prepare() {
    for (auto f : {k_ntt_pass<2>, k_ntt_pass<3>, k_ntt_pass<4>})
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LDE_SMEM_MAX) != cudaSuccess)
            return -1;
    return 0;
}

}  // namespace wg
