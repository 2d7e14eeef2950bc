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
#include "launch.h"
#include "gl.cuh"

namespace wg {

__device__ __forceinline__ u32 bitrev(u32 j, u32 bits) { return bits ? (__brev(j) >> (32 - bits)) : 0; }

// w_{2^logM}^e via the two-level table of w_{2^TW_LOG} powers.
__device__ __forceinline__ u64 twiddle(u64 e, u32 logM, const u64* hi, const u64* lo) {
    u64 E = (e & ((1ull << logM) - 1)) << (TW_LOG - logM);
    return gl_mul(hi[E >> TW_HALF], lo[E & ((1ull << TW_HALF) - 1)]);
}

__global__ void __launch_bounds__(256) k_ntt_pass(NttPassArgs a) {
    extern __shared__ u64 sm[];
    const u32 logR = a.logR, R = 1u << logR, W = 1u << a.logW, halfR = R >> 1;
    const u32 tileN = W << logR;
    u64* tws = sm + tileN;
    const u32 plane = blockIdx.y;
    const u64 N = 1ull << a.logN;
    const bool first = a.pass == 0, last = a.pass + 1 == a.npass;
    const u32 comp = plane / a.depth, blk = plane % a.depth;
    const u64* src = first ? a.src[comp] + (u64)blk * a.m : nullptr;
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

    // Load (bit-reversed within each column).
    if (!last) {
        for (u32 e = threadIdx.x; e < tileN; e += blockDim.x) {
            const u32 w = e & (W - 1), j = e >> a.logW;
            u64 v;
            if (first) {
                const u64 idx = (u64)j * S + col0 + w;
                v = idx < a.m ? src[idx] : 0;
            } else {
                v = tmp[(P * R + j) * S + col0 + w];
            }
            sm[(w << logR) + bitrev(j, logR)] = v;
        }
    } else {
        for (u32 e = threadIdx.x; e < tileN; e += blockDim.x) {
            const u32 w = e >> logR, j = e & (R - 1);
            u64 v;
            if (first) {
                v = j < a.m ? src[j] : 0;
            } else {
                const u64 i0 = i0base + w;
                const u64 row = a.npass == 2 ? i0 : (i0 << a.logR1) + i1;
                v = tmp[(row << logR) + j];
            }
            sm[(w << logR) + bitrev(j, logR)] = v;
        }
    }
    __syncthreads();

    // Radix-2 decimation-in-time stages, natural-order output.
    for (u32 s = 1; s <= logR; ++s) {
        const u32 half = 1u << (s - 1);
        for (u32 b = threadIdx.x; b < (tileN >> 1); b += blockDim.x) {
            const u32 w = b >> (logR - 1), bb = b & (halfR - 1);
            const u32 k = bb & (half - 1), g = bb >> (s - 1);
            const u32 x0 = (g << s) + k, x1 = x0 + half;
            u64* col = sm + (w << logR);
            const u64 t = tws[k << (logR - s)];
            const u64 u = col[x0], v = gl_mul(col[x1], t);
            col[x0] = gl_add(u, v);
            col[x1] = gl_sub(u, v);
        }
        __syncthreads();
    }

    // Store.
    if (!last) {
        const u32 logNs = logR + a.logS;  // size of the sub-transform this pass belongs to
        for (u32 e = threadIdx.x; e < tileN; e += blockDim.x) {
            const u32 w = e & (W - 1), i = e >> a.logW;
            const u64 col = col0 + w;
            u64 v = sm[(w << logR) + i];
            v = gl_mul(v, twiddle(col * i, logNs, a.tw_hi, a.tw_lo));
            tmp[(P * R + i) * S + col] = v;
        }
    } else {
        u64* out = a.out + (u64)plane * N;
        const u64 outer = N >> logR;
        const u64 obase = a.npass == 3 ? i0base + ((u64)i1 << a.logR0) : i0base;
        for (u32 e = threadIdx.x; e < tileN; e += blockDim.x) {
            const u32 w = e & (W - 1), i = e >> a.logW;
            out[obase + w + outer * i] = sm[(w << logR) + i];
        }
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

LdePlan plan_lde(u32 logN) {
    LdePlan p{};
    p.logN = logN;
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

size_t lde_smem_bytes(u32 logR, u32 logW) { return ((size_t)(1u << logW) << logR) * 8 + ((size_t)1 << logR) / 2 * 8 + 16; }

int launch_lde(const LdeArgs& L, cudaStream_t st) {
    const LdePlan pl = plan_lde(L.logN);
    if (L.logN > TW_LOG || L.planes == 0) return -1;
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
        dim3 grid;
        if (s + 1 < pl.npass) {
            a.logW = pick_w(a.logR, a.logS);
            u64 prefixes = s == 0 ? 1 : (1ull << pl.logR[0]);
            grid = dim3((unsigned)(prefixes << (a.logS - a.logW)), L.planes);
        } else if (pl.npass == 1) {
            a.logW = 0;
            grid = dim3(1, L.planes);
        } else {
            a.logW = pick_w(a.logR, pl.logR[0]);
            u64 groups = (1ull << pl.logR[0]) >> a.logW;
            if (pl.npass == 3) groups <<= pl.logR[1];
            grid = dim3((unsigned)groups, L.planes);
        }
        size_t smem = lde_smem_bytes(a.logR, a.logW);
        k_ntt_pass<<<grid, 256, smem, st>>>(a);
        count_launches(1);
    }
    return 0;
}

int lde_prepare() {
    cudaError_t e = cudaFuncSetAttribute(k_ntt_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    return e == cudaSuccess ? 0 : -1;
}

}  // namespace wg
