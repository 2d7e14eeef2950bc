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
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include "launch.h"
#include "gl.cuh"

namespace wg {

__device__ __forceinline__ u32 bitrev(u32 j, u32 bits) { return bits ? (__brev(j) >> (32 - bits)) : 0; }

// Global words a pass only reads (the message, the previous pass's scratch,
// the inter-pass tables) go through the read-only path, so the compiler may
// issue a batch of them ahead of the stores that follow.
__device__ __forceinline__ u64 ldg64(const u64* p) { return __ldg(reinterpret_cast<const unsigned long long*>(p)); }
// Loads and stores of the load and store phases go in batches of NTT_BATCH
// per thread: all loads of a batch are in flight before the first store.
constexpr int NTT_BATCH = 8;
// 16-byte accesses to two adjacent words (tile columns w, w + 1 of one row, or
// words j, j + 1 of one scratch row): half the memory instructions for the
// same bytes.  Used when the pass's bases are 16-byte aligned (NttPassArgs::vec2).
constexpr int NTT_BATCH2 = NTT_BATCH / 2;
__device__ __forceinline__ ulonglong2 ldg128(const u64* p) { return __ldg(reinterpret_cast<const ulonglong2*>(p)); }
__device__ __forceinline__ ulonglong2 ld128(const u64* p) { return *reinterpret_cast<const ulonglong2*>(p); }
__device__ __forceinline__ void st128(u64* p, u64 x, u64 y) { *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(x, y); }

// Shared-memory word of column element e: one pad word every 32 words keeps
// strided group accesses off a single bank.
__device__ __forceinline__ u32 pidx(u32 e) { return e + (e >> 5); }
// Word of twiddle u in the shared table: bits 0-3 of u are XORed with bits
// 4-7 and 8-11.  A butterfly group's lanes read twiddles lo 2^d + K (16
// consecutive lo, one d per stage, K shared); for every d <= 8 the swizzle
// puts those 16 words on 16 distinct 8-byte bank pairs, where the plain
// layout put them on one (d >= 4).  The map is XOR-linear, so the
// swizzle of lo 2^d + K is the lanes' part XOR a compile-time constant.
__host__ __device__ constexpr u32 twz(u32 u) { return u ^ (((u >> 4) ^ (u >> 8)) & 15u); }
// Words per column of a tile of 2^logW columns: the padded column, rounded up
// to 16 / W (mod 16) words, so that in the phases where a half-warp reads or
// writes W columns x 16 / W rows its 16 words fall on 16 distinct 8-byte bank
// pairs.  (In the butterfly groups a warp stays within one column.)
__host__ __device__ constexpr u32 col_stride(u32 logR, u32 logW) {
    const u32 base = (1u << logR) + ((1u << logR) >> 5);
    const u32 c = logW >= 1 && logW <= 3 ? 16u >> logW : 1u;
    return base + (c + 16 - base % 16) % 16;
}

// Stages s0+1 .. s0+RR of a radix-2 DIT on the 2^logW bit-reversed columns of
// 2^L words, done as independent radix-2^RR groups in registers: a group is
// the 2^RR elements base + j 2^s0 (j < 2^RR) of one column, and the
// butterflies of stage s pair j with j + 2^(t-1) (t = s - s0) under the twiddle
// w_{2^s}^(lo + c 2^s0), c = j mod 2^(t-1), lo = base mod 2^s0.
//
// L is a compile-time constant, so the twiddle of (t, c), table entry
// (lo << (L - s0 - t)) + (c << (L - t)), is read at tws[P_t ^ twz(c << (L - t))]
// with P_t = twz(lo << (L - s0 - t)) computed once per stage.  Word j of
// the group sits at pidx(base) + j 2^s0 + floor(j 2^s0 / 32): the group's
// 2^(s0 + RR)-word span never straddles a pad word except at the multiples
// of 32 its own steps cross.  That offset is a compile-time constant when s0
// is (S0C >= 0: the first group of a column, s0 = 0, and the second, s0 = 4),
// a uniform stride for s0 >= 5, and computed per word only for 1 <= s0 <= 3.
// S0ZERO: the group starts at stage 1 (s0 = 0), so lo = 0 and the butterflies
// with c = 0 have the twiddle w^0 = 1: their multiply is skipped (all of stage
// 1, half of stage 2, ...).
template <int RR, bool S0ZERO, int L, int S0C = -1>
__device__ __forceinline__ void dit_group(u64* sm, u32 logW, u32 cs, u32 s0_rt, const u64* tws) {
    constexpr int G = 1 << RR;
    constexpr u32 gpc_log = L - RR;  // groups per column (log2)
    const u32 s0 = S0ZERO ? 0u : (S0C >= 0 ? (u32)S0C : s0_rt);
    const u32 total = 1u << (logW + gpc_log);
    const bool wide = !S0ZERO && S0C < 0 && s0 >= 5;
    constexpr u32 SC = S0C < 0 ? 0 : (u32)S0C;
    const u32 D = wide ? (1u << s0) + (1u << (s0 - 5)) : 0u;
    for (u32 g = threadIdx.x; g < total; g += blockDim.x) {
        const u32 w = g >> gpc_log;
        const u32 gb = g & ((1u << gpc_log) - 1);
        const u32 lo = S0ZERO ? 0u : (gb & ((1u << s0) - 1));
        const u32 base = S0ZERO ? (gb << RR) : lo + ((gb >> s0) << (s0 + RR));
        u64* col = sm + w * cs;
        u64* p0 = col + pidx(base);
        u64 x[G];
#pragma unroll
        for (int j = 0; j < G; ++j) {
            if (S0ZERO) x[j] = p0[j];
            else if (S0C >= 0) x[j] = p0[(j << SC) + ((j << SC) >> 5)];
            else if (wide) x[j] = p0[j * D];
            else x[j] = col[pidx(base + ((u32)j << s0))];
        }
        const u32 X = S0ZERO ? 0u : (lo << (L - s0));  // entry of (t, c) = (X >> t) | (c << (L - t))
#pragma unroll
        for (int t = 1; t <= RR; ++t) {
            const int half = 1 << (t - 1);
            const u32 Pt = twz(X >> t);
#pragma unroll
            for (int j = 0; j < G; ++j) {
                if (j & half) continue;
                const int c = j & (half - 1);
                const u64 u = x[j];
                u64 v;
                if (S0ZERO && c == 0) {
                    v = x[j + half];
                } else {
                    v = gl_mul_fma(x[j + half], tws[Pt ^ twz((u32)c << (L - t))]);
                }
                x[j] = gl_add(u, v);
                x[j + half] = gl_sub(u, v);
            }
        }
#pragma unroll
        for (int j = 0; j < G; ++j) {
            if (S0ZERO) p0[j] = x[j];
            else if (S0C >= 0) p0[(j << SC) + ((j << SC) >> 5)] = x[j];
            else if (wide) p0[j * D] = x[j];
            else col[pidx(base + ((u32)j << s0))] = x[j];
        }
    }
}

// Stages s0+1 .. L in register groups of up to 16, natural-order output.
template <int L>
__device__ __forceinline__ void dit_stages(u64* sm, u32 logW, u32 cs, u32 s0, const u64* tws) {
    while (s0 < (u32)L) {
        const u32 left = L - s0;
        const u32 rr = left >= 8 ? 4 : (left > 4 ? (left + 1) / 2 : left);
        if (s0 == 0) {
            if constexpr (L >= 4) { if (rr == 4) dit_group<4, true, L>(sm, logW, cs, s0, tws); }
            if constexpr (L >= 3) { if (rr == 3) dit_group<3, true, L>(sm, logW, cs, s0, tws); }
            if constexpr (L >= 2) { if (rr == 2) dit_group<2, true, L>(sm, logW, cs, s0, tws); }
            if (rr == 1) dit_group<1, true, L>(sm, logW, cs, s0, tws);
        } else if (s0 == 4) {
            if constexpr (L >= 8) { if (rr == 4) dit_group<4, false, L, 4>(sm, logW, cs, s0, tws); }
            if constexpr (L >= 7) { if (rr == 3) dit_group<3, false, L, 4>(sm, logW, cs, s0, tws); }
            if constexpr (L >= 6) { if (rr == 2) dit_group<2, false, L, 4>(sm, logW, cs, s0, tws); }
            if constexpr (L >= 5) { if (rr == 1) dit_group<1, false, L, 4>(sm, logW, cs, s0, tws); }
        } else {
            if constexpr (L >= 4) { if (rr == 4) dit_group<4, false, L>(sm, logW, cs, s0, tws); }
            if constexpr (L >= 3) { if (rr == 3) dit_group<3, false, L>(sm, logW, cs, s0, tws); }
            if constexpr (L >= 2) { if (rr == 2) dit_group<2, false, L>(sm, logW, cs, s0, tws); }
            if (rr == 1) dit_group<1, false, L>(sm, logW, cs, s0, tws);
        }
        s0 += rr;
        __syncthreads();
    }
}

// w_{2^logM}^e via the two-level table of w_{2^TW_LOG} powers.
__device__ __forceinline__ u64 twiddle(u64 e, u32 logM, const u64* hi, const u64* lo) {
    u64 E = (e & ((1ull << logM) - 1)) << (TW_LOG - logM);
    return gl_mul(hi[E >> TW_HALF], lo[E & ((1ull << TW_HALF) - 1)]);
}

// ---- one tile of one pass --------------------------------------------------
// A tile is 2^logW columns x 2^L rows of one plane: for a middle (or first)
// pass the columns col0 .. col0 + W - 1 of prefix P, for the last pass W
// consecutive rows of its sub-transforms.
struct TileGeom {
    u64 S, P, col0, i0base;
    u32 i1, plane;
    const u64* src;  // the plane's message block (first pass, coset form), else null
    u64* tmp;        // the plane's scratch
};

template <int L>
__device__ __forceinline__ TileGeom tile_geom(const NttPassArgs& a, u32 bx, u32 plane) {
    TileGeom g{};
    const u64 N = 1ull << a.logN;
    const bool first = a.pass == 0, last = a.pass + 1 == a.npass;
    const u32 comp = plane / a.depth, blk = plane % a.depth;
    const u64* src0 = comp == 0 ? a.src[0] : (comp == 1 ? a.src[1] : a.src[2]);  // no dynamic param indexing
    g.plane = plane;
    g.src = first || a.twist ? src0 + (u64)blk * a.m : nullptr;
    g.tmp = a.tmp + (u64)plane * N;
    if (!last) {
        g.S = 1ull << a.logS;
        const u64 ngroups = g.S >> a.logW;
        g.P = bx / ngroups;
        g.col0 = (bx % ngroups) << a.logW;
    } else if (a.npass == 2) {
        g.i0base = (u64)bx << a.logW;
    } else if (a.npass == 3) {
        const u32 groups = (1u << a.logR0) >> a.logW;
        g.i1 = bx / groups;
        g.i0base = (u64)(bx % groups) << a.logW;
    }
    return g;
}

// Load (bit-reversed within each column).  Only the first R >> logE rows of
// a column can be nonzero (zero padding of the message); in bit-reversed
// order they land on multiples of E, and the first logE DIT stages would
// merely copy each of them over its block of E words -- done by
// tile_broadcast, the butterflies then start at stage logE.
template <int L>
__device__ __forceinline__ void tile_load(const NttPassArgs& a, const TileGeom& g, u64* sm) {
    constexpr u32 logR = L;
    const u32 W = 1u << a.logW, cs = a.cs;
    const bool first = a.pass == 0, last = a.pass + 1 == a.npass;
    const u32 mrows_log = logR - a.logE;
    const u64 S = g.S, col0 = g.col0;
    if (!last) {
        // Thread t always serves column w = t mod W; its rows advance by J.
        const u32 w = threadIdx.x & (W - 1), J = blockDim.x >> a.logW;
        const u32 nrows = 1u << mrows_log, j0 = threadIdx.x >> a.logW;
        u64* col = sm + w * cs;
        // Row 0 of this column.  The scratch of a middle pass is rewritten in
        // place by this kernel, so it is read with plain loads.
        const u64* p = first ? g.src + col0 + w : g.tmp + g.P * (1ull << logR) * S + col0 + w;
        const bool full = nrows % (NTT_BATCH * J) == 0 && (!first || ((u64)nrows << a.logS) <= a.m);
        if (full && a.vec2 && a.logW >= 1) {
            // Column pairs (2 wp, 2 wp + 1): one 16-byte load per row; rows
            // advance by 2 J, so a batch of NTT_BATCH2 pairs covers the rows a
            // batch of NTT_BATCH words does.
            const u32 wp = threadIdx.x & ((W >> 1) - 1), J2 = blockDim.x >> (a.logW - 1);
            const u32 jp0 = threadIdx.x >> (a.logW - 1);
            u64* c0 = sm + 2 * wp * cs;
            const u64* p2 = first ? g.src + col0 + 2 * wp : g.tmp + g.P * (1ull << logR) * S + col0 + 2 * wp;
            for (u32 jb = jp0; jb < nrows; jb += NTT_BATCH2 * J2) {
                ulonglong2 v[NTT_BATCH2];
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b) {
                    const u64* q = p2 + (u64)(jb + b * J2) * S;
                    v[b] = first ? ldg128(q) : ld128(q);
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b) {
                    const u32 r = pidx(bitrev(jb + b * J2, logR));
                    c0[r] = v[b].x;
                    c0[cs + r] = v[b].y;
                }
            }
        } else if (full && first) {
            for (u32 jb = j0; jb < nrows; jb += NTT_BATCH * J) {
                u64 v[NTT_BATCH];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) v[b] = ldg64(p + (u64)(jb + b * J) * S);
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) col[pidx(bitrev(jb + b * J, logR))] = v[b];
            }
        } else if (full) {
            for (u32 jb = j0; jb < nrows; jb += NTT_BATCH * J) {
                u64 v[NTT_BATCH];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) v[b] = p[(u64)(jb + b * J) * S];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) col[pidx(bitrev(jb + b * J, logR))] = v[b];
            }
        } else {
            for (u32 jb = j0; jb < nrows; jb += NTT_BATCH * J) {
                u64 v[NTT_BATCH];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) {
                    const u32 j = jb + b * J;
                    const u64 idx = (u64)j * S;
                    v[b] = j >= nrows || (first && idx + col0 + w >= a.m) ? 0 : first ? ldg64(p + idx) : p[idx];
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) {
                    const u32 j = jb + b * J;
                    if (j < nrows) col[pidx(bitrev(j, logR))] = v[b];
                }
            }
        }
    } else {
        const u32 n = W << mrows_log, jmask = (1u << mrows_log) - 1;
        if (!first && !a.twist && a.vec2 && mrows_log >= 1 && n % (NTT_BATCH * blockDim.x) == 0) {
            // The previous pass's rows by word pairs (j, j + 1), j even: one
            // 16-byte load; in bit-reversed order j + 1 lands R / 2 after j.
            for (u32 eb = threadIdx.x; 2 * eb < n; eb += NTT_BATCH2 * blockDim.x) {
                ulonglong2 v[NTT_BATCH2];
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b) {
                    const u32 e = 2 * (eb + b * blockDim.x);
                    const u64 i0 = g.i0base + (e >> mrows_log);
                    const u64 row = a.npass == 2 ? i0 : (i0 << a.logR1) + g.i1;
                    v[b] = ldg128(g.tmp + (row << logR) + (e & jmask));
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b) {
                    const u32 e = 2 * (eb + b * blockDim.x);
                    u64* c = sm + (e >> mrows_log) * cs;
                    const u32 r = bitrev(e & jmask, logR);
                    c[pidx(r)] = v[b].x;
                    c[pidx(r + (1u << (logR - 1)))] = v[b].y;
                }
            }
        } else if (!first && !a.twist && n % (NTT_BATCH * blockDim.x) == 0) {
            // The previous pass's rows, whole batches.
            for (u32 eb = threadIdx.x; eb < n; eb += NTT_BATCH * blockDim.x) {
                u64 v[NTT_BATCH];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) {
                    const u32 e = eb + b * blockDim.x;
                    const u64 i0 = g.i0base + (e >> mrows_log);
                    const u64 row = a.npass == 2 ? i0 : (i0 << a.logR1) + g.i1;
                    v[b] = ldg64(g.tmp + (row << logR) + (e & jmask));
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) {
                    const u32 e = eb + b * blockDim.x;
                    sm[(e >> mrows_log) * cs + pidx(bitrev(e & jmask, logR))] = v[b];
                }
            }
        } else {
            for (u32 eb = threadIdx.x; eb < n; eb += NTT_BATCH * blockDim.x) {
                u64 v[NTT_BATCH];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) {
                    const u32 e = eb + b * blockDim.x;
                    const u32 w = e >> mrows_log, j = e & jmask;
                    v[b] = 0;
                    if (e >= n) continue;
                    if (first) {
                        if (j < a.m) v[b] = ldg64(g.src + j);
                    } else if (a.twist) {
                        // Pass 0 would have broadcast message word j over its
                        // column and scaled row `row` by w_N^(row j): done here.
                        const u64 row = g.i0base + w;
                        const u64 x = j < a.m ? ldg64(g.src + j) : 0;
                        v[b] = gl_mul_fma(x, a.tw_pass ? ldg64(a.tw_pass + (row << logR) + j)
                                                       : twiddle(row * j, a.logN, a.tw_hi, a.tw_lo));
                    } else {
                        const u64 i0 = g.i0base + w;
                        const u64 row = a.npass == 2 ? i0 : (i0 << a.logR1) + g.i1;
                        v[b] = ldg64(g.tmp + (row << logR) + j);
                    }
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) {
                    const u32 e = eb + b * blockDim.x;
                    if (e < n) sm[(e >> mrows_log) * cs + pidx(bitrev(e & jmask, logR))] = v[b];
                }
            }
        }
    }
}

// The same loads as asynchronous global -> shared copies (cp.async, 8 bytes
// each; a word past the message is zero-filled with no read).  Used by the
// pipelined kernel, which issues a tile's copies while the previous tile is
// transformed.  Not for the coset-form last pass (its words are products).
__device__ __forceinline__ void cp_async8(u64* sdst, const u64* gsrc, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int L>
__device__ __forceinline__ void tile_load_async(const NttPassArgs& a, const TileGeom& g, u64* sm) {
    constexpr u32 logR = L;
    const u32 W = 1u << a.logW, cs = a.cs;
    const bool first = a.pass == 0, last = a.pass + 1 == a.npass;
    const u32 mrows_log = logR - a.logE;
    if (!last) {
        const u32 w = threadIdx.x & (W - 1), J = blockDim.x >> a.logW;
        const u32 nrows = 1u << mrows_log;
        u64* col = sm + w * cs;
        const u64* p = first ? g.src + g.col0 + w : g.tmp + g.P * (1ull << logR) * g.S + g.col0 + w;
        for (u32 j = threadIdx.x >> a.logW; j < nrows; j += J) {
            const u64 idx = (u64)j * g.S;
            const bool valid = !first || idx + g.col0 + w < a.m;
            // A zero-filled word reads nothing; its source operand is still the
            // plane's first word (column col0 + w itself may lie past the message).
            cp_async8(col + pidx(bitrev(j, logR)), valid ? p + idx : (first ? g.src : p), valid);
        }
    } else {
        const u32 n = W << mrows_log, jmask = (1u << mrows_log) - 1;
        for (u32 e = threadIdx.x; e < n; e += blockDim.x) {
            const u32 w = e >> mrows_log, j = e & jmask;
            u64* d = sm + w * cs + pidx(bitrev(j, logR));
            if (first) {
                cp_async8(d, j < a.m ? g.src + j : g.src, j < a.m);
            } else {
                const u64 i0 = g.i0base + w;
                const u64 row = a.npass == 2 ? i0 : (i0 << a.logR1) + g.i1;
                cp_async8(d, g.tmp + (row << logR) + j, true);
            }
        }
    }
}

// Copies each loaded head over its block of E = 2^logE words (the first logE
// stages of the zero-padded transform), then synchronises.
template <int L>
__device__ __forceinline__ void tile_broadcast(const NttPassArgs& a, u64* sm) {
    constexpr u32 logR = L, R = 1u << L;
    const u32 logE = a.logE, E = 1u << logE, cs = a.cs;
    if (!logE) return;
    const u32 W = 1u << a.logW, tileN = W << logR;
    const u32 mrows_log = logR - logE;
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

// Store: middle passes scale by the inter-pass factor and write the scratch
// in place; the last pass writes the codeword plane transposed.
template <int L>
__device__ __forceinline__ void tile_store(const NttPassArgs& a, const TileGeom& g, const u64* sm) {
    constexpr u32 logR = L, R = 1u << L;
    const u32 W = 1u << a.logW, cs = a.cs;
    const bool last = a.pass + 1 == a.npass;
    const u64 N = 1ull << a.logN;
    if (!last) {
        // Inter-pass twiddle w_{Ns}^(col i) (Ns: the sub-transform this pass
        // belongs to): read from the context's table, laid out like the tile
        // rows, or else generated -- thread t keeps col fixed and steps i by J,
        // so the factor advances by the constant w_{Ns}^(col J).
        const u64 S = g.S;
        const u32 w = threadIdx.x & (W - 1), J = blockDim.x >> a.logW;
        const u64 col = g.col0 + w;
        u32 i = threadIdx.x >> a.logW;
        const u64 stride = (u64)J * S;
        u64* dst = g.tmp + (g.P * R + i) * S + col;
        const u64* scol = sm + w * cs;
        if (a.tw_pass && a.vec2 && a.logW >= 1 && R % (NTT_BATCH * J) == 0) {
            // Column pairs: the factors and the scratch words of (2 wp, 2 wp + 1)
            // are adjacent, one 16-byte load and one 16-byte store per row.
            const u32 wp = threadIdx.x & ((W >> 1) - 1), J2 = blockDim.x >> (a.logW - 1);
            const u64 c2 = g.col0 + 2 * wp, stride2 = (u64)J2 * S;
            u32 i2 = threadIdx.x >> (a.logW - 1);
            u64* d2 = g.tmp + (g.P * R + i2) * S + c2;
            const u64* t2 = a.tw_pass + (u64)i2 * S + c2;
            const u64* s2 = sm + 2 * wp * cs;
            for (; i2 < R; i2 += NTT_BATCH2 * J2, d2 += NTT_BATCH2 * stride2, t2 += NTT_BATCH2 * stride2) {
                u64 x0[NTT_BATCH2], x1[NTT_BATCH2];
                ulonglong2 f[NTT_BATCH2];
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b) {
                    const u32 r = pidx(i2 + b * J2);
                    x0[b] = s2[r];
                    x1[b] = s2[cs + r];
                    f[b] = ldg128(t2 + b * stride2);
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b)
                    st128(d2 + b * stride2, gl_mul_fma(x0[b], f[b].x), gl_mul_fma(x1[b], f[b].y));
            }
        } else if (a.tw_pass && R % (NTT_BATCH * J) == 0) {
            const u64* tcol = a.tw_pass + (u64)i * S + col;
            for (; i < R; i += NTT_BATCH * J, dst += NTT_BATCH * stride, tcol += NTT_BATCH * stride) {
                u64 x[NTT_BATCH], f[NTT_BATCH];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) {
                    x[b] = scol[pidx(i + b * J)];
                    f[b] = ldg64(tcol + b * stride);
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) dst[b * stride] = gl_mul_fma(x[b], f[b]);
            }
        } else if (a.tw_pass) {
            const u64* tcol = a.tw_pass + (u64)i * S + col;
            for (; i < R; i += J, dst += stride, tcol += stride) *dst = gl_mul_fma(scol[pidx(i)], ldg64(tcol));
        } else {
            const u32 logNs = logR + a.logS;
            u64 tw = twiddle(col * i, logNs, a.tw_hi, a.tw_lo);
            const u64 step = twiddle(col * J, logNs, a.tw_hi, a.tw_lo);
#pragma unroll 2
            for (; i < R; i += J, dst += stride) {
                *dst = gl_mul(scol[pidx(i)], tw);
                tw = gl_mul(tw, step);
            }
        }
    } else {
        u64* out = a.out + (u64)g.plane * N;
        const u64 outer = N >> logR;
        const u64 obase = a.npass == 3 ? g.i0base + ((u64)g.i1 << a.logR0) : g.i0base;
        const u32 w = threadIdx.x & (W - 1), J = blockDim.x >> a.logW;
        const u64* scol = sm + w * cs;
        u32 i = threadIdx.x >> a.logW;
        u64* dst = out + obase + w + outer * i;
        const u64 stride = outer * J;
        if (a.vec2 && a.logW >= 1 && (outer & 1) == 0 && R % (NTT_BATCH * J) == 0) {
            // Column pairs: codeword words obase + 2 wp + outer i and the next
            // one, a 16-byte store (obase is a multiple of W, outer even).
            const u32 wp = threadIdx.x & ((W >> 1) - 1), J2 = blockDim.x >> (a.logW - 1);
            u32 i2 = threadIdx.x >> (a.logW - 1);
            const u64 stride2 = outer * J2;
            u64* d2 = out + obase + 2 * wp + outer * i2;
            const u64* s2 = sm + 2 * wp * cs;
            for (; i2 < R; i2 += NTT_BATCH2 * J2, d2 += NTT_BATCH2 * stride2) {
                u64 x0[NTT_BATCH2], x1[NTT_BATCH2];
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b) {
                    const u32 r = pidx(i2 + b * J2);
                    x0[b] = s2[r];
                    x1[b] = s2[cs + r];
                }
#pragma unroll
                for (int b = 0; b < NTT_BATCH2; ++b) st128(d2 + b * stride2, x0[b], x1[b]);
            }
        } else if (R % (NTT_BATCH * J) == 0) {
            for (; i < R; i += NTT_BATCH * J, dst += NTT_BATCH * stride) {
                u64 x[NTT_BATCH];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) x[b] = scol[pidx(i + b * J)];
#pragma unroll
                for (int b = 0; b < NTT_BATCH; ++b) dst[b * stride] = x[b];
            }
        } else {
            for (; i < R; i += J, dst += stride) *dst = scol[pidx(i)];
        }
    }
}

template <int L>
__device__ __forceinline__ void fill_twiddles(const NttPassArgs& a, u64* tws) {
    for (u32 u = threadIdx.x; u < (1u << L) / 2; u += blockDim.x) tws[twz(u)] = a.tw_stage[u << (TW_STAGE_LOG - L)];
}

// One pass over all planes, one tile per CTA (blockIdx.x = tile of the
// plane, blockIdx.y = plane).  MINB = CTAs per SM the register allocation is
// sized for (the pass plan picks the variant).
template <int MINB, int L>
__global__ void __launch_bounds__(256, MINB) k_ntt_pass(NttPassArgs a) {
    extern __shared__ u64 sm[];
    u64* tws = sm + (1u << a.logW) * a.cs;
    fill_twiddles<L>(a, tws);
    const TileGeom g = tile_geom<L>(a, blockIdx.x, blockIdx.y);
    tile_load<L>(a, g, sm);
    __syncthreads();
    tile_broadcast<L>(a, sm);
    // Decimation-in-time stages in register groups of up to 16, natural-order output.
    dit_stages<L>(sm, a.logW, a.cs, a.logE, tws);
    tile_store<L>(a, g, sm);
}

// The same pass as a persistent pipeline: each CTA walks tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... (tile = plane * tiles_per_plane +
// tile of the plane) with two tile buffers: the copies of the next tile are
// in flight (cp.async) while the current one is transformed and stored.  The
// stage twiddles are filled once per CTA.
template <int MINB, int L>
__global__ void __launch_bounds__(256, MINB) k_ntt_pipe(NttPassArgs a) {
    extern __shared__ u64 sm[];
    const u32 tile_words = (1u << a.logW) * a.cs;
    u64* tws = sm + 2 * tile_words;
    fill_twiddles<L>(a, tws);
    const u32 total = a.tiles_per_plane * a.planes;
    u32 tile = blockIdx.x;
    if (tile < total)
        tile_load_async<L>(a, tile_geom<L>(a, tile % a.tiles_per_plane, tile / a.tiles_per_plane), sm);
    cp_async_commit();
    for (u32 it = 0; tile < total; tile += gridDim.x, ++it) {
        u64* cur = (it & 1) ? sm + tile_words : sm;
        u64* nxt = (it & 1) ? sm : sm + tile_words;
        const u32 next = tile + gridDim.x;
        if (next < total)
            tile_load_async<L>(a, tile_geom<L>(a, next % a.tiles_per_plane, next / a.tiles_per_plane), nxt);
        cp_async_commit();
        cp_async_wait_prev();  // this tile's copies (all groups but the newest) have landed
        __syncthreads();
        tile_broadcast<L>(a, cur);
        dit_stages<L>(cur, a.logW, a.cs, a.logE, tws);
        tile_store<L>(a, tile_geom<L>(a, tile % a.tiles_per_plane, tile / a.tiles_per_plane), cur);
        __syncthreads();  // the buffer is refilled by the next iteration's copies
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

// Shared memory of a pass: the tile (two tiles when pipelined) and the twiddles.
size_t lde_smem_bytes(u32 logR, u32 logW, bool pipe = false) {
    return ((size_t)(1u << logW) * col_stride(logR, logW)) * 8 * (pipe ? 2 : 1) + ((size_t)1 << logR) / 2 * 8 + 16;
}
constexpr size_t LDE_SMEM_MAX = 100 * 1024, LDE_SMEM_PIPE_MAX = 200 * 1024;

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
    if (p.pipe > 1) return false;
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
        if (p.pipe && lde_smem_bytes(p.logR[s], pass_logW(p, s, rest), true) > LDE_SMEM_PIPE_MAX) return false;
    }
    return true;
}

static std::mutex g_plan_mu;
static std::map<u32, LdePlan> g_plans;  // key logN << 8 | logX
static std::atomic<u32> g_plan_epoch{0};

void lde_install_plan(u32 logX, const LdePlan& p) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    const u32 key = p.logN << 8 | logX;
    if (p.npass == 0) g_plans.erase(key);
    else g_plans[key] = p;
    ++g_plan_epoch;
}
void lde_clear_plans() {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plans.clear();
    ++g_plan_epoch;
}
u32 lde_plan_epoch() { return g_plan_epoch.load(); }
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

// The pass kernel for (CTAs per SM, log2 radix): one instantiation per radix
// 2^1 .. 2^TW_STAGE_LOG, so every index and stride of the stage groups is a
// compile-time constant.
typedef void (*NttPassKernel)(NttPassArgs);
template <int MINB, int... Ls>
static NttPassKernel pass_kernel_of(u32 l, bool pipe, std::integer_sequence<int, Ls...>) {
    static const NttPassKernel table[] = {k_ntt_pass<MINB, Ls + 1>...};
    static const NttPassKernel ptable[] = {k_ntt_pipe<MINB, Ls + 1>...};
    return pipe ? ptable[l - 1] : table[l - 1];
}
static NttPassKernel pass_kernel(u32 minb, u32 logR, bool pipe = false) {
    static_assert(TW_STAGE_LOG == 11, "one pass kernel per radix up to 2^TW_STAGE_LOG");
    const auto seq = std::make_integer_sequence<int, TW_STAGE_LOG>{};
    if (minb == 2) return pass_kernel_of<2>(logR, pipe, seq);
    if (minb == 4) return pass_kernel_of<4>(logR, pipe, seq);
    return pass_kernel_of<3>(logR, pipe, seq);
}

// Resident CTAs per SM of each pipelined kernel and tile width on this
// device (measured once by lde_prepare; sizes the persistent grids).
static std::mutex g_occ_mu;
static std::map<std::tuple<int, u32, u32, u32>, int> g_pipe_occ;  // (device, minb, logR, logW)
static int pipe_occupancy(u32 minb, u32 logR, u32 logW) {
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, minb, logR, logW);
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto it = g_pipe_occ.find(key);
    if (it != g_pipe_occ.end()) return it->second;
    int n = 0;
    const size_t smem = lde_smem_bytes(logR, logW, true);
    if (smem > LDE_SMEM_PIPE_MAX ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pass_kernel(minb, logR, true), 256, smem) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    g_pipe_occ[key] = n;
    return n;
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
    // Two passes where the message fits one row of the first (m <= 2^logR1):
    // every column of pass 0 holds at most one nonzero word, so pass 0 would
    // only broadcast it and apply the inter-pass factors.  The last pass then
    // reads the message and applies the factors itself (the coset form of the
    // LDE), and pass 0 is not launched.
    const bool twist = pl.npass == 2 && L.m <= (1ull << pl.logR[1]);
    a.planes = L.planes;
    // 16-byte word pairs need 16-byte aligned plane bases: the scratch and the
    // codeword (N >= 2 words a plane), and the message blocks (m even).
    auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    bool vec2 = al16(L.tmp) && al16(L.out) && L.m % 2 == 0 && L.logN >= 1 && L.depth > 0;
    for (u32 c = 0; L.depth > 0 && c < L.planes / L.depth && c < 3; ++c) vec2 = vec2 && al16(L.src[c]);
    u32 logrest = L.logN;
    for (u32 s = 0; s < pl.npass; ++s) {
        a.pass = s;
        a.logR = pl.logR[s];
        logrest -= a.logR;
        a.logS = logrest;
        if (twist && s == 0) continue;
        a.twist = twist ? 1u : 0u;
        a.logW = pass_logW(pl, s, a.logS);
        a.cs = col_stride(a.logR, a.logW);
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
        a.tw_pass = !L.tables ? nullptr
                    : s + 1 < pl.npass ? L.tables->get(a.logR + a.logS, a.logR)
                    : twist ? L.tables->get(L.logN, pl.logR[0]) : nullptr;
        a.vec2 = vec2 && (!a.tw_pass || al16(a.tw_pass)) ? 1u : 0u;
        const u32 mb = pl.minb ? pl.minb : LDE_MINB_DEFAULT;
        const int occ = pl.pipe && !twist ? pipe_occupancy(mb, a.logR, a.logW) : 0;
        if (occ > 0) {
            // Persistent CTAs: at most the resident count, each walking tiles.
            a.tiles_per_plane = grid.x;
            const u64 tiles = (u64)grid.x * L.planes;
            const u64 cap = (u64)occ * device_sms();
            const unsigned g1 = (unsigned)std::min<u64>(tiles, cap);
            pass_kernel(mb, a.logR, true)<<<g1, 256, lde_smem_bytes(a.logR, a.logW, true), st>>>(a);
        } else {
            pass_kernel(mb, a.logR)<<<grid, 256, lde_smem_bytes(a.logR, a.logW), st>>>(a);
        }
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

// ---- inter-pass twiddle tables ---------------------------------------------
// tab[i 2^logS + col] = w_{2^logNs}^(i col) for i < 2^(logNs - logS).
__global__ void k_pass_table(u64* tab, u32 logNs, u32 logS, const u64* hi, const u64* lo) {
    const u64 total = 1ull << logNs, mask = (1ull << logS) - 1;
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (u64)gridDim.x * blockDim.x)
        tab[k] = twiddle((k >> logS) * (k & mask), logNs, hi, lo);
}

long long lde_tables_prepare_plan(LdeTables& t, const LdePlan& pl, const u64* tw_hi, const u64* tw_lo,
                                  cudaStream_t st, u64 room) {
    if (!lde_plan_valid(pl)) return 0;
    u64* made[3] = {};
    u32 keys[3] = {};
    int nmade = 0;
    long long bytes = 0;
    u32 logNs = pl.logN;
    for (u32 s = 0; s + 1 < pl.npass; ++s) {
        const u32 logR = pl.logR[s];
        const u32 key = logNs * (TW_STAGE_LOG + 1) + logR;
        const size_t sz = (size_t)8 << logNs;
        if (t.tab[key].load() == nullptr && logNs <= LdeTables::MAX_LOG && (u64)bytes + sz <= room) {
            u64* p = nullptr;
            if (cudaMalloc(&p, sz) != cudaSuccess) {
                cudaGetLastError();
                break;
            }
            const u64 total = 1ull << logNs;
            const unsigned grid = (unsigned)std::min<u64>((total + 255) / 256, 4096);
            k_pass_table<<<grid, 256, 0, st>>>(p, logNs, logNs - logR, tw_hi, tw_lo);
            count_launches(1);
            made[nmade] = p;
            keys[nmade++] = key;
            bytes += (long long)sz;
        }
        logNs -= logR;
    }
    if (nmade == 0) return 0;
    if (cudaPeekAtLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
        for (int k = 0; k < nmade; ++k) cudaFree(made[k]);
        return -1;
    }
    for (int k = 0; k < nmade; ++k) {
        u64* expect = nullptr;
        if (!t.tab[keys[k]].compare_exchange_strong(expect, made[k])) {  // built meanwhile by another thread
            cudaFree(made[k]);
            bytes -= (long long)((size_t)8 << (keys[k] / (TW_STAGE_LOG + 1)));
        }
    }
    return bytes;
}

long long lde_tables_prepare(LdeTables& t, u32 logN, u32 logX, const u64* tw_hi, const u64* tw_lo, cudaStream_t st,
                             u64 room) {
    if (logN > TW_LOG) return 0;
    return lde_tables_prepare_plan(t, plan_lde(logN, logX), tw_hi, tw_lo, st, room);
}

void lde_tables_free(LdeTables& t) {
    for (auto& p : t.tab) {
        u64* q = p.exchange(nullptr);
        if (q) cudaFree(q);
    }
}

int lde_prepare() {
    for (u32 mb = 2; mb <= 4; ++mb)
        for (u32 l = 1; l <= TW_STAGE_LOG; ++l) {
            if (cudaFuncSetAttribute(pass_kernel(mb, l), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)LDE_SMEM_MAX) != cudaSuccess ||
                cudaFuncSetAttribute(pass_kernel(mb, l, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)LDE_SMEM_PIPE_MAX) != cudaSuccess)
                return -1;
            for (u32 lw = 0; lw <= 6 && lw <= l; ++lw) pipe_occupancy(mb, l, lw);
        }
    return 0;
}

}  // namespace wg
