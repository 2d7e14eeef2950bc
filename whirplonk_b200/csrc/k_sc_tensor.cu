// k_sc_tensor.cu -- the initial sumcheck of one committed vector, by block
// evaluation: the 2^n covector is never written.
//
// Reference: the covector of the statement and OOD constraints
// (cpp/include/whir/protocols/whir/whir_prover.hpp:150-197; eval_eq,
// multilinear.hpp:121-133; geometric_accumulate, utilities.hpp:261-307) and the
// initial sumcheck on it (whir_prover.hpp:199-209, protocols/
// sumcheck_protocol.hpp:81-144, algebra/sumcheck.hpp:43-116).
//
// Every term of that covector is a product over the index bits.  With
// i = (B, x), B the top k bits (the variables the initial sumcheck folds) and
// x the low L = n - k bits:
//   MLE form f:  crlc_f eq(p_f, i) = [crlc_f eq(p_f[0..k), B)] * eq(p_f[k..n), x)
//   OOD point z: crlc_j z^i        = [crlc_j (z^(2^L))^B]      * z^x
// i.e. b_t(B, x) = G_t(B) Bot_t(x).  Folding the first r variables of the
// vector a and of the covector by the challenges, and summing over x first,
//   sum_x a^(r)(B', x) b^(r)(B', x) = sum_t G_t^(r)(B') Z_t^(r)(B'),
//   Z_t(B) = sum_x a(B, x) Bot_t(x),
// because folding is linear.  So the k rounds are the reference's sumcheck on
// the 2^k-entry tables (Z_t, G_t), summed over the terms: the same c0, c2,
// challenges and running sum, byte for byte.  The work is one pass over the
// base coefficients for Z (k_tsc_eval), a one-CTA kernel for the rounds and
// the transcript (k_tsc_rounds), and one pass that writes the folded vector
// a^(k)(x) = sum_B eq(r, B) a(B, x) and covector b^(k)(x) = sum_t G_t^(k) Bot_t(x)
// at size 2^L (k_tsc_fold) -- the state the reference has after the initial
// sumcheck.  Bot_t(x) = HI_t[x >> LO] * LO_t[x mod 2^LO] from small tables.
#include <algorithm>

#include "launch.h"
#include "state.cuh"
#include "wtx.cuh"

namespace wg {

constexpr u32 TSC_LO = 10;         // low index bits of the Bot tables
constexpr u32 TSC_MAX_K = 5;       // initial-sumcheck rounds (2^k blocks)
constexpr int TSC_MAX_TERMS = 16;  // statement forms + OOD points
constexpr u32 TSC_SPAN_MAX = 512;  // columns (= threads) per CTA of k_tsc_eval
constexpr u32 TSC_ROWS_MAX = 256;  // rows per CTA of k_tsc_eval at most
constexpr u32 TSC_FOLD_THREADS = 256;

struct TscGeom {
    u32 L, lo_bits, hi_bits, span, threads, cg, chunks, rpc, parts;
};

// Split of the 2^L-word blocks into CTAs of k_tsc_eval: rows of 2^lo_bits
// words, `span` columns per CTA (cg column groups per row), `rpc` rows per CTA
// (`chunks` row ranges per block); parts = partial sums per (term, block).
constexpr u32 TSC_SMS_MAX = 1024;  // SM counts above this are treated as this (scratch bound)

static TscGeom tsc_geom(u32 n, u32 k, u32 sms) {
    sms = std::min(std::max(sms, 1u), TSC_SMS_MAX);
    TscGeom g{};
    g.L = n - k;
    g.lo_bits = std::min(g.L, TSC_LO);
    g.hi_bits = g.L - g.lo_bits;
    g.span = std::min(1u << g.lo_bits, TSC_SPAN_MAX);
    g.threads = g.span;
    g.cg = (1u << g.lo_bits) / g.span;
    const u32 rows = 1u << g.hi_bits;
    u32 chunks = std::max<u32>(1, (4 * sms) / ((1u << k) * g.cg));
    chunks = std::max(chunks, (rows + TSC_ROWS_MAX - 1) / TSC_ROWS_MAX);
    chunks = std::min(chunks, rows);
    g.rpc = (rows + chunks - 1) / chunks;
    g.chunks = (rows + g.rpc - 1) / g.rpc;
    g.parts = g.chunks * g.cg;
    return g;
}

bool tsc_applicable(u32 n, u32 k, int n_terms) {
    return k >= 1 && k <= TSC_MAX_K && n >= k + 6 && n <= 40 && n_terms >= 1 && n_terms <= TSC_MAX_TERMS;
}

namespace {
size_t al256(size_t v) { return (v + 255) / 256 * 256; }
struct TscLayout {
    size_t top, lo, hi, part, eqr, total;
};
TscLayout tsc_layout(u32 n, u32 k, int T, u32 parts) {
    const u32 L = n - k, lo_bits = std::min(L, TSC_LO), hi_bits = L - lo_bits;
    TscLayout l{};
    size_t o = 0;
    l.top = o; o = al256(o + (size_t)T * (1u << k) * sizeof(E3));
    l.lo = o;  o = al256(o + (size_t)T * (1u << lo_bits) * sizeof(E3));
    l.hi = o;  o = al256(o + (size_t)T * (1u << hi_bits) * sizeof(E3));
    l.part = o; o = al256(o + (size_t)T * (1u << k) * parts * sizeof(E3));
    l.eqr = o;  o = al256(o + (1u << k) * sizeof(E3));
    l.total = o;
    return l;
}
// Upper bound of tsc_geom's `parts` for any SM count.
u32 tsc_parts_bound(u32 n, u32 k) { return tsc_geom(n, k, TSC_SMS_MAX).parts; }
}  // namespace

// Scratch for up to n_terms terms (a plan sizes it for its largest statement;
// more than TSC_MAX_TERMS terms never take this path).
size_t tsc_scratch_bytes(u32 n, u32 k, int n_terms) {
    const int T = std::min(n_terms, TSC_MAX_TERMS);
    if (!tsc_applicable(n, k, T)) return 0;
    return tsc_layout(n, k, T, tsc_parts_bound(n, k)).total;
}

struct TscTabArgs {
    const u64* points;  // n_forms * n * 3 words
    u32 n, k, L, lo_bits, hi_bits;
    int n_forms, n_ood;
    const ProofScalars* sc;
    E3* top;  // [t][B]
    E3* lo;   // [t][l]
    E3* hi;   // [t][h]
};

// eq factor of an MLE point over coordinates [c0, c0 + bits) for the index
// value v (coordinate c <-> bit (c0 + bits - 1 - c) of v).
__device__ __forceinline__ E3 eq_range(const u64* pt, u32 c0, u32 bits, u32 v) {
    E3 r = e3_one();
    for (u32 c = 0; c < bits; ++c) {
        const E3 x{pt[3 * (c0 + c)], pt[3 * (c0 + c) + 1], pt[3 * (c0 + c) + 2]};
        r = e3_mul(r, ((v >> (bits - 1 - c)) & 1) ? x : e3_sub(e3_one(), x));
    }
    return r;
}

__global__ void k_tsc_tables(TscTabArgs a) {
    const u32 nt = 1u << a.k, nl = 1u << a.lo_bits, nh = 1u << a.hi_bits;
    const u32 per = nt + nl + nh;
    const int T = a.n_forms + a.n_ood;
    const u64 total = (u64)per * T;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const int t = (int)(e / per);
        const u32 q = (u32)(e % per);
        if (t < a.n_forms) {
            const u64* pt = a.points + (u64)t * a.n * 3;
            if (q < nt) {  // linear_forms[0] is accumulated with scalar ONE (whir_prover.hpp:161)
                a.top[(u64)t * nt + q] = e3_mul(t == 0 ? e3_one() : a.sc->crlc[t], eq_range(pt, 0, a.k, q));
            } else if (q < nt + nl) {
                a.lo[(u64)t * nl + (q - nt)] = eq_range(pt, a.n - a.lo_bits, a.lo_bits, q - nt);
            } else {
                a.hi[(u64)t * nh + (q - nt - nl)] = eq_range(pt, a.k, a.hi_bits, q - nt - nl);
            }
        } else {
            const E3 z = a.sc->init_ood_pts[t - a.n_forms];
            if (q < nt) a.top[(u64)t * nt + q] = e3_mul(a.sc->crlc[t], e3_pow(z, (u64)q << a.L));
            else if (q < nt + nl) a.lo[(u64)t * nl + (q - nt)] = e3_pow(z, q - nt);
            else a.hi[(u64)t * nh + (q - nt - nl)] = e3_pow(z, (u64)(q - nt - nl) << a.lo_bits);
        }
    }
}

struct TscEvalArgs {
    const u64* coeffs;
    u32 k, L, lo_bits, hi_bits, span, cg, chunks, rpc, parts;
    int t0, T;  // first term of this pass, all terms
    const E3* lo;
    const E3* hi;
    E3* part;  // [t][B][parts]
};

__device__ __forceinline__ E3 tsc_block_sum(E3 v, E3* red) {
    v = e3_warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    E3 r = e3_zero();
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = e3_add(r, red[w]);
    __syncthreads();
    return r;
}

__device__ __forceinline__ void mac3(Acc192 (&s)[3], const E3& w, u64 x) {
    acc_mac(s[0], w.c0, x);
    acc_mac(s[1], w.c1, x);
    acc_mac(s[2], w.c2, x);
}
__device__ __forceinline__ E3 red3(const Acc192 (&s)[3]) { return E3{acc_reduce(s[0]), acc_reduce(s[1]), acc_reduce(s[2])}; }

// Z_t(B) over one CTA's rows and columns: thread j owns column j of its
// column group and accumulates HI_t[h] * a over the rows (the weight is the
// same for every column of a row); the column factor LO_t is applied once at
// the end.  TT terms per pass.
template <int TT>
__global__ void __launch_bounds__(TSC_SPAN_MAX, 1) k_tsc_eval(TscEvalArgs a) {
    __shared__ E3 red[32];
    const u32 per_b = a.chunks * a.cg;
    const u32 B = blockIdx.x / per_b, rem = blockIdx.x % per_b;
    const u32 chunk = rem / a.cg, g = rem % a.cg;
    const u32 rows = 1u << a.hi_bits, nh = rows, nl = 1u << a.lo_bits;
    const u32 h0 = chunk * a.rpc, h1 = min(h0 + a.rpc, rows);
    const u32 col = g * a.span + threadIdx.x;
    const u64* base = a.coeffs + ((u64)B << a.L) + col;
    Acc192 s[TT][3];
#pragma unroll
    for (int t = 0; t < TT; ++t)
#pragma unroll
        for (int c = 0; c < 3; ++c) s[t][c] = Acc192{0, 0, 0};
    const E3* hi = a.hi + (u64)a.t0 * nh;
    u32 h = h0;
    // four rows' loads in flight before their products
    for (; h + 4 <= h1; h += 4) {
        u64 v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = __ldg(base + ((u64)(h + q) << a.lo_bits));
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int t = 0; t < TT; ++t) mac3(s[t], hi[(u64)t * nh + h + q], v[q]);
    }
    for (; h < h1; ++h) {
        const u64 v = __ldg(base + ((u64)h << a.lo_bits));
#pragma unroll
        for (int t = 0; t < TT; ++t) mac3(s[t], hi[(u64)t * nh + h], v);
    }
#pragma unroll
    for (int t = 0; t < TT; ++t) {
        const E3 val = e3_mul(red3(s[t]), a.lo[(u64)(a.t0 + t) * nl + col]);
        const E3 tot = tsc_block_sum(val, red);
        if (threadIdx.x == 0) a.part[((u64)(a.t0 + t) * (1u << a.k) + B) * a.parts + rem] = tot;
    }
}

struct TscRoundArgs {
    u32 k, parts, hi_bits;
    int T, r_slot;
    const E3* part;
    const E3* top;
    E3* hi;   // rescaled in place by the folded G_t
    E3* eqr;  // eq(r, B), B < 2^k
    TxState* tx;
    ProofScalars* sc;
};

// The k rounds on the (Z_t, G_t) tables, one CTA: Z from the partials, then
// warp 0 runs each round's messages, challenge and fold (transcript order of
// sumcheck_protocol.hpp:99-135, no round PoW), then eq(r, .) for the fold
// pass and HI_t scaled by the folded G_t.
__global__ void __launch_bounds__(256) k_tsc_rounds(TscRoundArgs a) {
    __shared__ E3 Z[TSC_MAX_TERMS << TSC_MAX_K];
    __shared__ E3 G[TSC_MAX_TERMS << TSC_MAX_K];
    __shared__ E3 rs[TSC_MAX_K];
    __shared__ E3 scr[256];
    const u32 nb = 1u << a.k;
    const u32 nv = (u32)a.T * nb;
    if (nv <= blockDim.x && blockDim.x <= 256) {
        // blockDim / nv threads per value, each over a strided share of its
        // partials (independent loads in flight), then one sum per value.
        const u32 per = blockDim.x / nv, v = threadIdx.x % nv, s = threadIdx.x / nv;
        E3 z = e3_zero();
        if (s < per) {
            const E3* p = a.part + (u64)v * a.parts;
            for (u32 q = s; q < a.parts; q += per) z = e3_add(z, p[q]);
        }
        scr[threadIdx.x] = z;
        __syncthreads();
        if (threadIdx.x < nv) {
            E3 t = scr[threadIdx.x];
            for (u32 k = 1; k < per; ++k) t = e3_add(t, scr[threadIdx.x + k * nv]);
            Z[threadIdx.x] = t;
            G[threadIdx.x] = a.top[threadIdx.x];
        }
    } else {
        for (u32 v = threadIdx.x; v < nv; v += blockDim.x) {
            E3 z = e3_zero();
            const E3* p = a.part + (u64)v * a.parts;
            for (u32 q = 0; q < a.parts; ++q) z = e3_add(z, p[q]);
            Z[v] = z;
            G[v] = a.top[v];
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const u32 lane = threadIdx.x;
        ProofScalars* sc = a.sc;
        WarpTx wt;
        wtx_load(wt, a.tx);
        for (u32 r = 0; r < a.k; ++r) {
            const u32 h = nb >> (r + 1);
            E3 c0 = e3_zero(), c2 = e3_zero();
            for (u32 v = lane; v < (u32)a.T * h; v += 32) {
                const u32 t = v / h, i = v % h;
                const E3 zl = Z[t * nb + i], zh = Z[t * nb + i + h], gl = G[t * nb + i], gh = G[t * nb + i + h];
                c0 = e3_add(c0, e3_mul(zl, gl));
                c2 = e3_add(c2, e3_mul(e3_sub(zh, zl), e3_sub(gh, gl)));
            }
            c0 = wtx_sum(c0);
            c2 = wtx_sum(c2);
            wtx_message_t(wt, c0);
            wtx_message_t(wt, c2);
            const E3 rn = wtx_challenge_t(wt);
            if (lane == 0) {
                const E3 c1 = e3_sub(e3_sub(sc->sum, e3_add(c0, c0)), c2);
                sc->c0 = c0;
                sc->c2 = c2;
                sc->sc_r[a.r_slot + r] = rn;
                sc->sum = e3_add(e3_mul(e3_add(e3_mul(c2, rn), c1), rn), c0);
                rs[r] = rn;
            }
            __syncwarp();
            for (u32 v = lane; v < (u32)a.T * h; v += 32) {
                const u32 t = v / h, i = v % h;
                E3& zl = Z[t * nb + i];
                E3& gl = G[t * nb + i];
                zl = e3_add(zl, e3_mul(rn, e3_sub(Z[t * nb + i + h], zl)));
                gl = e3_add(gl, e3_mul(rn, e3_sub(G[t * nb + i + h], gl)));
            }
            __syncwarp();
        }
        wtx_store(wt, a.tx);
    }
    __syncthreads();
    for (u32 B = threadIdx.x; B < nb; B += blockDim.x) {
        E3 e = e3_one();
        for (u32 c = 0; c < a.k; ++c) e = e3_mul(e, ((B >> (a.k - 1 - c)) & 1) ? rs[c] : e3_sub(e3_one(), rs[c]));
        a.eqr[B] = e;
    }
    const u32 nh = 1u << a.hi_bits;
    for (u32 v = threadIdx.x; v < (u32)a.T * nh; v += blockDim.x) a.hi[v] = e3_mul(G[(v / nh) * nb], a.hi[v]);
}

struct TscFoldArgs {
    const u64* coeffs;
    u32 k, L, lo_bits;
    int T;
    const E3* eqr;
    const E3* lo;
    const E3* hi;  // already scaled by the folded G_t
    u64* a_out[3];
    u64* cov_out[3];
};

// a^(k)(x) = sum_B eq(r, B) a(B, x) and b^(k)(x) = sum_t HI'_t[h] LO_t[l],
// two consecutive x per thread (16-byte loads and stores).
__global__ void __launch_bounds__(TSC_FOLD_THREADS) k_tsc_fold(TscFoldArgs a) {
    __shared__ E3 eq[1u << TSC_MAX_K];
    const u32 nb = 1u << a.k;
    for (u32 B = threadIdx.x; B < nb; B += blockDim.x) eq[B] = a.eqr[B];
    __syncthreads();
    const u64 half = 1ull << (a.L - 1);
    const u32 nl = 1u << a.lo_bits, nh = 1u << (a.L - a.lo_bits);
    for (u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x; j < half; j += (u64)gridDim.x * blockDim.x) {
        const u64 x = 2 * j;
        Acc192 s[2][3];
#pragma unroll
        for (int e = 0; e < 2; ++e)
#pragma unroll
            for (int c = 0; c < 3; ++c) s[e][c] = Acc192{0, 0, 0};
        for (u32 B0 = 0; B0 < nb; B0 += 8) {
            ulonglong2 v[8];
            const u32 cnt = min(8u, nb - B0);
#pragma unroll
            for (u32 q = 0; q < 8; ++q)
                if (q < cnt) v[q] = __ldg(reinterpret_cast<const ulonglong2*>(a.coeffs + ((u64)(B0 + q) << a.L) + x));
#pragma unroll
            for (u32 q = 0; q < 8; ++q)
                if (q < cnt) {
                    mac3(s[0], eq[B0 + q], v[q].x);
                    mac3(s[1], eq[B0 + q], v[q].y);
                }
        }
        const E3 a0 = red3(s[0]), a1 = red3(s[1]);
        const u32 h = (u32)(x >> a.lo_bits), l = (u32)(x & (nl - 1));
        E3Acc b0 = e3acc_zero(), b1 = e3acc_zero();
        for (int t = 0; t < a.T; ++t) {
            const E3 w = a.hi[(u64)t * nh + h];
            e3acc_mac(b0, w, a.lo[(u64)t * nl + l]);
            e3acc_mac(b1, w, a.lo[(u64)t * nl + l + 1]);
        }
        const E3 c0 = e3acc_reduce(b0), c1 = e3acc_reduce(b1);
        *reinterpret_cast<ulonglong2*>(a.a_out[0] + x) = make_ulonglong2(a0.c0, a1.c0);
        *reinterpret_cast<ulonglong2*>(a.a_out[1] + x) = make_ulonglong2(a0.c1, a1.c1);
        *reinterpret_cast<ulonglong2*>(a.a_out[2] + x) = make_ulonglong2(a0.c2, a1.c2);
        *reinterpret_cast<ulonglong2*>(a.cov_out[0] + x) = make_ulonglong2(c0.c0, c1.c0);
        *reinterpret_cast<ulonglong2*>(a.cov_out[1] + x) = make_ulonglong2(c0.c1, c1.c1);
        *reinterpret_cast<ulonglong2*>(a.cov_out[2] + x) = make_ulonglong2(c0.c2, c1.c2);
    }
}

int launch_tsc(const TscArgs& s, cudaStream_t st) {
    const int T = s.n_forms + s.n_ood;
    if (!tsc_applicable(s.n, s.k, T) || s.n_forms > MAX_FORMS || s.n_ood > MAX_INIT_OOD) return -1;
    for (int c = 0; c < 3; ++c)
        if ((reinterpret_cast<uintptr_t>(s.a_out[c]) | reinterpret_cast<uintptr_t>(s.cov_out[c])) & 15) return -1;
    if (reinterpret_cast<uintptr_t>(s.coeffs) & 15) return -1;
    const u32 sms = device_sms();
    const TscGeom g = tsc_geom(s.n, s.k, sms);
    if (g.parts > tsc_parts_bound(s.n, s.k)) return -1;
    const TscLayout l = tsc_layout(s.n, s.k, T, g.parts);
    if (l.total > s.scratch_bytes) return -1;
    char* base = reinterpret_cast<char*>(s.scratch);
    E3* top = reinterpret_cast<E3*>(base + l.top);
    E3* lo = reinterpret_cast<E3*>(base + l.lo);
    E3* hi = reinterpret_cast<E3*>(base + l.hi);
    E3* part = reinterpret_cast<E3*>(base + l.part);
    E3* eqr = reinterpret_cast<E3*>(base + l.eqr);

    TscTabArgs ta{s.points, s.n, s.k, g.L, g.lo_bits, g.hi_bits, s.n_forms, s.n_ood, s.sc, top, lo, hi};
    const u64 entries = (u64)T * ((1u << s.k) + (1u << g.lo_bits) + (1u << g.hi_bits));
    k_tsc_tables<<<(unsigned)std::min<u64>(2ull * sms, (entries + 255) / 256), 256, 0, st>>>(ta);
    count_launches(1);

    const unsigned grid = (1u << s.k) * g.chunks * g.cg;
    for (int t0 = 0; t0 < T; t0 += 2) {
        TscEvalArgs ea{s.coeffs, s.k, g.L, g.lo_bits, g.hi_bits, g.span, g.cg, g.chunks, g.rpc, g.parts, t0, T, lo, hi,
                       part};
        if (T - t0 >= 2) k_tsc_eval<2><<<grid, g.threads, 0, st>>>(ea);
        else k_tsc_eval<1><<<grid, g.threads, 0, st>>>(ea);
        count_launches(1);
    }

    TscRoundArgs ra{s.k, g.parts, g.hi_bits, T, s.r_slot, part, top, hi, eqr, s.tx, s.sc};
    k_tsc_rounds<<<1, 256, 0, st>>>(ra);
    count_launches(1);

    TscFoldArgs fa{};
    fa.coeffs = s.coeffs;
    fa.k = s.k;
    fa.L = g.L;
    fa.lo_bits = g.lo_bits;
    fa.T = T;
    fa.eqr = eqr;
    fa.lo = lo;
    fa.hi = hi;
    for (int c = 0; c < 3; ++c) {
        fa.a_out[c] = s.a_out[c];
        fa.cov_out[c] = s.cov_out[c];
    }
    const u64 pairs = 1ull << (g.L - 1);
    const u64 want = (pairs + TSC_FOLD_THREADS - 1) / TSC_FOLD_THREADS;
    k_tsc_fold<<<(unsigned)std::min<u64>(want, 8ull * sms), TSC_FOLD_THREADS, 0, st>>>(fa);
    count_launches(1);
    return 0;
}

}  // namespace wg
