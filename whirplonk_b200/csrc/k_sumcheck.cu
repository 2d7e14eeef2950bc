// k_sumcheck.cu -- extension-field sumcheck and the covector it runs against.
//
// Sumcheck round (cpp/include/whir/algebra/sumcheck.hpp:43-116,
// protocols/sumcheck_protocol.hpp:99-135): on vectors a, b of size s,
//   c0 = sum_{i<s/2} a_i b_i,  c2 = sum_{i<s/2} (a_{i+s/2}-a_i)(b_{i+s/2}-b_i),
// prover messages c0, c2, optional PoW, challenge r, then the fold
//   a_i <- a_i + r (a_{i+s/2} - a_i)  (same for b), sum <- (c2 r + c1) r + c0.
// Here the fold of round t is fused into the kernel of round t+1 (one HBM pass
// per round), partial sums are warp-reduced, and the last CTA to finish
// (atomic ticket) does the transcript step on one thread.
//
// Covector (whir_prover.hpp:150-197, linear_form.hpp:186-206,
// multilinear.hpp:121-133): cov[i] = sum_f crlc_f eq(p_f, i) + sum_j crlc_j z_j^i,
// later cov[i] += sum_j stir_rlc_j z_j^i per round (utilities.hpp:261-307).
#include <algorithm>
#include <mutex>

#include "launch.h"
#include "state.cuh"
#include "wtx.cuh"

namespace wg {

// SC_GRID: capacity of the per-CTA partials array (the grid never exceeds it).
constexpr int SC_THREADS = 256, SC_GRID = 1024;
// CTAs per SM the round kernel's registers are sized for.
#ifndef SC_MINB
#define SC_MINB 3
#endif
#ifndef SC_MINB_FOLD
#define SC_MINB_FOLD 2
#endif

__device__ __forceinline__ E3 block_sum(E3 v, E3* red) {
    v = e3_warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    E3 r = e3_zero();
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = e3_add(r, red[k]);
    __syncthreads();
    return r;
}

__device__ __forceinline__ E3 ld3(u64* const p[3], u64 i) { return E3{p[0][i], p[1][i], p[2][i]}; }
__device__ __forceinline__ void st3(u64* const p[3], u64 i, E3 v) { p[0][i] = v.c0; p[1][i] = v.c1; p[2][i] = v.c2; }

struct ScKernelArgs {
    const u64* a_base;
    u64* a_in[3];
    u64* a_out[3];
    u64* b[3];
    u64 size;
    int fold, fold_r, r_slot;
    u64 pow_threshold;
    TxState* tx;
    ProofScalars* sc;
    E3* partials;
    unsigned* counter;
    int ext2;
};

// The fold x0 + r (x1 - x0) by the round challenge r, a constant of the
// kernel: the X and X^2 parts of r are doubled once (X^3 = 2), x0 seeds the
// 192-bit accumulators and each component is reduced once -- no separate
// doubling or addition per fold.  ext2: fold X^2 = 7 afterwards (e2_fold).
struct FoldR {
    u64 r0, r1, r2, r1d, r2d;
};
__device__ __forceinline__ FoldR fold_r(const E3& r) { return FoldR{r.c0, r.c1, r.c2, gl_add(r.c1, r.c1), gl_add(r.c2, r.c2)}; }
__device__ __forceinline__ E3 fold_e3(const E3& x0, const E3& x1, const FoldR& R, bool ext2) {
    const E3 d = e3_sub(x1, x0);
    Acc192 s0{x0.c0, 0, 0}, s1{x0.c1, 0, 0}, s2{x0.c2, 0, 0};
    acc_mac(s0, R.r0, d.c0);
    acc_mac(s0, R.r2d, d.c1);
    acc_mac(s0, R.r1d, d.c2);
    acc_mac(s1, R.r1, d.c0);
    acc_mac(s1, R.r0, d.c1);
    acc_mac(s1, R.r2d, d.c2);
    acc_mac(s2, R.r2, d.c0);
    acc_mac(s2, R.r1, d.c1);
    acc_mac(s2, R.r0, d.c2);
    return ef_fix(E3{acc_reduce(s0), acc_reduce(s1), acc_reduce(s2)}, ext2);
}

// Loads a_i of the round vector, folding on the fly when requested.
__device__ __forceinline__ E3 load_a(const ScKernelArgs& a, u64 i, const FoldR& r) {
    if (!a.fold) return a.a_base ? e3_base(a.a_base[i]) : ld3(a.a_in, i);
    if (a.a_base) {
        const u64 x0 = a.a_base[i], x1 = a.a_base[i + a.size];
        return e3_add(e3_base(x0), e3_mul_base(E3{r.r0, r.r1, r.r2}, gl_sub(x1, x0)));
    }
    return fold_e3(ld3(a.a_in, i), ld3(a.a_in, i + a.size), r, a.ext2);
}
__device__ __forceinline__ E3 load_b(const ScKernelArgs& a, u64 i, const FoldR& r) {
    if (!a.fold) return ld3(a.b, i);
    return fold_e3(ld3(a.b, i), ld3(a.b, i + a.size), r, a.ext2);
}

// Unreduced sums of Ext3 products (X^3 = 2): the doubled cross terms are fed
// with 2 a1, 2 a2, so three 192-bit accumulators suffice.  A thread adds at
// most 3 products per accumulator per pair it visits, far below the 2^31
// products acc_reduce allows.
struct E3AccL {
    Acc192 s0, s1, s2;
};
__device__ __forceinline__ void accl_mac(E3AccL& x, const E3& a, const E3& b) {
    const u64 a1d = gl_add(a.c1, a.c1), a2d = gl_add(a.c2, a.c2);
    acc_mac(x.s0, a.c0, b.c0);
    acc_mac(x.s0, a1d, b.c2);
    acc_mac(x.s0, a2d, b.c1);
    acc_mac(x.s1, a.c0, b.c1);
    acc_mac(x.s1, a.c1, b.c0);
    acc_mac(x.s1, a2d, b.c2);
    acc_mac(x.s2, a.c0, b.c2);
    acc_mac(x.s2, a.c1, b.c1);
    acc_mac(x.s2, a.c2, b.c0);
}
__device__ __forceinline__ void accl_mac_base(E3AccL& x, u64 a, const E3& b) {
    acc_mac(x.s0, a, b.c0);
    acc_mac(x.s1, a, b.c1);
    acc_mac(x.s2, a, b.c2);
}
__device__ __forceinline__ E3 accl_reduce(const E3AccL& x) {
    return E3{acc_reduce(x.s0), acc_reduce(x.s1), acc_reduce(x.s2)};
}

// CTA sums of (c0, c2), then the last CTA (ticket) sums the partials and does
// the transcript step on one thread.
__device__ __forceinline__ void sc_round_finish(const ScKernelArgs& a, E3 c0, E3 c2, E3* red, bool* is_last) {
    const E3 s0 = block_sum(c0, red);
    const E3 s2 = block_sum(c2, red);
    if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x] = s0;
        a.partials[2 * blockIdx.x + 1] = s2;
        __threadfence();
        *is_last = atomicAdd(a.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!*is_last) return;
    E3 t0 = e3_zero(), t2 = e3_zero();
    for (u32 k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
        const E3* p0 = &a.partials[2 * k];
        const E3* p2 = &a.partials[2 * k + 1];
        t0 = e3_add(t0, E3{__ldcg(&p0->c0), __ldcg(&p0->c1), __ldcg(&p0->c2)});
        t2 = e3_add(t2, E3{__ldcg(&p2->c0), __ldcg(&p2->c1), __ldcg(&p2->c2)});
    }
    const E3 C0s = block_sum(t0, red);
    const E3 C2s = block_sum(t2, red);
    if (threadIdx.x == 0) {
        red[0] = C0s;  // block_sum is done with red: hand the totals to warp 0
        red[1] = C2s;
    }
    __syncwarp();
    if (threadIdx.x < 32) {  // warp 0: c0, c2 messages, [PoW challenge | r], sum
        const E3 C0 = red[0], C2 = red[1];
        ProofScalars* sc = a.sc;
        WarpTx t;
        wtx_load(t, a.tx);
        wtx_message_t(t, C0);
        wtx_message_t(t, C2);
        if (a.pow_threshold != ~0ull) {
            // PoW follows in-stream (ordered windows, then k_sc_after_pow).
            wtx_squeeze_bytes(t, sc->pow_ch, 32);
            if (threadIdx.x == 0) {
                sc->c0 = C0;
                sc->c2 = C2;
                sc->pow_best = ~0ull;
                sc->pow_next = 0;
            }
        } else {
            const E3 rn = wtx_challenge_t(t);
            if (threadIdx.x == 0) {
                const E3 c1 = e3_sub(e3_sub(sc->sum, e3_add(C0, C0)), C2);
                sc->c0 = C0;
                sc->c2 = C2;
                sc->sc_r[a.r_slot] = rn;
                const bool x2 = t.deg == 2;
                sc->sum = e3_add(ef_mul(e3_add(ef_mul(C2, rn, x2), c1), rn, x2), C0);
            }
        }
        wtx_store(t, a.tx);
        if (threadIdx.x == 0) *a.counter = 0;
    }
}

// One round on pairs (i, i + s/2).  FOLD: the vectors still hold the previous
// round's size-2s arrays, folded with its challenge on load (and written back
// folded).  BASE: a is the base-field coefficient array (first rounds only).
template <bool FOLD, bool BASE>
__global__ void __launch_bounds__(SC_THREADS, FOLD ? SC_MINB_FOLD : SC_MINB) k_sumcheck_round(ScKernelArgs a) {
    __shared__ E3 red[32];
    __shared__ bool is_last;
    const E3 r = FOLD ? a.sc->sc_r[a.fold_r] : e3_zero();
    const FoldR R = fold_r(r);
    const u64 half = a.size >> 1;
    E3AccL c0{}, c2{};
    const u64 T = (u64)gridDim.x * blockDim.x;
    u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (!FOLD) {
        // Round 0 is memory-latency bound: two pairs per iteration, every load of
        // both issued before their products.
        for (; i0 + T < half; i0 += 2 * T) {
            const u64 j = i0 + T;
            if (BASE) {
                const u64 al = a.a_base[i0], ah = a.a_base[i0 + half], al2 = a.a_base[j], ah2 = a.a_base[j + half];
                const E3 bl = ld3(a.b, i0), bh = ld3(a.b, i0 + half), bl2 = ld3(a.b, j), bh2 = ld3(a.b, j + half);
                accl_mac_base(c0, al, bl);
                accl_mac_base(c2, gl_sub(ah, al), e3_sub(bh, bl));
                accl_mac_base(c0, al2, bl2);
                accl_mac_base(c2, gl_sub(ah2, al2), e3_sub(bh2, bl2));
            } else {
                const E3 al = ld3(a.a_in, i0), bl = ld3(a.b, i0), ah = ld3(a.a_in, i0 + half), bh = ld3(a.b, i0 + half);
                const E3 al2 = ld3(a.a_in, j), bl2 = ld3(a.b, j), ah2 = ld3(a.a_in, j + half), bh2 = ld3(a.b, j + half);
                accl_mac(c0, al, bl);
                accl_mac(c2, e3_sub(ah, al), e3_sub(bh, bl));
                accl_mac(c0, al2, bl2);
                accl_mac(c2, e3_sub(ah2, al2), e3_sub(bh2, bl2));
            }
        }
    }
    for (u64 i = i0; i < half; i += T) {
        if (BASE && !FOLD) {
            const u64 al = a.a_base[i], ah = a.a_base[i + half];
            const E3 bl = ld3(a.b, i), bh = ld3(a.b, i + half);
            accl_mac_base(c0, al, bl);
            accl_mac_base(c2, gl_sub(ah, al), e3_sub(bh, bl));
        } else if (FOLD) {
            // Every load of the pair before any store: the stores (i, i + half)
            // alias no load of another pair, and the compiler cannot see that.
            const u64 s = a.size;
            E3 x0, x1, x2, x3;
            if (BASE) {
                const u64 p0 = a.a_base[i], p1 = a.a_base[i + s], p2 = a.a_base[i + half], p3 = a.a_base[i + half + s];
                x0 = e3_base(p0); x1 = e3_base(p1); x2 = e3_base(p2); x3 = e3_base(p3);
            } else {
                x0 = ld3(a.a_in, i); x1 = ld3(a.a_in, i + s); x2 = ld3(a.a_in, i + half); x3 = ld3(a.a_in, i + half + s);
            }
            const E3 y0 = ld3(a.b, i), y1 = ld3(a.b, i + s), y2 = ld3(a.b, i + half), y3 = ld3(a.b, i + half + s);
            E3 al, ah;
            if (BASE) {
                al = e3_add(x0, e3_mul_base(r, gl_sub(x1.c0, x0.c0)));
                ah = e3_add(x2, e3_mul_base(r, gl_sub(x3.c0, x2.c0)));
            } else {
                al = fold_e3(x0, x1, R, a.ext2);
                ah = fold_e3(x2, x3, R, a.ext2);
            }
            const E3 bl = fold_e3(y0, y1, R, a.ext2);
            const E3 bh = fold_e3(y2, y3, R, a.ext2);
            st3(a.a_out, i, al); st3(a.b, i, bl);
            st3(a.a_out, i + half, ah); st3(a.b, i + half, bh);
            accl_mac(c0, al, bl);
            accl_mac(c2, e3_sub(ah, al), e3_sub(bh, bl));
        } else {
            const E3 al = ld3(a.a_in, i), bl = ld3(a.b, i), ah = ld3(a.a_in, i + half), bh = ld3(a.b, i + half);
            accl_mac(c0, al, bl);
            accl_mac(c2, e3_sub(ah, al), e3_sub(bh, bl));
        }
    }
    sc_round_finish(a, ef_fix(accl_reduce(c0), a.ext2), ef_fix(accl_reduce(c2), a.ext2), red, &is_last);
}

// After a round PoW: send the nonce, squeeze r, update the sum.
// One warp.
__global__ void k_sc_after_pow(TxState* tx, ProofScalars* sc, int r_slot) {
    if (threadIdx.x >= 32) return;
    const u64 n = sc->pow_best;
    WarpTx t;
    wtx_load(t, tx);
    if (n == ~0ull) t.err |= TX_ERR_POW_EXHAUSTED;
    wtx_message_u64(t, n);
    const E3 rn = wtx_challenge_t(t);
    if (threadIdx.x == 0) {
        const E3 C0 = sc->c0, C2 = sc->c2;
        const E3 c1 = e3_sub(e3_sub(sc->sum, e3_add(C0, C0)), C2);
        sc->sc_r[r_slot] = rn;
        const bool x2 = t.deg == 2;
        sc->sum = e3_add(ef_mul(e3_add(ef_mul(C2, rn, x2), c1), rn, x2), C0);
    }
    wtx_store(t, tx);
}

// ---------------------------------------------------------------------------
// Small sumchecks (size <= SC_SMALL_MAX, no round PoW): all rounds of one
// sumcheck, and the fold after the last one, in ONE CTA.  Round t folds with
// the previous challenge on load exactly as k_sumcheck_round does; warp 0
// carries the transcript across the rounds; __syncthreads orders the rounds.
// This replaces a chain of grid launches whose fixed cost dominates at these
// sizes.
// ---------------------------------------------------------------------------
constexpr u64 SC_SMALL_MAX = 1ull << 12;
// 512 threads leave the kernel 128 registers a thread: at 1024 its 192-bit
// accumulators and the transcript state spilled to local memory.
constexpr int SC_SMALL_THREADS = 512;
constexpr int SC_SMALL_WARPS = SC_SMALL_THREADS / 32;

struct ScSmallArgs {
    const u64* a_base;  // base-field coefficients (first sumcheck) or null
    u64* a[3];
    u64* b[3];
    u64 size;           // size of round 0
    int rounds, r_slot, fold_after;
    TxState* tx;
    ProofScalars* sc;
    int ext2;
};

__global__ void __launch_bounds__(SC_SMALL_THREADS) k_sumcheck_small(ScSmallArgs a) {
    __shared__ E3 red[2][SC_SMALL_WARPS];
    __shared__ E3 rsh;  // the round's challenge, handed from warp 0 to the CTA
    ProofScalars* sc = a.sc;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpTx wt;
    E3 sum{};
    if (warp == 0) {
        wtx_load(wt, a.tx);
        sum = sc->sum;
    }
    for (int t = 0; t <= a.rounds; ++t) {
        const bool last = t == a.rounds;  // only the trailing fold
        if (last && !a.fold_after) break;
        const u64 size = a.size >> t;
        const bool fold = t > 0;
        const bool base = a.a_base && t <= 1;
        const FoldR r = fold_r(fold ? rsh : e3_zero());
        ScKernelArgs k{};
        k.a_base = base ? a.a_base : nullptr;
        for (int c = 0; c < 3; ++c) { k.a_in[c] = a.a[c]; k.a_out[c] = a.a[c]; k.b[c] = a.b[c]; }
        k.size = size;
        k.fold = fold;
        k.ext2 = a.ext2;
        if (last) {  // fold only
            for (u64 i = threadIdx.x; i < size; i += blockDim.x) {
                st3(k.a_out, i, load_a(k, i, r));
                st3(k.b, i, load_b(k, i, r));
            }
            break;
        }
        const u64 half = size >> 1;
        E3AccL c0{}, c2{};
        for (u64 i = threadIdx.x; i < half; i += blockDim.x) {
            if (base && !fold) {
                const u64 al = a.a_base[i], ah = a.a_base[i + half];
                const E3 bl = ld3(k.b, i), bh = ld3(k.b, i + half);
                accl_mac_base(c0, al, bl);
                accl_mac_base(c2, gl_sub(ah, al), e3_sub(bh, bl));
            } else {
                const E3 al = load_a(k, i, r), bl = load_b(k, i, r);
                if (fold) { st3(k.a_out, i, al); st3(k.b, i, bl); }
                accl_mac(c0, al, bl);
                const E3 ah = load_a(k, i + half, r), bh = load_b(k, i + half, r);
                if (fold) { st3(k.a_out, i + half, ah); st3(k.b, i + half, bh); }
                accl_mac(c2, e3_sub(ah, al), e3_sub(bh, bl));
            }
        }
        // Both sums in one barrier: warp partials to shared memory, then warp 0
        // adds them lane-parallel (field sums are exact, so order is free).
        const E3 w0 = e3_warp_sum(ef_fix(accl_reduce(c0), a.ext2));
        const E3 w2 = e3_warp_sum(ef_fix(accl_reduce(c2), a.ext2));
        if (lane == 0) {
            red[0][warp] = w0;
            red[1][warp] = w2;
        }
        __syncthreads();
        if (warp == 0) {
            const int nwarps = (int)(blockDim.x >> 5);
            const E3 C0 = e3_warp_sum(lane < nwarps ? red[0][lane] : e3_zero());
            const E3 C2 = e3_warp_sum(lane < nwarps ? red[1][lane] : e3_zero());
            wtx_message_t(wt, C0);
            wtx_message_t(wt, C2);
            const E3 rn = wtx_challenge_t(wt);
            const bool x2 = wt.deg == 2;
            const E3 c1 = e3_sub(e3_sub(sum, e3_add(C0, C0)), C2);
            sum = e3_add(ef_mul(e3_add(ef_mul(C2, rn, x2), c1), rn, x2), C0);
            if (lane == 0) {
                sc->c0 = C0;
                sc->c2 = C2;
                sc->sc_r[a.r_slot + t] = rn;
                rsh = rn;
            }
        }
        __syncthreads();
    }
    if (warp == 0) {
        if (lane == 0) sc->sum = sum;
        wtx_store(wt, a.tx);
    }
}

int launch_sumcheck_small(const SumcheckArgs& s, int rounds, int fold_after, cudaStream_t st) {
    if (s.size > SC_SMALL_MAX || s.pow_threshold != ~0ull || rounds < 1) return 1;  // not this path
    if ((s.size >> rounds) < 1) return -1;
    ScSmallArgs a{};
    a.a_base = s.a_base;
    for (int c = 0; c < 3; ++c) { a.a[c] = s.a_in[c]; a.b[c] = s.b[c]; }
    a.size = s.size;
    a.rounds = rounds;
    a.r_slot = s.r_slot;
    a.fold_after = fold_after;
    a.tx = s.tx;
    a.sc = s.sc;
    a.ext2 = s.ext2;
    // As many warps as round 0 has pairs for (one warp up to 32 pairs): the
    // rounds are chains of transcript steps, and barriers and cross-warp sums
    // over idle warps only lengthen them.
    u32 threads = 32;
    while (threads < (u32)SC_SMALL_THREADS && threads < (s.size >> 1)) threads <<= 1;
    k_sumcheck_small<<<1, threads, 0, st>>>(a);
    count_launches(1);
    return 0;
}

static ScKernelArgs make_sc(const SumcheckArgs& s) {
    ScKernelArgs a{};
    a.a_base = s.a_base;
    for (int c = 0; c < 3; ++c) { a.a_in[c] = s.a_in[c]; a.a_out[c] = s.a_out[c]; a.b[c] = s.b[c]; }
    a.size = s.size;
    a.fold = s.fold;
    a.fold_r = s.fold_r;
    a.r_slot = s.r_slot;
    a.pow_threshold = s.pow_threshold;
    a.tx = s.tx;
    a.sc = s.sc;
    a.ext2 = s.ext2;
    a.partials = reinterpret_cast<E3*>(s.scratch);
    a.counter = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(s.scratch) + (size_t)SC_GRID * 2 * sizeof(E3));
    return a;
}

size_t sumcheck_scratch_bytes() { return (size_t)SC_GRID * 2 * sizeof(E3) + 256; }

int launch_pow_grind_only(ProofScalars* sc, u64 threshold, int hash, cudaStream_t st);  // k_tx.cu

constexpr int MAX_DEVICES = 64;
static u32 g_sms[MAX_DEVICES];  // 0 = not looked up yet
static std::mutex g_sms_mu;

u32 device_sms() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return 148;
    std::lock_guard<std::mutex> lk(g_sms_mu);
    if (!g_sms[dev]) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) return 148;
        g_sms[dev] = (u32)sms;
    }
    return g_sms[dev];
}

// Resident CTAs per SM of k_sumcheck_round<fold, base> (index 2 fold + base);
// a grid of at most SMs x this many runs in one wave (the grid-stride loop
// does the rest).  Occupancy depends on the kernel and the architecture only.
static int g_sc_occ[4] = {1, 1, 1, 1};

int sumcheck_prepare() {
    const void* fns[4] = {(const void*)k_sumcheck_round<false, false>, (const void*)k_sumcheck_round<false, true>,
                          (const void*)k_sumcheck_round<true, false>, (const void*)k_sumcheck_round<true, true>};
    for (int k = 0; k < 4; ++k) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fns[k], SC_THREADS, 0) != cudaSuccess) return -1;
        g_sc_occ[k] = occ < 1 ? 1 : occ;
    }
    return device_sms() ? 0 : -1;
}

int launch_sumcheck_round(const SumcheckArgs& s, cudaStream_t st) {
    if (s.size < 2) return -1;
    ScKernelArgs a = make_sc(s);
    const u64 half = s.size >> 1;
    const bool base = a.a_base != nullptr;
    const u64 resident = (u64)device_sms() * (u64)g_sc_occ[(a.fold ? 2 : 0) + (base ? 1 : 0)];
    const u64 cap = resident > (u64)SC_GRID ? (u64)SC_GRID : resident;
    u64 want = (half + SC_THREADS - 1) / SC_THREADS;
    const unsigned grid = (unsigned)(want > cap ? cap : (want < 1 ? 1 : want));
    if (a.fold) {
        if (base) k_sumcheck_round<true, true><<<grid, SC_THREADS, 0, st>>>(a);
        else k_sumcheck_round<true, false><<<grid, SC_THREADS, 0, st>>>(a);
    } else {
        if (base) k_sumcheck_round<false, true><<<grid, SC_THREADS, 0, st>>>(a);
        else k_sumcheck_round<false, false><<<grid, SC_THREADS, 0, st>>>(a);
    }
    count_launches(1);
    if (s.pow_threshold != ~0ull) {
        launch_pow_grind_only(s.sc, s.pow_threshold, s.hash, st);
        k_sc_after_pow<<<1, 32, 0, st>>>(s.tx, s.sc, s.r_slot);
        count_launches(1);
    }
    return 0;
}

__global__ void __launch_bounds__(SC_THREADS) k_fold(ScKernelArgs a) {
    const FoldR r = fold_r(a.sc->sc_r[a.fold_r]);
    const u64 T = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < a.size; i += T) {
        st3(a.a_out, i, load_a(a, i, r));
        st3(a.b, i, load_b(a, i, r));
    }
}

int launch_fold(const SumcheckArgs& s, cudaStream_t st) {
    ScKernelArgs a = make_sc(s);
    a.fold = 1;
    u64 want = (s.size + SC_THREADS - 1) / SC_THREADS;
    const u64 cap = std::min<u64>((u64)device_sms() * 4, (u64)SC_GRID);
    const unsigned grid = (unsigned)(want > cap ? cap : (want < 1 ? 1 : want));
    k_fold<<<grid, SC_THREADS, 0, st>>>(a);
    count_launches(1);
    return 0;
}

// ---------------------------------------------------------------------------
// Initial covector.  i = hi * 2^LO + lo; per form f the factors
// eq_hi_f[hi] (scaled by crlc_f) and eq_lo_f[lo] are tabulated, per OOD point
// z_j the powers crlc_{F+j} z_j^(hi 2^LO) and z_j^lo; then
//   cov[i] = sum_f eq_hi_f[hi] eq_lo_f[lo] + sum_j zhi_j[hi] zlo_j[lo].
// ---------------------------------------------------------------------------
constexpr u32 COV_LO = 10;

__global__ void k_cov_tables(const u64* points, u32 logS, int n_forms, int n_ood, u32 dense_mask, ProofScalars* sc,
                             E3* tab, bool ext2, TxState* tx) {
    const u32 lo_bits = logS < COV_LO ? logS : COV_LO, hi_bits = logS - lo_bits;
    const u32 nlo = 1u << lo_bits, nhi = 1u << hi_bits;
    const u32 per = nlo + nhi;
    const u32 nterms = (u32)(n_forms + n_ood);
    const u64 total = (u64)per * nterms;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u32 term = (u32)(e / per), k = (u32)(e % per);
        E3 v;
        if ((int)term < n_forms && ((dense_mask >> term) & 1)) {
            v = e3_zero();  // dense covector: not tabulated (k_cov_init reads it)
        } else if ((int)term < n_forms) {
            const u64* pt = points + (u64)term * logS * 3;
            // coordinate c <-> bit (logS - 1 - c) of i; hi bits are coordinates 0..hi_bits-1
            v = e3_one();
            if (ext2 && k == 0)  // a GoldilocksExt2 point has no X^2 coordinate
                for (u32 c = 0; c < logS; ++c)
                    if (pt[3 * c + 2]) atomicOr(&tx->err, TX_ERR_FIELD);
            if (k < nlo) {
                for (u32 c = hi_bits; c < logS; ++c) {
                    const E3 x{pt[3 * c], pt[3 * c + 1], pt[3 * c + 2]};
                    const bool bit = (k >> (logS - 1 - c)) & 1;
                    v = ef_mul(v, bit ? x : e3_sub(e3_one(), x), ext2);
                }
            } else {
                const u32 h = k - nlo;
                for (u32 c = 0; c < hi_bits; ++c) {
                    const E3 x{pt[3 * c], pt[3 * c + 1], pt[3 * c + 2]};
                    const bool bit = (h >> (hi_bits - 1 - c)) & 1;
                    v = ef_mul(v, bit ? x : e3_sub(e3_one(), x), ext2);
                }
                // linear_forms[0] is accumulated with scalar ONE (whir_prover.hpp:161)
                v = ef_mul(v, term == 0 ? e3_one() : sc->crlc[term], ext2);
            }
        } else {
            const int j = (int)term - n_forms;
            const E3 z = sc->init_ood_pts[j];
            if (k < nlo) v = ef_pow(z, k, ext2);
            else v = ef_mul(sc->crlc[n_forms + j], ef_pow(z, (u64)(k - nlo) << lo_bits, ext2), ext2);
        }
        tab[e] = v;
    }
}

__global__ void __launch_bounds__(256) k_cov_init(CovInitArgs a, const E3* tab) {
    const u32 lo_bits = a.logS < COV_LO ? a.logS : COV_LO, hi_bits = a.logS - lo_bits;
    const u32 nlo = 1u << lo_bits, nhi = 1u << hi_bits;
    const u32 per = nlo + nhi;
    const int nterms = a.n_forms + a.n_ood;
    const u64 S = 1ull << a.logS;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < S; i += (u64)gridDim.x * blockDim.x) {
        const u32 hi = (u32)(i >> lo_bits), lo = (u32)(i & (nlo - 1));
        E3Acc s = e3acc_zero();
        for (int t = 0; t < nterms; ++t) {
            if (t < a.n_forms && ((a.dense_mask >> t) & 1)) {
                // Covector::accumulate: scalar * vector (linear_form.hpp:75-78)
                const u64* d = a.dense[t] + 3 * i;
                if (a.ext2 && d[2]) atomicOr(&a.tx->err, TX_ERR_FIELD);  // not a GoldilocksExt2 value
                e3acc_mac(s, t == 0 ? e3_one() : a.sc->crlc[t], E3{d[0], d[1], d[2]});
            } else {
                e3acc_mac(s, tab[(u64)t * per + nlo + hi], tab[(u64)t * per + lo]);
            }
        }
        const E3 acc = ef_fix(e3acc_reduce(s), a.ext2);
        a.cov[0][i] = acc.c0;
        a.cov[1][i] = acc.c1;
        a.cov[2][i] = acc.c2;
        if (a.write_vec) {
            E3Acc r = e3acc_zero();
            for (u32 v = 0; v < a.nvec; ++v) e3acc_mac_base(r, a.sc->vrlc[v], a.vecs[(u64)v * S + i]);
            const E3 x = e3acc_reduce(r);
            a.vec_out[0][i] = x.c0;
            a.vec_out[1][i] = x.c1;
            a.vec_out[2][i] = x.c2;
        }
    }
    (void)nhi;
}

size_t cov_init_scratch_bytes(u32 logS, int n_forms, int n_ood) {
    const u32 lo_bits = logS < COV_LO ? logS : COV_LO, hi_bits = logS - lo_bits;
    return ((size_t)(1u << lo_bits) + (1u << hi_bits)) * (size_t)(n_forms + n_ood) * sizeof(E3) + 256;
}

int launch_cov_init(const CovInitArgs& a, cudaStream_t st) {
    if (a.n_forms > MAX_FORMS || a.n_ood > MAX_INIT_OOD || a.nvec < 1 || a.nvec > (u32)MAX_VECTORS) return -1;
    if (a.nvec > 1 && !a.write_vec) return -1;
    E3* tab = reinterpret_cast<E3*>(a.scratch);
    const int nterms = a.n_forms + a.n_ood;
    const u64 S = 1ull << a.logS;
    if (nterms == 0 && !a.write_vec) {  // no constraint and no vector to write: a zero covector
        for (int c = 0; c < 3; ++c) cudaMemsetAsync(a.cov[c], 0, S * 8, st);
        return 0;
    }
    for (int f = 0; f < a.n_forms; ++f)
        if (((a.dense_mask >> f) & 1) && !a.dense[f]) return -1;
    if (nterms > 0) {
        k_cov_tables<<<device_sms(), 256, 0, st>>>(a.points, a.logS, a.n_forms, a.n_ood, a.dense_mask, a.sc, tab, a.ext2 != 0, a.tx);
        count_launches(1);
    }
    u64 want = (S + 255) / 256;
    const u64 cap = (u64)device_sms() * 16;
    k_cov_init<<<(unsigned)(want > cap ? cap : want), 256, 0, st>>>(a, tab);
    count_launches(1);
    return 0;
}

// ---------------------------------------------------------------------------
// STIR covector update: cov[i] += sum_j rlc_j z_j^i for the round's OOD points
// (Ext3) and in-domain points (base field, lifted).  With i = h 2^LO + l the
// tables hold T_j[h] = rlc_j z_j^(h 2^LO) (Ext3) and z_j^l; an element's sum
// over the points is accumulated as unreduced 192-bit products (3 per base
// point, 9 per Ext3 point) and reduced once.  LO = 8 keeps every point's
// z_j^l table (2 KiB for a base point) resident in L1 next to the others.
// ---------------------------------------------------------------------------
constexpr u32 CA_LO = 8;

// Point j's table: z_j^l (l < 2^LO) then rlc_j z_j^(h 2^LO).  For the base-field
// (in-domain) points z_j^l is a base element and goes to the compact array
// lo_base[j - n_ext][l] instead, so a warp reads 8 contiguous bytes per lane.
__global__ void k_cov_acc_tables(const ProofScalars* sc, int n_ext, int n_points, u32 hi_count, E3* tab, u64* lo_base,
                                 bool ext2) {
    const u32 per = (1u << CA_LO) + hi_count;
    const u64 total = (u64)per * n_points;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (u64)gridDim.x * blockDim.x) {
        const u32 j = (u32)(e / per), k = (u32)(e % per);
        const E3 z = sc->stir_pts[j];
        if ((int)j < n_ext) {
            tab[e] = k < (1u << CA_LO) ? ef_pow(z, k, ext2)
                                       : ef_mul(sc->stir_rlc[j], ef_pow(z, (u64)(k - (1u << CA_LO)) << CA_LO, ext2), ext2);
        } else if (k < (1u << CA_LO)) {
            lo_base[(u64)(j - n_ext) * (1u << CA_LO) + k] = gl_pow(z.c0, k);
        } else {
            tab[e] = e3_mul_base(sc->stir_rlc[j], gl_pow(z.c0, (u64)(k - (1u << CA_LO)) << CA_LO));
        }
    }
}

// Two consecutive elements (same row h) per thread: each T_j[h] load serves
// both.  The Ext3 points (the OOD samples, few) take full Ext3 products and are
// reduced first; the base points then accumulate into three 192-bit sums per
// element, two points at a time with their loads first -- small enough
// accumulators for three CTAs per SM.
__global__ void __launch_bounds__(256, 3) k_cov_accumulate(CovAccArgs a, const E3* tab, const u64* lo_base,
                                                           u32 hi_count) {
    constexpr u32 NL = 1u << CA_LO;
    const u32 per = NL + hi_count;
    const int npts = a.n_ext + a.n_base;
    const u64 npair = (a.size + 1) >> 1;
    for (u64 pi = (u64)blockIdx.x * blockDim.x + threadIdx.x; pi < npair; pi += (u64)gridDim.x * blockDim.x) {
        const u64 i = 2 * pi;
        const bool two = i + 1 < a.size;
        const u32 hi = (u32)(i >> CA_LO), lo = (u32)(i & (NL - 1));  // lo even: lo + 1 < NL
        E3 e0 = e3_zero(), e1 = e3_zero();
        for (u32 k = 0; k < 2 && a.n_ext > 0; ++k) {  // one element at a time: one E3Acc live
            E3Acc s = e3acc_zero();
            for (int j = 0; j < a.n_ext; ++j) e3acc_mac(s, tab[(u64)j * per + NL + hi], tab[(u64)j * per + lo + k]);
            const E3 r = e3acc_reduce(s);
            if (k == 0) e0 = r;
            else e1 = r;
        }
        Acc192 b0[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, b1[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        int j = a.n_ext;
        for (; j + 2 <= npts; j += 2) {
            E3 w[2];
            u64 x0[2], x1[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                w[q] = tab[(u64)(j + q) * per + NL + hi];
                const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(lo_base + (u64)(j + q - a.n_ext) * NL + lo);
                x0[q] = x.x;
                x1[q] = x.y;
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                acc_mac(b0[0], w[q].c0, x0[q]);
                acc_mac(b0[1], w[q].c1, x0[q]);
                acc_mac(b0[2], w[q].c2, x0[q]);
                acc_mac(b1[0], w[q].c0, x1[q]);
                acc_mac(b1[1], w[q].c1, x1[q]);
                acc_mac(b1[2], w[q].c2, x1[q]);
            }
        }
        for (; j < npts; ++j) {
            const E3 wj = tab[(u64)j * per + NL + hi];
            const u64* lb = lo_base + (u64)(j - a.n_ext) * NL + lo;
            acc_mac(b0[0], wj.c0, lb[0]);
            acc_mac(b0[1], wj.c1, lb[0]);
            acc_mac(b0[2], wj.c2, lb[0]);
            acc_mac(b1[0], wj.c0, lb[1]);
            acc_mac(b1[1], wj.c1, lb[1]);
            acc_mac(b1[2], wj.c2, lb[1]);
        }
        const E3 add0 = ef_fix(e3_add(e0, E3{acc_reduce(b0[0]), acc_reduce(b0[1]), acc_reduce(b0[2])}), a.ext2);
        const E3 add1 = ef_fix(e3_add(e1, E3{acc_reduce(b1[0]), acc_reduce(b1[1]), acc_reduce(b1[2])}), a.ext2);
        if (two) {
            const u64 d0[3] = {add0.c0, add0.c1, add0.c2}, d1[3] = {add1.c0, add1.c1, add1.c2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                ulonglong2* p = reinterpret_cast<ulonglong2*>(a.cov[c] + i);
                const ulonglong2 v = *p;
                *p = make_ulonglong2(gl_add(v.x, d0[c]), gl_add(v.y, d1[c]));
            }
        } else {
            a.cov[0][i] = gl_add(a.cov[0][i], add0.c0);
            a.cov[1][i] = gl_add(a.cov[1][i], add0.c1);
            a.cov[2][i] = gl_add(a.cov[2][i], add0.c2);
        }
    }
}

// Small vectors (few pairs, tens of points): a CTA of CA_SPLIT warps over 32
// pairs, warp w taking the points j = w, w + CA_SPLIT, ...; the partial sums
// meet in shared memory and warp 0 adds them to the covector.  The same field
// sums as k_cov_accumulate (exact, so the grouping is free), with the point
// loop spread over 8x the threads: at these sizes the loop's latency, not its
// multiply-accumulates, is the cost.
constexpr int CA_SPLIT = 8;
constexpr u64 CA_SPLIT_MAX_PAIRS = 2048;
__global__ void __launch_bounds__(32 * CA_SPLIT) k_cov_accumulate_split(CovAccArgs a, const E3* tab, const u64* lo_base,
                                                                         u32 hi_count) {
    constexpr u32 NL = 1u << CA_LO;
    __shared__ E3 part[CA_SPLIT][2][32];
    const u32 per = NL + hi_count;
    const int npts = a.n_ext + a.n_base;
    const u32 lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const u64 npair = (a.size + 1) >> 1;
    const u64 pi = (u64)blockIdx.x * 32 + lane;
    const u64 i = 2 * pi;
    E3 s0 = e3_zero(), s1 = e3_zero();
    if (pi < npair) {
        const u32 hi = (u32)(i >> CA_LO), lo = (u32)(i & (NL - 1));  // lo even: lo + 1 < NL
        for (int j = (int)w; j < npts; j += CA_SPLIT) {
            const E3 h = tab[(u64)j * per + NL + hi];
            if (j < a.n_ext) {
                s0 = e3_add(s0, e3_mul(h, tab[(u64)j * per + lo]));
                s1 = e3_add(s1, e3_mul(h, tab[(u64)j * per + lo + 1]));
            } else {
                const u64* lb = lo_base + (u64)(j - a.n_ext) * NL + lo;
                s0 = e3_add(s0, e3_mul_base(h, lb[0]));
                s1 = e3_add(s1, e3_mul_base(h, lb[1]));
            }
        }
    }
    part[w][0][lane] = s0;
    part[w][1][lane] = s1;
    __syncthreads();
    if (w != 0 || pi >= npair) return;
#pragma unroll 1
    for (int k = 1; k < CA_SPLIT; ++k) {
        s0 = e3_add(s0, part[k][0][lane]);
        s1 = e3_add(s1, part[k][1][lane]);
    }
    s0 = ef_fix(s0, a.ext2);
    s1 = ef_fix(s1, a.ext2);
    a.cov[0][i] = gl_add(a.cov[0][i], s0.c0);
    a.cov[1][i] = gl_add(a.cov[1][i], s0.c1);
    a.cov[2][i] = gl_add(a.cov[2][i], s0.c2);
    if (i + 1 < a.size) {
        a.cov[0][i + 1] = gl_add(a.cov[0][i + 1], s1.c0);
        a.cov[1][i + 1] = gl_add(a.cov[1][i + 1], s1.c1);
        a.cov[2][i + 1] = gl_add(a.cov[2][i + 1], s1.c2);
    }
}

static u32 ca_hi_count(u64 size) { return (u32)((size + (1ull << CA_LO) - 1) >> CA_LO) + 1; }

size_t cov_acc_scratch_bytes(u64 size, int n_points) {
    return ((size_t)(1u << CA_LO) + ca_hi_count(size)) * (size_t)n_points * sizeof(E3) + 256 +
           (size_t)n_points * (1u << CA_LO) * sizeof(u64);
}

int launch_cov_accumulate(const CovAccArgs& a, cudaStream_t st) {
    const int npts = a.n_ext + a.n_base;
    if (npts == 0 || a.size == 0) return 0;
    const u32 hc = ca_hi_count(a.size);
    E3* tab = reinterpret_cast<E3*>(a.scratch);
    const size_t tab_bytes = ((size_t)(1u << CA_LO) + hc) * (size_t)npts * sizeof(E3);
    u64* lo_base = reinterpret_cast<u64*>(reinterpret_cast<char*>(a.scratch) + (tab_bytes + 255) / 256 * 256);
    k_cov_acc_tables<<<2 * device_sms(), 256, 0, st>>>(a.sc, a.n_ext, npts, hc, tab, lo_base, a.ext2 != 0);
    count_launches(1);
    for (int c = 0; c < 3; ++c)
        if (reinterpret_cast<uintptr_t>(a.cov[c]) & 15) return -1;  // 16-byte pairs
    const u64 npair = (a.size + 1) / 2;
    if (npair <= CA_SPLIT_MAX_PAIRS) {
        k_cov_accumulate_split<<<(unsigned)((npair + 31) / 32), 32 * CA_SPLIT, 0, st>>>(a, tab, lo_base, hc);
        count_launches(1);
        return 0;
    }
    u64 want = (npair + 255) / 256;
    const u64 cap = (u64)device_sms() * 16;
    k_cov_accumulate<<<(unsigned)(want > cap ? cap : want), 256, 0, st>>>(a, tab, lo_base, hc);
    count_launches(1);
    return 0;
}

}  // namespace wg

namespace wg {

// MLE evaluation sum_i v_i eq(p, i): eq factors from k_cov_tables (one form,
// scalar one), then a CTA-reduced dot product with a last-CTA finish.
__global__ void __launch_bounds__(256) k_mle_dot(const u64* v, u32 logS, const E3* tab, E3* partials,
                                                 unsigned* counter, u64* out) {
    __shared__ E3 red[32];
    __shared__ bool is_last;
    const u32 lo_bits = logS < COV_LO ? logS : COV_LO;
    const u32 nlo = 1u << lo_bits;
    const u64 S = 1ull << logS;
    E3 acc = e3_zero();
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < S; i += (u64)gridDim.x * blockDim.x) {
        const u32 hi = (u32)(i >> lo_bits), lo = (u32)(i & (nlo - 1));
        acc = e3_add(acc, e3_mul_base(e3_mul(tab[nlo + hi], tab[lo]), v[i]));
    }
    const E3 s = block_sum(acc, red);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = s;
        __threadfence();
        is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    E3 t = e3_zero();
    for (u32 k = threadIdx.x; k < gridDim.x; k += blockDim.x)
        t = e3_add(t, E3{__ldcg(&partials[k].c0), __ldcg(&partials[k].c1), __ldcg(&partials[k].c2)});
    const E3 tot = block_sum(t, red);
    if (threadIdx.x == 0) {
        out[0] = tot.c0;
        out[1] = tot.c1;
        out[2] = tot.c2;
        *counter = 0;
    }
}

// Capacity of the per-CTA partials of k_mle_dot in the scratch layout below.
constexpr u32 MLE_MAX_CTAS = 592;

size_t mle_eval_scratch_bytes(u32 logS) { return 256 + MLE_MAX_CTAS * sizeof(E3) + cov_init_scratch_bytes(logS, 1, 0); }

int launch_mle_eval(const u64* coeffs, u32 logS, const u64* point, void* scratch, u64* out, cudaStream_t st) {
    // [ticket counter | per-CTA partials | eq tables]: the counter keeps a
    // fixed offset whatever logS, and is cleared before every launch.
    // Returns 0, or the CUDA error of the memset or of a launch (the caller
    // makes sure no error was pending before, so a launch error is this call's).
    char* base = reinterpret_cast<char*>(scratch);
    unsigned* counter = reinterpret_cast<unsigned*>(base);
    E3* partials = reinterpret_cast<E3*>(base + 256);
    E3* tab = reinterpret_cast<E3*>(base + 256 + MLE_MAX_CTAS * sizeof(E3));
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return (int)e;
    k_cov_tables<<<device_sms(), 256, 0, st>>>(point, logS, 1, 0, 0u, nullptr, tab, false, nullptr);
    count_launches(1);
    if ((e = cudaPeekAtLastError()) != cudaSuccess) return (int)e;
    const u64 S = 1ull << logS;
    u64 want = (S + 255) / 256;
    const u64 cap = std::min<u64>((u64)device_sms() * 4, MLE_MAX_CTAS);
    const unsigned grid = (unsigned)(want > cap ? cap : want);
    k_mle_dot<<<grid, 256, 0, st>>>(coeffs, logS, tab, partials, counter, out);
    count_launches(1);
    return (int)cudaPeekAtLastError();
}

}  // namespace wg
