// wtx.cuh -- the Fiat-Shamir transcript run by one warp.
//
// The byte semantics of transcript.cuh (the reference ProverState over a
// SHAKE128 duplex sponge, transcript.hpp:80-139, 375-453, 595-662); the sponge
// lives in registers of one warp: lane l < 25
// holds lane l of the hasher and of the XOF reader, Keccak-f[1600] runs with
// one state word per lane (theta / rho-pi / chi data exchange by shuffles), and
// aligned absorbs and squeezes move whole 8-byte words.  The bookkeeping values
// (positions, stream lengths) are warp-uniform; stream bytes are written by
// lane 0.
//
// Every function is warp-collective: all 32 lanes of the warp call it with the
// same arguments.  A kernel loads the state with wtx_load, runs its steps and
// writes it back with wtx_store.
#pragma once
#include "transcript.cuh"

namespace wg {

struct WarpTx {
    u64 h, r;  // this lane's hasher / reader word (lanes 0..24)
    unsigned hpos, rpos, has_reader, err, deg;
    u64 narg_len, hints_len, narg_cap, hints_cap;
    u8* narg;
    u8* hints;
};

__device__ __forceinline__ unsigned wtx_lane() { return threadIdx.x & 31; }

__device__ __forceinline__ u64 rotl64_var(u64 v, unsigned s) { return s ? ((v << s) | (v >> (64 - s))) : v; }

// Source lane of pi for lane (X, Y): pi moves A[x][y] to (y, 2x + 3y), so lane
// (X, Y) receives from (3 (Y - 3X) mod 5, X).
__device__ __forceinline__ unsigned keccak_pi_src(unsigned x, unsigned y) {
    return ((5 + 3 * ((y + 15 - 3 * x) % 5)) % 5) + 5 * x;
}

// Keccak-f[1600] with state word l in lane l (lanes 25..31 carry a dummy).
// Lane (x, y) = x + 5 y.  Each lane rotates its own word (rho), then fetches
// the three pi-permuted words chi needs -- B[X][Y], B[X+1][Y], B[X+2][Y] --
// straight from their source lanes: three shuffle stages per round (theta's
// column sums, theta's D, pi + chi).
static __device__ __noinline__ u64 keccak_f1600_warp(u64 a) {
    const unsigned l = wtx_lane();
    const bool live = l < 25;
    const unsigned x = live ? l % 5 : 0, y = live ? l / 5 : 0;
    unsigned th[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) th[k] = live ? x + 5 * ((y + 1 + k) % 5) : l;
    const unsigned cl = live ? (x + 4) % 5 + 5 * y : l, cr = live ? (x + 1) % 5 + 5 * y : l;
    const unsigned p0 = live ? keccak_pi_src(x, y) : l;
    const unsigned p1 = live ? keccak_pi_src((x + 1) % 5, y) : l;
    const unsigned p2 = live ? keccak_pi_src((x + 2) % 5, y) : l;
    unsigned rot = 0;
#pragma unroll
    for (int yy = 0; yy < 5; ++yy)
#pragma unroll
        for (int xx = 0; xx < 5; ++xx)
            if (live && x == (unsigned)xx && y == (unsigned)yy) rot = keccak_rho(xx, yy);
#pragma unroll 1
    for (int round = 0; round < 24; ++round) {
        u64 c = a;
#pragma unroll
        for (int k = 0; k < 4; ++k) c ^= __shfl_sync(0xFFFFFFFFu, a, th[k]);
        const u64 d = __shfl_sync(0xFFFFFFFFu, c, cl) ^ rotl64_var(__shfl_sync(0xFFFFFFFFu, c, cr), 1);
        a ^= d;
        const u64 r = rotl64_var(a, rot);
        const u64 b0 = __shfl_sync(0xFFFFFFFFu, r, p0), b1 = __shfl_sync(0xFFFFFFFFu, r, p1),
                  b2 = __shfl_sync(0xFFFFFFFFu, r, p2);
        a = b0 ^ (~b1 & b2);
        if (l == 0) a ^= KECCAK_RC[round];
    }
    return a;
}

__device__ __forceinline__ void wtx_load(WarpTx& t, const TxState* g) {
    const unsigned l = wtx_lane();
    t.h = l < 25 ? g->hasher[l] : 0;
    t.r = l < 25 ? g->reader[l] : 0;
    t.hpos = g->hpos;
    t.rpos = g->rpos;
    t.has_reader = g->has_reader;
    t.err = g->err;
    t.deg = g->deg;
    t.narg_len = g->narg_len;
    t.hints_len = g->hints_len;
    t.narg_cap = g->narg_cap;
    t.hints_cap = g->hints_cap;
    t.narg = g->narg;
    t.hints = g->hints;
}
__device__ __forceinline__ void wtx_store(const WarpTx& t, TxState* g) {
    const unsigned l = wtx_lane();
    if (l < 25) {
        g->hasher[l] = t.h;
        g->reader[l] = t.r;
    }
    if (l == 0) {
        g->hpos = t.hpos;
        g->rpos = t.rpos;
        g->has_reader = t.has_reader;
        g->err = t.err;
        g->deg = t.deg;
        g->narg_len = t.narg_len;
        g->hints_len = t.hints_len;
        g->narg_cap = t.narg_cap;
        g->hints_cap = t.hints_cap;
        g->narg = t.narg;
        g->hints = t.hints;
    }
    __syncwarp();
}

// absorb: continue the hasher; a pending reader is dropped.
__device__ __forceinline__ void wtx_absorb_byte(WarpTx& t, u8 v) {
    if (wtx_lane() == (t.hpos >> 3)) t.h ^= (u64)v << (8 * (t.hpos & 7));
    if (++t.hpos == TX_RATE) {
        t.h = keccak_f1600_warp(t.h);
        t.hpos = 0;
    }
}
__device__ __forceinline__ void wtx_absorb_words(WarpTx& t, const u64* w, unsigned nw) {
    t.has_reader = 0;
    for (unsigned i = 0; i < nw; ++i) {
        const u64 v = w[i];
        if ((t.hpos & 7) == 0) {
            if (wtx_lane() == (t.hpos >> 3)) t.h ^= v;
            t.hpos += 8;
            if (t.hpos == TX_RATE) {
                t.h = keccak_f1600_warp(t.h);
                t.hpos = 0;
            }
        } else {
#pragma unroll 1
            for (int b = 0; b < 8; ++b) wtx_absorb_byte(t, (u8)(v >> (8 * b)));
        }
    }
}
__device__ __forceinline__ void wtx_absorb_bytes(WarpTx& t, const u8* src, unsigned n) {
    t.has_reader = 0;
    for (unsigned i = 0; i < n; ++i) wtx_absorb_byte(t, src[i]);
}

// The first squeeze after an absorb finalises a copy of the hasher.
__device__ __forceinline__ void wtx_reader(WarpTx& t) {
    if (t.has_reader) return;
    const unsigned l = wtx_lane();
    u64 r = t.h;
    if (l == (t.hpos >> 3)) r ^= (u64)0x1F << (8 * (t.hpos & 7));
    if (l == (TX_RATE - 1) >> 3) r ^= (u64)0x80 << (8 * ((TX_RATE - 1) & 7));
    t.r = keccak_f1600_warp(r);
    t.rpos = 0;
    t.has_reader = 1;
}
// Next 8 squeezed bytes as a LE word (any alignment); the result is warp-uniform.
__device__ __forceinline__ u64 wtx_squeeze_word(WarpTx& t) {
    wtx_reader(t);
    if ((t.rpos & 7) == 0) {
        if (t.rpos == TX_RATE) {
            t.r = keccak_f1600_warp(t.r);
            t.rpos = 0;
        }
        const u64 v = __shfl_sync(0xFFFFFFFFu, t.r, t.rpos >> 3);
        t.rpos += 8;
        return v;
    }
    u64 v = 0;
#pragma unroll 1
    for (int b = 0; b < 8; ++b) {
        if (t.rpos == TX_RATE) {
            t.r = keccak_f1600_warp(t.r);
            t.rpos = 0;
        }
        const u64 w = __shfl_sync(0xFFFFFFFFu, t.r, t.rpos >> 3);
        v |= ((w >> (8 * (t.rpos & 7))) & 0xFF) << (8 * b);
        ++t.rpos;
    }
    return v;
}
// n squeezed bytes into dst (shared or global memory), written by the warp.
__device__ __forceinline__ void wtx_squeeze_bytes(WarpTx& t, u8* dst, unsigned n) {
    if (n == 0) return;
    wtx_reader(t);
    const unsigned l = wtx_lane();
    unsigned done = 0;
    while (done < n) {
        if (t.rpos == TX_RATE) {
            t.r = keccak_f1600_warp(t.r);
            t.rpos = 0;
        }
        const unsigned take = min(n - done, TX_RATE - t.rpos);
        // every lane runs the same iterations so that all shuffles are full-warp
        for (unsigned k0 = 0; k0 < take; k0 += 32) {
            const unsigned k = k0 + l;
            const unsigned pos = t.rpos + (k < take ? k : take - 1);
            const u64 w = __shfl_sync(0xFFFFFFFFu, t.r, pos >> 3);
            if (k < take) dst[done + k] = (u8)(w >> (8 * (pos & 7)));
        }
        done += take;
        t.rpos += take;
    }
    __syncwarp();
}

__device__ __forceinline__ void wtx_narg_append(WarpTx& t, const u8* src, unsigned n) {
    if (t.narg_len + n > t.narg_cap) {
        t.err |= TX_ERR_NARG_OVERFLOW;
        return;
    }
    const unsigned l = wtx_lane();
    for (unsigned i = l; i < n; i += 32) t.narg[t.narg_len + i] = src[i];
    t.narg_len += n;
}
__device__ __forceinline__ void wtx_message_words(WarpTx& t, const u64* w, unsigned nw) {
    wtx_absorb_words(t, w, nw);
    wtx_narg_append(t, reinterpret_cast<const u8*>(w), 8 * nw);
}
__device__ __forceinline__ void wtx_message_e3(WarpTx& t, E3 v) {
    u64 w[3] = {v.c0, v.c1, v.c2};
    wtx_message_words(t, w, 3);
}
__device__ __forceinline__ void wtx_message_u64(WarpTx& t, u64 v) { wtx_message_words(t, &v, 1); }

// 40 squeezed bytes as a LE integer mod p (five words folded from the top).
__device__ __forceinline__ u64 wtx_challenge_base(WarpTx& t) {
    u64 w[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) w[i] = wtx_squeeze_word(t);
    u64 acc = gl_reduce(w[4], 0);
    for (int i = 3; i >= 0; --i) acc = gl_reduce(w[i], acc);
    return acc;
}

// ncomp (<= 3) consecutive base-field challenges, lane-parallel when their
// 40 ncomp bytes start word-aligned inside the current reader block: lane k <
// 5 ncomp takes squeezed word k and scales it by 2^(64 (k mod 5)) mod p (the
// powers are 1, 2^32 - 1, p - 2^32, 1, 2^32 - 1), and lane c sums the five
// terms of challenge c -- the integer sum_i w_i 2^(64 i) mod p that the
// word-by-word fold above computes.  Otherwise the challenges are squeezed
// word by word.  Returns challenge c in component c.
__device__ __forceinline__ E3 wtx_challenges(WarpTx& t, u32 ncomp) {
    wtx_reader(t);
    const unsigned l = wtx_lane();
    if ((t.rpos & 7) == 0 && t.rpos + 40 * ncomp <= TX_RATE) {
        const u32 k = l < 5 * ncomp ? l : 0;
        const u64 w = __shfl_sync(0xFFFFFFFFu, t.r, (t.rpos >> 3) + k);
        const u32 i = k % 5;
        const u64 scale = (i == 0 || i == 3) ? 1ull : (i == 2 ? GL_P - (1ull << 32) : GL_EPS);
        const u64 term = gl_mul(w, scale);
        const u32 src = l < ncomp ? 5 * l : 0;
        u64 s = __shfl_sync(0xFFFFFFFFu, term, src);
#pragma unroll 1
        for (u32 q = 1; q < 5; ++q) s = gl_add(s, __shfl_sync(0xFFFFFFFFu, term, src + q));
        t.rpos += 40 * ncomp;
        const u64 c0 = __shfl_sync(0xFFFFFFFFu, s, 0);
        const u64 c1 = __shfl_sync(0xFFFFFFFFu, s, 1);
        const u64 c2 = __shfl_sync(0xFFFFFFFFu, s, 2);
        return E3{c0, ncomp > 1 ? c1 : 0, ncomp > 2 ? c2 : 0};
    }
    E3 r{0, 0, 0};
    r.c0 = wtx_challenge_base(t);
    if (ncomp > 1) r.c1 = wtx_challenge_base(t);
    if (ncomp > 2) r.c2 = wtx_challenge_base(t);
    return r;
}
__device__ __forceinline__ E3 wtx_challenge_e3(WarpTx& t) { return wtx_challenges(t, 3); }

// Elements of the protocol's target field.  With the base field as target
// (Identity<Goldilocks>) its elements are carried as Ext3 values (x, 0, 0) --
// a subfield, so every kernel's arithmetic is unchanged -- and cross the
// transcript as one 8-byte word / one 40-byte challenge; GoldilocksExt2
// elements are carried as (c0, c1, 0) (products folded by e2_fold) and cross
// it as two words / two 40-byte chunks (transcript.hpp:375-453).
__device__ __forceinline__ E3 wtx_challenge_t(WarpTx& t) {
    return wtx_challenges(t, t.deg == 1 ? 1u : (t.deg == 2 ? 2u : 3u));
}
__device__ __forceinline__ void wtx_message_t(WarpTx& t, E3 v) {
    if (t.deg == 1) {
        if (v.c1 | v.c2) t.err |= TX_ERR_FIELD;  // outside the base field: caller input was not base-field
        wtx_message_u64(t, v.c0);
    } else if (t.deg == 2) {
        if (v.c2) t.err |= TX_ERR_FIELD;  // outside GoldilocksExt2's (c0, c1)
        u64 w[2] = {v.c0, v.c1};
        wtx_message_words(t, w, 2);
    } else {
        wtx_message_e3(t, v);
    }
}

// geometric_challenge (geometric_challenge.hpp:39-44): [] / [1] / squeeze x ->
// [1, x, x^2, ...]; the powers are formed 32 at a time (lane k: x^(32 j + k)).
__device__ __forceinline__ void wtx_geometric(WarpTx& t, E3* out, int count) {
    if (count <= 0) return;
    const unsigned l = wtx_lane();
    if (count == 1) {
        if (l == 0) out[0] = e3_one();
        __syncwarp();
        return;
    }
    const E3 x = wtx_challenge_t(t);
    // lane k: x^k by an in-warp prefix product (Hillis-Steele on multipliers;
    // rolled: one copy of the product's code to fetch)
    E3 p = l == 0 ? e3_one() : x;
#pragma unroll 1
    for (int o = 1; o < 32; o <<= 1) {
        const E3 q{__shfl_up_sync(0xFFFFFFFFu, p.c0, o), __shfl_up_sync(0xFFFFFFFFu, p.c1, o),
                   __shfl_up_sync(0xFFFFFFFFu, p.c2, o)};
        if (l >= (unsigned)o) p = ef_mul(p, q, t.deg == 2);
    }
    // x^32 = (x^31) * x
    E3 x31{__shfl_sync(0xFFFFFFFFu, p.c0, 31), __shfl_sync(0xFFFFFFFFu, p.c1, 31), __shfl_sync(0xFFFFFFFFu, p.c2, 31)};
    const E3 x32 = ef_mul(x31, x, t.deg == 2);
    for (int base = 0; base < count; base += 32) {
        if (base + (int)l < count) out[base + l] = p;
        p = ef_mul(p, x32, t.deg == 2);
    }
    __syncwarp();
}

// Warp-wide field sum (exact; association order free).
__device__ __forceinline__ E3 wtx_sum(E3 v) { return e3_warp_sum(v); }

}  // namespace wg
