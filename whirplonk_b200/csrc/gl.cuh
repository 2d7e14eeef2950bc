// gl.cuh -- Goldilocks (p = 2^64 - 2^32 + 1) and its cubic extension
// Fp[X]/(X^3 - 2) on the device.
//
// Field semantics follow the reference's host types
// (cpp/include/whir/algebra/goldilocks.hpp:54-202, goldilocks_ext3.hpp:33-137):
// every value is kept canonical in [0, p).  The 64x64 product is formed with
// mul.lo/mul.hi and reduced with the sparse-prime identities
//   2^64 == 2^32 - 1,   2^96 == -1   (mod p).
// This is exact integer work for the CUDA cores; there is nothing for the
// tensor cores here.
#pragma once
#include <cstdint>

namespace wg {

typedef uint64_t u64;
typedef unsigned int u32;

constexpr u64 GL_P = 0xFFFFFFFF00000001ull;
constexpr u64 GL_EPS = 0xFFFFFFFFull;  // 2^64 mod p

// Host forms (also the device fallback for the reference formulas).
__host__ __device__ __forceinline__ u64 gl_add_ref(u64 a, u64 b) {
    u64 s = a + b;
    if (s < a) s += GL_EPS;  // cannot overflow again: s + EPS < p when a, b < p
    if (s >= GL_P) s -= GL_P;
    return s;
}
__host__ __device__ __forceinline__ u64 gl_sub_ref(u64 a, u64 b) {
    u64 d = a - b;
    if (a < b) d += GL_P;  // wraps back into [0, p)
    return d;
}
__host__ __device__ __forceinline__ u64 gl_neg(u64 a) { return a ? GL_P - a : 0; }

__host__ __device__ __forceinline__ u64 gl_reduce(u64 lo, u64 hi) {
    u64 hh = hi >> 32, hl = hi & GL_EPS;
    u64 t = lo - hh;
    if (lo < hh) t -= GL_EPS;         // borrowed 2^64 == EPS
    u64 m = (hl << 32) - hl;          // hl * EPS
    u64 s = t + m;
    if (s < t) s += GL_EPS;
    if (s >= GL_P) s -= GL_P;
    return s;
}

// Device forms on 32-bit carry chains.  A borrow or carry out of the top limb is
// worth 2^64 == EPS (mod p).  After a subtract chain `subc.u32 m, 0, 0` turns
// the borrow into the mask m = 0 or 0xFFFFFFFF = EPS; after an add chain the
// carry is read with `addc` and negated.  The mask is then added or subtracted.

// a + b for canonical a, b: d = a - (p - b); a borrow means a + b < p, and the
// wrapped difference is then corrected by -EPS (== +p - 2^64).
__device__ __forceinline__ u64 gl_add(u64 a, u64 b) {
    unsigned d0, d1;
    asm("{\n\t.reg .u32 n0, n1, m;\n\t"
        "sub.cc.u32 n0, 1, %4;\n\t"          // n = p - b  (p = 0xFFFFFFFF:00000001)
        "subc.u32 n1, 0xFFFFFFFF, %5;\n\t"
        "sub.cc.u32 %0, %2, n0;\n\t"         // d = a - n
        "subc.cc.u32 %1, %3, n1;\n\t"
        "subc.u32 m, 0, 0;\n\t"              // m = borrow ? EPS : 0
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t}"
        : "=&r"(d0), "=&r"(d1)
        : "r"((unsigned)a), "r"((unsigned)(a >> 32)), "r"((unsigned)b), "r"((unsigned)(b >> 32)));
    return ((u64)d1 << 32) | d0;
}
// a - b for canonical a, b; on borrow subtract EPS (== add p - 2^64).
__device__ __forceinline__ u64 gl_sub(u64 a, u64 b) {
    unsigned d0, d1;
    asm("{\n\t.reg .u32 m;\n\t"
        "sub.cc.u32 %0, %2, %4;\n\t"
        "subc.cc.u32 %1, %3, %5;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t}"
        : "=&r"(d0), "=&r"(d1)
        : "r"((unsigned)a), "r"((unsigned)(a >> 32)), "r"((unsigned)b), "r"((unsigned)(b >> 32)));
    return ((u64)d1 << 32) | d0;
}
// (hi 2^64 + lo) mod p, canonical, for any 64-bit lo, hi:
//   x == lo - hh + hl * (2^32 - 1)   with hi = hh 2^32 + hl.
__device__ __forceinline__ u64 gl_reduce_dev(u64 lo, u64 hi) {
    unsigned r0, r1;
    asm("{\n\t.reg .u32 r2, r3, m;\n\t"
        "mov.b64 {%0, %1}, %2;\n\t"
        "mov.b64 {r2, r3}, %3;\n\t"
        // t = lo - hh ; on borrow subtract EPS
        "sub.cc.u32 %0, %0, r3;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        // u = hl * 2^32 - hl  ->  (r3 : m)
        "sub.cc.u32 m, 0, r2;\n\t"
        "subc.u32 r3, r2, 0;\n\t"
        // s = t + u ; on carry add EPS.  The carry of an add chain is read with
        // addc (subc's borrow-in is only defined after a subtract chain).
        "add.cc.u32 %0, %0, m;\n\t"
        "addc.cc.u32 %1, %1, r3;\n\t"
        "addc.u32 m, 0, 0;\n\t"
        "sub.u32 m, 0, m;\n\t"
        "add.cc.u32 %0, %0, m;\n\t"
        "addc.u32 %1, %1, 0;\n\t"
        // canonical: s >= p  <=>  s + EPS carries out; then keep s + EPS (mod 2^64)
        "add.cc.u32 r2, %0, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 r3, %1, 0;\n\t"
        "addc.u32 m, 0, 0;\n\t"
        "sub.u32 m, 0, m;\n\t"
        "add.cc.u32 %0, %0, m;\n\t"
        "addc.u32 %1, %1, 0;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "l"(lo), "l"(hi));
    return ((u64)r1 << 32) | r0;
}
// (a * b) mod p, canonical output for any 64-bit a, b.  The 128-bit product
// is left to the compiler's 64-bit multiply (measured ~2 % faster on B200 than
// a hand-written 32-bit limb chain in a butterfly-like mix).
__device__ __forceinline__ u64 gl_mul(u64 a, u64 b) {
    u64 lo, hi;
    asm("mul.lo.u64 %0, %2, %3;\n\tmul.hi.u64 %1, %2, %3;" : "=l"(lo), "=l"(hi) : "l"(a), "l"(b));
    return gl_reduce_dev(lo, hi);
}
// The same reduction with its add-carry corrections moved to the FMA pipe: the
// carry c of an add becomes `mad.wide.u32 s, c, EPS, s` (s + c EPS cannot wrap
// there), and hl * EPS one wide multiply.  Bit-identical to gl_reduce_dev; it
// trades ~4 ALU-pipe instructions for ~3 FMA-pipe ones, which pays in kernels
// whose ALU pipe is the bottleneck while the FMA pipe idles (the NTT passes).
__device__ __forceinline__ u64 gl_reduce_fma(u64 lo, u64 hi) {
    u64 s;
    asm("{\n\t.reg .u32 l0, l1, h0, h1, t0, t1, m, c;\n\t.reg .u64 t, u;\n\t"
        "mov.b64 {l0, l1}, %1;\n\t"
        "mov.b64 {h0, h1}, %2;\n\t"
        // t = lo - hh ; on borrow subtract EPS
        "sub.cc.u32 t0, l0, h1;\n\t"
        "subc.cc.u32 t1, l1, 0;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 t0, t0, m;\n\t"
        "subc.u32 t1, t1, 0;\n\t"
        "mov.b64 t, {t0, t1};\n\t"
        // s = t + hl * EPS ; on carry add EPS
        "mul.wide.u32 u, h0, 0xFFFFFFFF;\n\t"
        "add.cc.u64 %0, t, u;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "mad.wide.u32 %0, c, 0xFFFFFFFF, %0;\n\t"
        // canonical: s >= p  <=>  s + EPS carries; then s + EPS (mod 2^64) = s - p
        "add.cc.u64 t, %0, 0xFFFFFFFF;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "mad.wide.u32 %0, c, 0xFFFFFFFF, %0;\n\t}"
        : "=l"(s)
        : "l"(lo), "l"(hi));
    return s;
}
__device__ __forceinline__ u64 gl_mul_fma(u64 a, u64 b) {
    u64 lo, hi;
    asm("mul.lo.u64 %0, %2, %3;\n\tmul.hi.u64 %1, %2, %3;" : "=l"(lo), "=l"(hi) : "l"(a), "l"(b));
    return gl_reduce_fma(lo, hi);
}
__host__ __forceinline__ u64 gl_mul_host(u64 a, u64 b) {
    unsigned __int128 x = (unsigned __int128)a * b;
    return gl_reduce((u64)x, (u64)(x >> 64));
}
__device__ __forceinline__ u64 gl_pow(u64 b, u64 e) {
    u64 r = 1;
    while (e) {
        if (e & 1) r = gl_mul(r, b);
        b = gl_mul(b, b);
        e >>= 1;
    }
    return r;
}
__host__ inline u64 gl_pow_host(u64 b, u64 e) {
    u64 r = 1;
    while (e) {
        if (e & 1) r = gl_mul_host(r, b);
        b = gl_mul_host(b, b);
        e >>= 1;
    }
    return r;
}

struct E3 {
    u64 c0, c1, c2;
};
__host__ __device__ __forceinline__ E3 e3_zero() { return E3{0, 0, 0}; }
__host__ __device__ __forceinline__ E3 e3_one() { return E3{1, 0, 0}; }
__host__ __device__ __forceinline__ E3 e3_base(u64 a) { return E3{a, 0, 0}; }
__device__ __forceinline__ E3 e3_add(E3 a, E3 b) { return E3{gl_add(a.c0, b.c0), gl_add(a.c1, b.c1), gl_add(a.c2, b.c2)}; }
__device__ __forceinline__ E3 e3_sub(E3 a, E3 b) { return E3{gl_sub(a.c0, b.c0), gl_sub(a.c1, b.c1), gl_sub(a.c2, b.c2)}; }
__host__ __device__ __forceinline__ bool e3_eq(E3 a, E3 b) { return a.c0 == b.c0 && a.c1 == b.c1 && a.c2 == b.c2; }
// 192-bit accumulator for sums of 64x64 products (delayed reduction).
struct Acc192 {
    u64 w0, w1, w2;
};
__device__ __forceinline__ void acc_mul(Acc192& x, u64 a, u64 b) {
    asm("{\n\t.reg .u64 l, h;\n\t"
        "mul.lo.u64 l, %3, %4;\n\t"
        "mul.hi.u64 h, %3, %4;\n\t"
        "add.cc.u64 %0, %0, l;\n\t"
        "addc.cc.u64 %1, %1, h;\n\t"
        "addc.u64 %2, %2, 0;\n\t}"
        : "+l"(x.w0), "+l"(x.w1), "+l"(x.w2)
        : "l"(a), "l"(b));
}
__device__ __forceinline__ Acc192 acc_product(u64 a, u64 b) {
    Acc192 x;
    asm("mul.lo.u64 %0, %2, %3;\n\t"
        "mul.hi.u64 %1, %2, %3;"
        : "=l"(x.w0), "=l"(x.w1)
        : "l"(a), "l"(b));
    x.w2 = 0;
    return x;
}
// x += a * b with the full 128-bit product formed on 32-bit limbs.
__device__ __forceinline__ void acc_mac(Acc192& x, u64 a, u64 b) {
    unsigned r0, r1, r2, r3;
    asm("mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
        : "r"((unsigned)a), "r"((unsigned)(a >> 32)), "r"((unsigned)b), "r"((unsigned)(b >> 32)));
    asm("add.cc.u64 %0, %0, %3;\n\t"
        "addc.cc.u64 %1, %1, %4;\n\t"
        "addc.u64 %2, %2, 0;"
        : "+l"(x.w0), "+l"(x.w1), "+l"(x.w2)
        : "l"(((u64)r1 << 32) | r0), "l"(((u64)r3 << 32) | r2));
}
__device__ __forceinline__ void acc_add(Acc192& x, const Acc192& y) {
    asm("add.cc.u64 %0, %0, %3;\n\t"
        "addc.cc.u64 %1, %1, %4;\n\t"
        "addc.u64 %2, %2, %5;"
        : "+l"(x.w0), "+l"(x.w1), "+l"(x.w2)
        : "l"(y.w0), "l"(y.w1), "l"(y.w2));
}
__device__ __forceinline__ void acc_double(Acc192& x) {
    x.w2 = (x.w2 << 1) | (x.w1 >> 63);
    x.w1 = (x.w1 << 1) | (x.w0 >> 63);
    x.w0 <<= 1;
}
// x mod p for x = w0 + w1 2^64 + w2 2^128 with w2 < 2^32:
// 2^64 == EPS and 2^128 == -2^32 (mod p); w2 2^32 < p is already canonical.
__device__ __forceinline__ u64 acc_reduce(const Acc192& x) {
    return gl_sub(gl_reduce_dev(x.w0, x.w1), x.w2 << 32);
}

__device__ __forceinline__ E3 e3_mul(E3 a, E3 b) {
    // X^3 = 2:  c0 = a0b0 + 2(a1b2 + a2b1), c1 = a0b1 + a1b0 + 2 a2b2, c2 = a0b2 + a1b1 + a2b0
    Acc192 s0 = acc_product(a.c1, b.c2);
    acc_mul(s0, a.c2, b.c1);
    acc_double(s0);
    acc_mul(s0, a.c0, b.c0);
    Acc192 s1 = acc_product(a.c2, b.c2);
    acc_double(s1);
    acc_mul(s1, a.c0, b.c1);
    acc_mul(s1, a.c1, b.c0);
    Acc192 s2 = acc_product(a.c0, b.c2);
    acc_mul(s2, a.c1, b.c1);
    acc_mul(s2, a.c2, b.c0);
    return E3{acc_reduce(s0), acc_reduce(s1), acc_reduce(s2)};
}
// Delayed-reduction Ext3 multiply-accumulate: sum a_k b_k over many k, reduced once.
struct E3Acc {
    Acc192 s0, s1, s2;  // plain terms of c0, c1, c2
    Acc192 d0, d1;      // terms of c0, c1 that carry the factor 2 of X^3 = 2
};
__device__ __forceinline__ E3Acc e3acc_zero() { return E3Acc{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}; }
__device__ __forceinline__ void e3acc_mac(E3Acc& x, const E3& a, const E3& b) {
    acc_mac(x.s0, a.c0, b.c0);
    acc_mac(x.d0, a.c1, b.c2);
    acc_mac(x.d0, a.c2, b.c1);
    acc_mac(x.s1, a.c0, b.c1);
    acc_mac(x.s1, a.c1, b.c0);
    acc_mac(x.d1, a.c2, b.c2);
    acc_mac(x.s2, a.c0, b.c2);
    acc_mac(x.s2, a.c1, b.c1);
    acc_mac(x.s2, a.c2, b.c0);
}
__device__ __forceinline__ void e3acc_mac_base(E3Acc& x, const E3& a, u64 b) {
    acc_mac(x.s0, a.c0, b);
    acc_mac(x.s1, a.c1, b);
    acc_mac(x.s2, a.c2, b);
}
// Valid while every accumulator's top word stays below 2^31 (< 2^31 products).
__device__ __forceinline__ E3 e3acc_reduce(E3Acc x) {
    acc_double(x.d0);
    acc_double(x.d1);
    acc_add(x.s0, x.d0);
    acc_add(x.s1, x.d1);
    return E3{acc_reduce(x.s0), acc_reduce(x.s1), acc_reduce(x.s2)};
}
__device__ __forceinline__ E3 e3_mul_base(E3 a, u64 b) { return E3{gl_mul(a.c0, b), gl_mul(a.c1, b), gl_mul(a.c2, b)}; }
__device__ __forceinline__ E3 e3_pow(E3 b, u64 e) {
    E3 r = e3_one();
    while (e) {
        if (e & 1) r = e3_mul(r, b);
        b = e3_mul(b, b);
        e >>= 1;
    }
    return r;
}

// Basefield<GoldilocksExt2> (goldilocks_ext2.hpp: Fp[X]/(X^2 - 7)) rides on
// the same representation: an Ext2 value is (c0, c1, 0).  For two such values
// the X^3 = 2 rule of e3_mul / E3Acc leaves the plain polynomial product
// (a0 b0, a0 b1 + a1 b0, a1 b1) -- no term of degree 3 or 4 arises -- and
// X^2 = 7 folds the X^2 coefficient back: e2_fold.  It is the identity on
// values whose c2 is zero, so an Ext2 proof applies it after every product.
constexpr u64 GL_EXT2_NR = 7;
__device__ __forceinline__ E3 e2_fold(E3 v) { return E3{gl_add(v.c0, gl_mul(v.c2, GL_EXT2_NR)), v.c1, 0}; }
// Product in the target field: Ext3, or Ext2 when ext2 is set.
__device__ __forceinline__ E3 ef_mul(E3 a, E3 b, bool ext2) {
    const E3 r = e3_mul(a, b);
    return ext2 ? e2_fold(r) : r;
}
__device__ __forceinline__ E3 ef_fix(E3 v, bool ext2) { return ext2 ? e2_fold(v) : v; }
__device__ __forceinline__ E3 ef_pow(E3 b, u64 e, bool ext2) {
    E3 r = e3_one();
    while (e) {
        if (e & 1) r = ef_mul(r, b, ext2);
        b = ef_mul(b, b, ext2);
        e >>= 1;
    }
    return r;
}

// Ext3 vectors live in HBM as three component planes (structure of arrays):
// every component access is a coalesced 8-byte stream.
struct E3Planes {
    u64* c0;
    u64* c1;
    u64* c2;
};
__device__ __forceinline__ E3 e3_load(const E3Planes& p, u64 i) { return E3{p.c0[i], p.c1[i], p.c2[i]}; }
__device__ __forceinline__ void e3_store(const E3Planes& p, u64 i, E3 v) { p.c0[i] = v.c0; p.c1[i] = v.c1; p.c2[i] = v.c2; }

// Warp-wide field sum (exact; any association order gives the same value).
// The loops stay rolled: these sums run once per warp per launch, mostly in
// single-warp kernels whose time goes to fetching straight-line code.
__device__ __forceinline__ u64 gl_warp_sum(u64 v) {
#pragma unroll 1
    for (int o = 16; o > 0; o >>= 1) v = gl_add(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
__device__ __forceinline__ E3 e3_warp_sum(E3 v) {
#pragma unroll 1
    for (int o = 16; o > 0; o >>= 1) {
        v.c0 = gl_add(v.c0, __shfl_xor_sync(0xFFFFFFFFu, v.c0, o));
        v.c1 = gl_add(v.c1, __shfl_xor_sync(0xFFFFFFFFu, v.c1, o));
        v.c2 = gl_add(v.c2, __shfl_xor_sync(0xFFFFFFFFu, v.c2, o));
    }
    return v;
}

}  // namespace wg
