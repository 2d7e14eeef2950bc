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

__host__ __device__ __forceinline__ u64 gl_add(u64 a, u64 b) {
    u64 s = a + b;
    if (s < a) s += GL_EPS;  // cannot overflow again: s + EPS < p when a, b < p
    if (s >= GL_P) s -= GL_P;
    return s;
}
__host__ __device__ __forceinline__ u64 gl_sub(u64 a, u64 b) {
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
__device__ __forceinline__ u64 gl_mul(u64 a, u64 b) { return gl_reduce(a * b, __umul64hi(a, b)); }
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
__host__ __device__ __forceinline__ E3 e3_add(E3 a, E3 b) { return E3{gl_add(a.c0, b.c0), gl_add(a.c1, b.c1), gl_add(a.c2, b.c2)}; }
__host__ __device__ __forceinline__ E3 e3_sub(E3 a, E3 b) { return E3{gl_sub(a.c0, b.c0), gl_sub(a.c1, b.c1), gl_sub(a.c2, b.c2)}; }
__host__ __device__ __forceinline__ bool e3_eq(E3 a, E3 b) { return a.c0 == b.c0 && a.c1 == b.c1 && a.c2 == b.c2; }
__device__ __forceinline__ E3 e3_mul(E3 a, E3 b) {
    // X^3 = 2:  c0 = a0b0 + 2(a1b2 + a2b1), c1 = a0b1 + a1b0 + 2 a2b2, c2 = a0b2 + a1b1 + a2b0
    u64 t12 = gl_add(gl_mul(a.c1, b.c2), gl_mul(a.c2, b.c1));
    u64 t22 = gl_mul(a.c2, b.c2);
    E3 r;
    r.c0 = gl_add(gl_mul(a.c0, b.c0), gl_add(t12, t12));
    r.c1 = gl_add(gl_add(gl_mul(a.c0, b.c1), gl_mul(a.c1, b.c0)), gl_add(t22, t22));
    r.c2 = gl_add(gl_add(gl_mul(a.c0, b.c2), gl_mul(a.c1, b.c1)), gl_mul(a.c2, b.c0));
    return r;
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
__device__ __forceinline__ u64 gl_warp_sum(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = gl_add(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
__device__ __forceinline__ E3 e3_warp_sum(E3 v) { return E3{gl_warp_sum(v.c0), gl_warp_sum(v.c1), gl_warp_sum(v.c2)}; }

}  // namespace wg
