// sha256.cuh -- SHA-256 compression on the device (FIPS 180-4), the reference's
// second hash engine (cpp/include/whir/hash/sha2_engine.hpp:47-81): selected
// by a configuration's hash_id for leaves, Merkle parents and proof of work
// (irs_commit.hpp:62-74, whir.hpp:134-140).
//
// The round constants and the initial hash value are derived at compile time
// from their definitions: the first 32 fractional bits of the cube roots of the
// first 64 primes and of the square roots of the first 8 primes.  Message
// words are big-endian; digests are stored so that their bytes in memory are
// the digest's bytes.
#pragma once
#include <cstdint>

namespace wg {

__host__ __device__ constexpr unsigned long long sha_prime(int k) {
    unsigned long long n = 1;
    for (int found = -1; found < k;) {
        ++n;
        bool prime = true;
        for (unsigned long long d = 2; d * d <= n; ++d)
            if (n % d == 0) { prime = false; break; }
        if (prime) ++found;
    }
    return n;
}
// floor(root-th root of p with 32 fractional bits) mod 2^32, by bisection on x
// with x^root <= p 2^(32 root), the powers compared in 128-bit arithmetic.
__host__ __device__ constexpr unsigned sha_root_frac(unsigned long long p, int root) {
    using u128 = unsigned __int128;
    const u128 target = (u128)p << (32 * root);
    unsigned long long lo = 0, hi = 1ull << 40;
    while (lo + 1 < hi) {
        const unsigned long long mid = (lo + hi) / 2;
        u128 v = 1;
        for (int i = 0; i < root; ++i) v *= mid;
        if (v <= target) lo = mid;
        else hi = mid;
    }
    return (unsigned)lo;
}
#define WG_SHA_K4(i) sha_root_frac(sha_prime(i), 3), sha_root_frac(sha_prime(i + 1), 3), \
                     sha_root_frac(sha_prime(i + 2), 3), sha_root_frac(sha_prime(i + 3), 3)
__constant__ const unsigned SHA256_K[64] = {WG_SHA_K4(0),  WG_SHA_K4(4),  WG_SHA_K4(8),  WG_SHA_K4(12),
                                            WG_SHA_K4(16), WG_SHA_K4(20), WG_SHA_K4(24), WG_SHA_K4(28),
                                            WG_SHA_K4(32), WG_SHA_K4(36), WG_SHA_K4(40), WG_SHA_K4(44),
                                            WG_SHA_K4(48), WG_SHA_K4(52), WG_SHA_K4(56), WG_SHA_K4(60)};
#undef WG_SHA_K4

__device__ __forceinline__ unsigned sha_ror(unsigned x, int s) { return __funnelshift_r(x, x, s); }
__device__ __forceinline__ unsigned bswap32(unsigned x) { return __byte_perm(x, 0, 0x0123); }

#define WG_SHA_H(i) sha_root_frac(sha_prime(i), 2)
__constant__ const unsigned SHA256_H0[8] = {WG_SHA_H(0), WG_SHA_H(1), WG_SHA_H(2), WG_SHA_H(3),
                                            WG_SHA_H(4), WG_SHA_H(5), WG_SHA_H(6), WG_SHA_H(7)};
#undef WG_SHA_H

__device__ __forceinline__ void sha256_init(unsigned h[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = SHA256_H0[i];
}

// h <- compress(h, w) for one 64-byte block given as 16 big-endian words.
__device__ __forceinline__ void sha256_compress(unsigned h[8], const unsigned w_in[16]) {
    unsigned w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = w_in[i];
    unsigned a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
#pragma unroll
    for (int t = 0; t < 64; ++t) {
        unsigned wt;
        if (t < 16) {
            wt = w[t];
        } else {
            const unsigned x15 = w[(t - 15) & 15], x2 = w[(t - 2) & 15];
            const unsigned s0 = sha_ror(x15, 7) ^ sha_ror(x15, 18) ^ (x15 >> 3);
            const unsigned s1 = sha_ror(x2, 17) ^ sha_ror(x2, 19) ^ (x2 >> 10);
            wt = w[t & 15] + s0 + w[(t - 7) & 15] + s1;
            w[t & 15] = wt;
        }
        const unsigned t1 = hh + (sha_ror(e, 6) ^ sha_ror(e, 11) ^ sha_ror(e, 25)) + ((e & f) ^ (~e & g)) + SHA256_K[t] + wt;
        const unsigned t2 = (sha_ror(a, 2) ^ sha_ror(a, 13) ^ sha_ror(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}

// The padding block of a message of `bytes` bytes that ended on a block boundary.
__device__ __forceinline__ void sha256_pad_block(unsigned w[16], unsigned long long bytes) {
    w[0] = 0x80000000u;
#pragma unroll
    for (int i = 1; i < 14; ++i) w[i] = 0;
    w[14] = (unsigned)((bytes * 8) >> 32);
    w[15] = (unsigned)(bytes * 8);
}

// SHA-256 of a 64-byte message whose 16 words are given as little-endian
// loads of its bytes (a Merkle parent's two child digests, a PoW input).
__device__ __forceinline__ void sha256_hash64(const unsigned m_le[16], unsigned out_le[8]) {
    unsigned h[8], w[16];
    sha256_init(h);
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = bswap32(m_le[i]);
    sha256_compress(h, w);
    sha256_pad_block(w, 64);
    sha256_compress(h, w);
#pragma unroll
    for (int i = 0; i < 8; ++i) out_le[i] = bswap32(h[i]);
}

}  // namespace wg
