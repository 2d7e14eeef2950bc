// blake3.cuh -- BLAKE3 compression on the device (public BLAKE3 spec).
//
// Most messages of the WHIR path are single chunks whose length is a multiple
// of 64 bytes: codeword rows (128 B base, 384 B Ext3), Merkle parents and
// proof-of-work inputs (64 B).  Each such hash is a chain of compressions with
// counter 0, block_len 64, CHUNK_START on the first block and CHUNK_END|ROOT on
// the last -- the reference's blake3_hash_many call
// (cpp/include/whir/hash/blake3_engine.hpp:90-199).  Rows of several committed
// vectors can span several chunks; those use the chunk counter and the PARENT
// flag of the tree mode.  ~700 integer ops per compression (add, xor,
// funnel-shift rotates), all on the CUDA cores.
#pragma once
#include <cstdint>

namespace wg {

constexpr unsigned B3_IV0 = 0x6A09E667u, B3_IV1 = 0xBB67AE85u, B3_IV2 = 0x3C6EF372u, B3_IV3 = 0xA54FF53Au;
constexpr unsigned B3_IV4 = 0x510E527Fu, B3_IV5 = 0x9B05688Cu, B3_IV6 = 0x1F83D9ABu, B3_IV7 = 0x5BE0CD19u;
constexpr unsigned B3_CHUNK_START = 1u, B3_CHUNK_END = 2u, B3_PARENT = 4u, B3_ROOT = 8u;

// Message word used by G-call slot s (0..15) in round r: the spec's message
// permutation applied r times.  Folded to a constant after unrolling.
__host__ __device__ constexpr int b3_perm(int s) {
    return s == 0 ? 2 : s == 1 ? 6 : s == 2 ? 3 : s == 3 ? 10 : s == 4 ? 7 : s == 5 ? 0 : s == 6 ? 4 : s == 7 ? 13
         : s == 8 ? 1 : s == 9 ? 11 : s == 10 ? 12 : s == 11 ? 5 : s == 12 ? 9 : s == 13 ? 14 : s == 14 ? 15 : 8;
}
__host__ __device__ constexpr int b3_msg(int r, int s) { return r == 0 ? s : b3_msg(r - 1, b3_perm(s)); }

__device__ __forceinline__ unsigned b3_rotr(unsigned v, int s) { return __funnelshift_r(v, v, s); }

#define WG_B3_G(a, b, c, d, x, y)                  \
    do {                                           \
        a = a + b + (x); d = b3_rotr(d ^ a, 16);   \
        c = c + d;       b = b3_rotr(b ^ c, 12);   \
        a = a + b + (y); d = b3_rotr(d ^ a, 8);    \
        c = c + d;       b = b3_rotr(b ^ c, 7);    \
    } while (0)

// One round of the compression function; the message schedule of round R is
// resolved at compile time (constexpr locals), so `m` stays in registers.
template <int R>
__device__ __forceinline__ void b3_round(unsigned& v0, unsigned& v1, unsigned& v2, unsigned& v3, unsigned& v4,
                                         unsigned& v5, unsigned& v6, unsigned& v7, unsigned& v8, unsigned& v9,
                                         unsigned& v10, unsigned& v11, unsigned& v12, unsigned& v13, unsigned& v14,
                                         unsigned& v15, const unsigned m[16]) {
    constexpr int s0 = b3_msg(R, 0), s1 = b3_msg(R, 1), s2 = b3_msg(R, 2), s3 = b3_msg(R, 3);
    constexpr int s4 = b3_msg(R, 4), s5 = b3_msg(R, 5), s6 = b3_msg(R, 6), s7 = b3_msg(R, 7);
    constexpr int s8 = b3_msg(R, 8), s9 = b3_msg(R, 9), s10 = b3_msg(R, 10), s11 = b3_msg(R, 11);
    constexpr int s12 = b3_msg(R, 12), s13 = b3_msg(R, 13), s14 = b3_msg(R, 14), s15 = b3_msg(R, 15);
    WG_B3_G(v0, v4, v8, v12, m[s0], m[s1]);
    WG_B3_G(v1, v5, v9, v13, m[s2], m[s3]);
    WG_B3_G(v2, v6, v10, v14, m[s4], m[s5]);
    WG_B3_G(v3, v7, v11, v15, m[s6], m[s7]);
    WG_B3_G(v0, v5, v10, v15, m[s8], m[s9]);
    WG_B3_G(v1, v6, v11, v12, m[s10], m[s11]);
    WG_B3_G(v2, v7, v8, v13, m[s12], m[s13]);
    WG_B3_G(v3, v4, v9, v14, m[s14], m[s15]);
}

// cv <- first half of compress(cv, m, counter, block_len, flags); counters
// stay below 2^32 on this path (chunk index within one row).
__device__ __forceinline__ void b3_compress(unsigned cv[8], const unsigned m[16], unsigned flags, unsigned block_len = 64,
                                            unsigned counter = 0) {
    unsigned v0 = cv[0], v1 = cv[1], v2 = cv[2], v3 = cv[3], v4 = cv[4], v5 = cv[5], v6 = cv[6], v7 = cv[7];
    unsigned v8 = B3_IV0, v9 = B3_IV1, v10 = B3_IV2, v11 = B3_IV3;
    unsigned v12 = counter, v13 = 0, v14 = block_len, v15 = flags;
    b3_round<0>(v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15, m);
    b3_round<1>(v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15, m);
    b3_round<2>(v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15, m);
    b3_round<3>(v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15, m);
    b3_round<4>(v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15, m);
    b3_round<5>(v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15, m);
    b3_round<6>(v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12, v13, v14, v15, m);
    cv[0] = v0 ^ v8; cv[1] = v1 ^ v9; cv[2] = v2 ^ v10; cv[3] = v3 ^ v11;
    cv[4] = v4 ^ v12; cv[5] = v5 ^ v13; cv[6] = v6 ^ v14; cv[7] = v7 ^ v15;
}

__device__ __forceinline__ void b3_init(unsigned cv[8]) {
    cv[0] = B3_IV0; cv[1] = B3_IV1; cv[2] = B3_IV2; cv[3] = B3_IV3;
    cv[4] = B3_IV4; cv[5] = B3_IV5; cv[6] = B3_IV6; cv[7] = B3_IV7;
}

// Flags of block t of an nblocks-block single-chunk message.
__device__ __forceinline__ unsigned b3_flags(int t, int nblocks) {
    return (t == 0 ? B3_CHUNK_START : 0u) | (t == nblocks - 1 ? (B3_CHUNK_END | B3_ROOT) : 0u);
}

// BLAKE3 of a 64-byte message given as 16 LE words (Merkle parent, PoW input).
__device__ __forceinline__ void b3_hash64(const unsigned m[16], unsigned out[8]) {
    b3_init(out);
    b3_compress(out, m, B3_CHUNK_START | B3_CHUNK_END | B3_ROOT);
}

}  // namespace wg
