// transcript.cuh -- device-resident Fiat-Shamir transcript.
//
// Byte-for-byte the reference ProverState over a SHAKE128 duplex sponge
// (cpp/include/whir/transcript/transcript.hpp:80-139, 595-662):
//   * absorb(bytes)  continues the SHAKE128 hasher (rate 168 B);
//   * the first squeeze after an absorb finalises a *clone* of the hasher
//     (pad 0x1F .. 0x80, Keccak-f) and later squeezes keep reading that XOF
//     reader until the next absorb;
//   * prover_message(T) = absorb(raw LE bytes of T) + append them to narg;
//   * prover_hint(vector<T>) = u64 LE length + raw elements appended to hints,
//     prover_hint(Hash) = 32 raw bytes; hints are not absorbed;
//   * a base-field challenge decodes 40 squeezed bytes as a LE integer mod p,
//     an Ext3 challenge three such chunks (:375-453).
// The state lives in HBM between kernels so that the whole proof can run as
// one stream of kernels (and be captured in a CUDA graph) without the host ever
// reading a challenge back; within a kernel one warp carries it (wtx.cuh).
#pragma once
#include "gl.cuh"

namespace wg {

typedef unsigned char u8;

// Keccak-f[1600] constants, derived at compile time from their FIPS 202
// definitions (round-constant LFSR x^8+x^6+x^5+x^4+1; rho offsets
// (t+1)(t+2)/2 along the (x,y) -> (y, 2x+3y) orbit).
__host__ __device__ constexpr int keccak_rc_bit(int t) {
    int r = 0x80;  // R[0..7] with R[0] in bit 7
    for (int i = 1; i <= t % 255; ++i) {
        int r8 = r & 1;
        r >>= 1;
        if (r8) r ^= 0x8E;  // R[0], R[4], R[5], R[6]
    }
    return (t % 255 == 0) ? 1 : ((r >> 7) & 1);
}
__host__ __device__ constexpr unsigned long long keccak_rc(int round) {
    unsigned long long v = 0;
    for (int j = 0; j <= 6; ++j)
        if (keccak_rc_bit(j + 7 * round)) v |= 1ull << ((1 << j) - 1);
    return v;
}
__host__ __device__ constexpr int keccak_rho(int x, int y) {
    if (x == 0 && y == 0) return 0;
    int cx = 1, cy = 0;
    for (int t = 0; t < 24; ++t) {
        if (cx == x && cy == y) return ((t + 1) * (t + 2) / 2) % 64;
        int nx = cy, ny = (2 * cx + 3 * cy) % 5;
        cx = nx;
        cy = ny;
    }
    return 0;
}

__constant__ const unsigned long long KECCAK_RC[24] = {
    keccak_rc(0),  keccak_rc(1),  keccak_rc(2),  keccak_rc(3),  keccak_rc(4),  keccak_rc(5),
    keccak_rc(6),  keccak_rc(7),  keccak_rc(8),  keccak_rc(9),  keccak_rc(10), keccak_rc(11),
    keccak_rc(12), keccak_rc(13), keccak_rc(14), keccak_rc(15), keccak_rc(16), keccak_rc(17),
    keccak_rc(18), keccak_rc(19), keccak_rc(20), keccak_rc(21), keccak_rc(22), keccak_rc(23)};

constexpr unsigned TX_RATE = 168;

// Error bits recorded in TxState::err (never a trap: the host reads them).
constexpr unsigned TX_ERR_NARG_OVERFLOW = 1u, TX_ERR_HINT_OVERFLOW = 2u, TX_ERR_POW_EXHAUSTED = 4u,
                   TX_ERR_BAD_INDEX = 8u, TX_ERR_FIELD = 16u;

struct TxState {
    u64 hasher[25];
    u64 reader[25];
    unsigned hpos, rpos, has_reader, err;
    unsigned deg;  // degree of the target field over Goldilocks: 3 (Ext3), 2 (Ext2) or 1 (the base field)
    u64 narg_len, hints_len;
    u64 narg_cap, hints_cap;
    u8* narg;
    u8* hints;
};

}  // namespace wg
