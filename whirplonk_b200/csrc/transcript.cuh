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
// The state lives in HBM so that the whole proof can run as one stream of
// kernels (and be captured in a CUDA graph) without the host ever reading a
// challenge back.  All functions here are executed by ONE thread.
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

__device__ __forceinline__ u64 rotl64(u64 v, int s) { return s == 0 ? v : ((v << s) | (v >> (64 - s))); }

// rho-pi as one in-place cycle: lane PI_LANE[i] receives lane PI_LANE[i-1]
// (PI_LANE[-1] = 1) rotated by RHO_CYCLE[i].  Both follow the orbit
// (x, y) -> (y, 2x + 3y) starting at (1, 0), as keccak_rho does.
__host__ __device__ constexpr int keccak_pi_lane(int i) {
    int x = 1, y = 0;
    for (int t = 0; t <= i; ++t) {
        const int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    return x + 5 * y;
}
__host__ __device__ constexpr int keccak_pi_rot(int i) {
    int x = 1, y = 0;
    for (int t = 0; t < i; ++t) {
        const int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    return keccak_rho(x, y);
}

// Keccak-f[1600] on a 25-lane state in memory: lanes are pulled into
// registers (constant indices only), permuted in place with at most five
// temporaries (so the state stays in registers even under a tight register
// budget of the calling kernel), written back.
static __device__ __noinline__ void keccak_f1600(u64* st) {
    u64 a[25];
#pragma unroll
    for (int i = 0; i < 25; ++i) a[i] = st[i];
#pragma unroll 1
    for (int round = 0; round < 24; ++round) {
        {  // theta
            u64 c[5];
#pragma unroll
            for (int x = 0; x < 5; ++x) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
            for (int x = 0; x < 5; ++x) {
                const u64 d = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
#pragma unroll
                for (int y = 0; y < 5; ++y) a[x + 5 * y] ^= d;
            }
        }
        {  // rho and pi
            u64 t = a[1];
#pragma unroll
            for (int i = 0; i < 24; ++i) {
                const int j = keccak_pi_lane(i);
                const u64 nxt = a[j];
                a[j] = rotl64(t, keccak_pi_rot(i));
                t = nxt;
            }
        }
#pragma unroll
        for (int y = 0; y < 5; ++y) {  // chi
            const u64 r0 = a[5 * y], r1 = a[5 * y + 1], r2 = a[5 * y + 2], r3 = a[5 * y + 3], r4 = a[5 * y + 4];
            a[5 * y] = r0 ^ (~r1 & r2);
            a[5 * y + 1] = r1 ^ (~r2 & r3);
            a[5 * y + 2] = r2 ^ (~r3 & r4);
            a[5 * y + 3] = r3 ^ (~r4 & r0);
            a[5 * y + 4] = r4 ^ (~r0 & r1);
        }
        a[0] ^= KECCAK_RC[round];  // iota
    }
#pragma unroll
    for (int i = 0; i < 25; ++i) st[i] = a[i];
}

constexpr unsigned TX_RATE = 168;

// Error bits recorded in TxState::err (never a trap: the host reads them).
constexpr unsigned TX_ERR_NARG_OVERFLOW = 1u, TX_ERR_HINT_OVERFLOW = 2u, TX_ERR_POW_EXHAUSTED = 4u,
                   TX_ERR_BAD_INDEX = 8u;

struct TxState {
    u64 hasher[25];
    u64 reader[25];
    unsigned hpos, rpos, has_reader, err;
    u64 narg_len, hints_len;
    u64 narg_cap, hints_cap;
    u8* narg;
    u8* hints;
};

__device__ __forceinline__ void lane_xor_byte(u64* s, unsigned pos, u8 v) { s[pos >> 3] ^= (u64)v << (8 * (pos & 7)); }
__device__ __forceinline__ u8 lane_byte(const u64* s, unsigned pos) { return (u8)(s[pos >> 3] >> (8 * (pos & 7))); }

__device__ inline void tx_absorb(TxState* t, const u8* src, unsigned n) {
    t->has_reader = 0;
    unsigned pos = t->hpos;
    for (unsigned i = 0; i < n; ++i) {
        lane_xor_byte(t->hasher, pos++, src[i]);
        if (pos == TX_RATE) { keccak_f1600(t->hasher); pos = 0; }
    }
    t->hpos = pos;
}
// Absorb 8-byte words (every WHIR message is a whole number of u64 words).
__device__ inline void tx_absorb_words(TxState* t, const u64* w, unsigned nw) {
    t->has_reader = 0;
    unsigned pos = t->hpos;
    for (unsigned i = 0; i < nw; ++i) {
        u64 v = w[i];
        if ((pos & 7) == 0) {
            t->hasher[pos >> 3] ^= v;
            pos += 8;
            if (pos == TX_RATE) { keccak_f1600(t->hasher); pos = 0; }
        } else {
            for (int b = 0; b < 8; ++b) {
                lane_xor_byte(t->hasher, pos++, (u8)(v >> (8 * b)));
                if (pos == TX_RATE) { keccak_f1600(t->hasher); pos = 0; }
            }
        }
    }
    t->hpos = pos;
}
__device__ inline void tx_squeeze(TxState* t, u8* dst, unsigned n) {
    if (n == 0) return;
    if (!t->has_reader) {
        for (int i = 0; i < 25; ++i) t->reader[i] = t->hasher[i];
        lane_xor_byte(t->reader, t->hpos, 0x1F);
        lane_xor_byte(t->reader, TX_RATE - 1, 0x80);
        keccak_f1600(t->reader);
        t->rpos = 0;
        t->has_reader = 1;
    }
    unsigned pos = t->rpos;
    for (unsigned i = 0; i < n; ++i) {
        if (pos == TX_RATE) { keccak_f1600(t->reader); pos = 0; }
        dst[i] = lane_byte(t->reader, pos++);
    }
    t->rpos = pos;
}
__device__ inline void tx_narg_append(TxState* t, const u8* src, unsigned n) {
    if (t->narg_len + n > t->narg_cap) { t->err |= TX_ERR_NARG_OVERFLOW; return; }
    for (unsigned i = 0; i < n; ++i) t->narg[t->narg_len + i] = src[i];
    t->narg_len += n;
}
__device__ inline void tx_message_words(TxState* t, const u64* w, unsigned nw) {
    tx_absorb_words(t, w, nw);
    tx_narg_append(t, reinterpret_cast<const u8*>(w), 8 * nw);
}
__device__ inline void tx_message_e3(TxState* t, E3 v) {
    u64 w[3] = {v.c0, v.c1, v.c2};
    tx_message_words(t, w, 3);
}
__device__ inline void tx_message_u64(TxState* t, u64 v) { tx_message_words(t, &v, 1); }
__device__ inline void tx_hint(TxState* t, const u8* src, u64 n) {
    if (t->hints_len + n > t->hints_cap) { t->err |= TX_ERR_HINT_OVERFLOW; return; }
    for (u64 i = 0; i < n; ++i) t->hints[t->hints_len + i] = src[i];
    t->hints_len += n;
}
// 40 LE bytes as an integer mod p: five 64-bit limbs folded from the top,
// acc <- acc * 2^64 + limb (mod p).
__device__ inline u64 tx_decode40(const u8* b) {
    u64 w[5];
    for (int i = 0; i < 5; ++i) {
        u64 v = 0;
        for (int j = 7; j >= 0; --j) v = (v << 8) | b[8 * i + j];
        w[i] = v;
    }
    u64 acc = gl_reduce(w[4], 0);
    for (int i = 3; i >= 0; --i) acc = gl_reduce(w[i], acc);
    return acc;
}
__device__ inline E3 tx_challenge_e3(TxState* t) {
    u8 b[120];
    tx_squeeze(t, b, 120);
    return E3{tx_decode40(b), tx_decode40(b + 40), tx_decode40(b + 80)};
}
__device__ inline u64 tx_challenge_base(TxState* t) {
    u8 b[40];
    tx_squeeze(t, b, 40);
    return tx_decode40(b);
}

}  // namespace wg
