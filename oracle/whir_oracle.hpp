// whir_oracle.hpp -- TEST INFRASTRUCTURE ONLY (the oracle), never the product.
//
// A plain, single-file CPU restatement of the reference WHIR prover path
// (hxd77/WhirPlonk, C++ port under cpp/include/whir) for
//   M = Basefield<GoldilocksExt3>, hash = BLAKE3 or SHA-256, MLE / dense
//   covector statements, one or more witnesses of batch_size vectors each.
// It is written for clarity: simple loops, no SIMD, OpenMP only on loops whose
// result does not depend on the order (all arithmetic is exact field math).
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it,
// as the checker.  It is pinned against (a) the reference's committed golden
// dumps (cpp/dump_output/*) and (b) the reference prover itself compiled in
// place (oracle/_ref/ref_driver); see tests/test_oracle_pins.py.
//
// Every function cites the reference file:line whose behaviour it restates.
#pragma once

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

using u8 = std::uint8_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;
using u128 = unsigned __int128;

// ---------------------------------------------------------------------------
// Goldilocks field, p = 2^64 - 2^32 + 1 (cpp/include/whir/algebra/goldilocks.hpp:54-202).
// Canonical representative in [0, p).  Reduction of a 128-bit product uses the
// identities 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
// ---------------------------------------------------------------------------
constexpr u64 P = 0xFFFFFFFF00000001ull;
constexpr u64 EPS = 0xFFFFFFFFull;  // 2^64 mod p

inline u64 fadd(u64 a, u64 b) {
    u64 s = a + b;
    bool carry = s < a;
    if (carry) s += EPS;            // dropped 2^64 == EPS (mod p); cannot carry again
    if (s >= P) s -= P;
    return s;
}
inline u64 fsub(u64 a, u64 b) { return a >= b ? a - b : a + (P - b); }
inline u64 fneg(u64 a) { return a == 0 ? 0 : P - a; }
inline u64 reduce128(u128 x) {
    u64 lo = (u64)x, hi = (u64)(x >> 64);
    u64 hh = hi >> 32, hl = hi & EPS;
    // x = lo + hl*2^64 + hh*2^96 = lo + hl*EPS - hh
    u64 t = lo - hh;
    if (lo < hh) t -= EPS;          // borrowed 2^64 == EPS
    u64 m = hl * EPS;               // < 2^64
    u64 s = t + m;
    if (s < t) s += EPS;
    if (s >= P) s -= P;
    return s;
}
inline u64 fmul(u64 a, u64 b) { return reduce128((u128)a * b); }
inline u64 fpow(u64 b, u64 e) {
    u64 r = 1;
    while (e) {
        if (e & 1) r = fmul(r, b);
        b = fmul(b, b);
        e >>= 1;
    }
    return r;
}
inline u64 finv(u64 a) { return fpow(a, P - 2); }
inline u64 canon(u64 v) { return v >= P ? v - P : v; }  // Goldilocks::from_u64 (:73-75)

// Primitive N-th root of unity used by the reference NTT engine:
// (7^(2^32-1))^(2^32/N) == 7^((p-1)/N)  (goldilocks.hpp:155-159,
// cooley_tukey_goldilocks.hpp:24-29, cooley_tukey.hpp:161-171).
inline u64 root_of_unity(u64 n) {
    assert(n && (n & (n - 1)) == 0 && n <= (1ull << 32));
    return fpow(7, (P - 1) / n);
}

// ---------------------------------------------------------------------------
// Ext3 = Fp[X]/(X^3 - 2) (goldilocks_ext3.hpp:33-137); layout c0 + c1 X + c2 X^2.
// ---------------------------------------------------------------------------
struct E3 {
    u64 c[3] = {0, 0, 0};
    static E3 from_base(u64 a) { E3 r; r.c[0] = a; return r; }
    static E3 one() { return from_base(1); }
    bool operator==(const E3& o) const { return c[0] == o.c[0] && c[1] == o.c[1] && c[2] == o.c[2]; }
    bool operator!=(const E3& o) const { return !(*this == o); }
};
inline E3 operator+(const E3& a, const E3& b) { E3 r; for (int i = 0; i < 3; ++i) r.c[i] = fadd(a.c[i], b.c[i]); return r; }
inline E3 operator-(const E3& a, const E3& b) { E3 r; for (int i = 0; i < 3; ++i) r.c[i] = fsub(a.c[i], b.c[i]); return r; }
inline E3 operator*(const E3& a, const E3& b) {
    const u64 *x = a.c, *y = b.c;
    E3 r;
    u64 t12 = fadd(fmul(x[1], y[2]), fmul(x[2], y[1]));
    r.c[0] = fadd(fmul(x[0], y[0]), fadd(t12, t12));
    u64 t22 = fmul(x[2], y[2]);
    r.c[1] = fadd(fadd(fmul(x[0], y[1]), fmul(x[1], y[0])), fadd(t22, t22));
    r.c[2] = fadd(fadd(fmul(x[0], y[2]), fmul(x[1], y[1])), fmul(x[2], y[0]));
    return r;
}
inline E3 smul(const E3& a, u64 b) { E3 r; for (int i = 0; i < 3; ++i) r.c[i] = fmul(a.c[i], b); return r; }
inline E3 e3pow(E3 b, u64 e) {
    E3 r = E3::one();
    while (e) {
        if (e & 1) r = r * b;
        b = b * b;
        e >>= 1;
    }
    return r;
}

// ---------------------------------------------------------------------------
// Keccak-f[1600], SHAKE128, SHA3-256/512 (FIPS 202), restated from the
// specification; the reference vendors its own in cpp/third_party/keccak.
// Round constants and rotation offsets are derived from their FIPS 202
// definitions at start-up rather than tabulated.
// ---------------------------------------------------------------------------
struct KeccakTables {
    u64 rc[24];
    int rot[25];
    KeccakTables() {
        // rc(t): LFSR x^8 + x^6 + x^5 + x^4 + 1 (FIPS 202 Alg. 5)
        auto rcbit = [](int t) {
            if (t % 255 == 0) return 1;
            // R[0..7] kept in one byte, R[0] in bit 7.  Each step prepends a
            // zero (shift right), then folds the dropped bit R[8] into
            // R[0], R[4], R[5], R[6].
            unsigned r = 0x80;
            for (int i = 1; i <= t % 255; ++i) {
                unsigned r8 = r & 1;
                r >>= 1;
                if (r8) r ^= 0x80 | 0x08 | 0x04 | 0x02;
            }
            return (int)((r >> 7) & 1);
        };
        for (int ir = 0; ir < 24; ++ir) {
            u64 v = 0;
            for (int j = 0; j <= 6; ++j)
                if (rcbit(j + 7 * ir)) v |= 1ull << ((1 << j) - 1);
            rc[ir] = v;
        }
        for (int i = 0; i < 25; ++i) rot[i] = 0;
        int x = 1, y = 0;
        for (int t = 0; t < 24; ++t) {
            rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
            int nx = y, ny = (2 * x + 3 * y) % 5;
            x = nx;
            y = ny;
        }
    }
};
inline const KeccakTables& ktab() { static const KeccakTables t; return t; }

inline u64 rotl64(u64 v, int s) { return s == 0 ? v : (v << s) | (v >> (64 - s)); }

inline void keccak_f1600(u64 a[25]) {
    const auto& T = ktab();
    for (int round = 0; round < 24; ++round) {
        u64 c[5], d[5], b[25];
        for (int x = 0; x < 5; ++x) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
        for (int x = 0; x < 5; ++x) d[x] = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
        for (int i = 0; i < 25; ++i) a[i] ^= d[i % 5];
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(a[x + 5 * y], T.rot[x + 5 * y]);
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= T.rc[round];
    }
}

inline void state_xor_byte(u64 s[25], size_t pos, u8 v) { s[pos / 8] ^= (u64)v << (8 * (pos % 8)); }
inline u8 state_byte(const u64 s[25], size_t pos) { return (u8)(s[pos / 8] >> (8 * (pos % 8))); }

// Generic Keccak sponge with byte-granular absorb and pad suffix.
struct Sponge {
    u64 s[25] = {};
    size_t rate, pos = 0;
    explicit Sponge(size_t r) : rate(r) {}
    void absorb(const u8* d, size_t n) {
        for (size_t i = 0; i < n; ++i) {
            state_xor_byte(s, pos++, d[i]);
            if (pos == rate) { keccak_f1600(s); pos = 0; }
        }
    }
    void finalize(u8 suffix) {
        state_xor_byte(s, pos, suffix);
        state_xor_byte(s, rate - 1, 0x80);
        keccak_f1600(s);
        pos = 0;
    }
    void squeeze(u8* out, size_t n) {  // after finalize
        for (size_t i = 0; i < n; ++i) {
            if (pos == rate) { keccak_f1600(s); pos = 0; }
            out[i] = state_byte(s, pos++);
        }
    }
};
inline void sha3_256(const u8* d, size_t n, u8 out[32]) { Sponge sp(136); sp.absorb(d, n); sp.finalize(0x06); sp.squeeze(out, 32); }
inline void sha3_512(const u8* d, size_t n, u8 out[64]) { Sponge sp(72); sp.absorb(d, n); sp.finalize(0x06); sp.squeeze(out, 64); }
inline void shake128(const u8* d, size_t n, u8* out, size_t m) { Sponge sp(168); sp.absorb(d, n); sp.finalize(0x1F); sp.squeeze(out, m); }

// ---------------------------------------------------------------------------
// BLAKE3 (public specification).  Messages of one chunk (<= 1024 bytes) are
// most of what the WHIR path hashes: leaves of 128 B (base rows) or 384 B
// (Ext3 rows), Merkle parents and PoW inputs of 64 B.  For sizes that are a
// multiple of 64 this is exactly the reference's blake3_hash_many call with
// flags_start = CHUNK_START, flags_end = CHUNK_END|ROOT
// (cpp/include/whir/hash/blake3_engine.hpp:90-199).  Rows of several
// committed vectors can be wider than a chunk; those take the tree below.
// ---------------------------------------------------------------------------
constexpr u32 B3_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                          0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
constexpr int B3_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
constexpr u32 B3_CHUNK_START = 1, B3_CHUNK_END = 2, B3_ROOT = 8;

inline u32 rotr32(u32 v, int s) { return (v >> s) | (v << (32 - s)); }
inline void b3_g(u32 v[16], int a, int b, int c, int d, u32 x, u32 y) {
    v[a] = v[a] + v[b] + x; v[d] = rotr32(v[d] ^ v[a], 16);
    v[c] = v[c] + v[d];     v[b] = rotr32(v[b] ^ v[c], 12);
    v[a] = v[a] + v[b] + y; v[d] = rotr32(v[d] ^ v[a], 8);
    v[c] = v[c] + v[d];     v[b] = rotr32(v[b] ^ v[c], 7);
}
inline void b3_compress(u32 cv[8], const u32 blk[16], u64 counter, u32 len, u32 flags) {
    u32 v[16], m[16], t[16];
    for (int i = 0; i < 8; ++i) v[i] = cv[i];
    for (int i = 0; i < 4; ++i) v[8 + i] = B3_IV[i];
    v[12] = (u32)counter; v[13] = (u32)(counter >> 32); v[14] = len; v[15] = flags;
    for (int i = 0; i < 16; ++i) m[i] = blk[i];
    for (int r = 0; r < 7; ++r) {
        b3_g(v, 0, 4, 8, 12, m[0], m[1]);   b3_g(v, 1, 5, 9, 13, m[2], m[3]);
        b3_g(v, 2, 6, 10, 14, m[4], m[5]);  b3_g(v, 3, 7, 11, 15, m[6], m[7]);
        b3_g(v, 0, 5, 10, 15, m[8], m[9]);  b3_g(v, 1, 6, 11, 12, m[10], m[11]);
        b3_g(v, 2, 7, 8, 13, m[12], m[13]); b3_g(v, 3, 4, 9, 14, m[14], m[15]);
        if (r < 6) { for (int i = 0; i < 16; ++i) t[i] = m[B3_PERM[i]]; for (int i = 0; i < 16; ++i) m[i] = t[i]; }
    }
    for (int i = 0; i < 8; ++i) cv[i] = v[i] ^ v[i + 8];
}
using Hash = std::array<u8, 32>;
constexpr u32 B3_PARENT = 4;
// Chaining value of one chunk (<= 1024 bytes) with chunk counter `counter`.
inline void b3_chunk(const u8* d, size_t n, u64 counter, u32 extra_end_flags, u32 cv[8]) {
    for (int i = 0; i < 8; ++i) cv[i] = B3_IV[i];
    size_t nblocks = n == 0 ? 1 : (n + 63) / 64;
    for (size_t b = 0; b < nblocks; ++b) {
        u8 buf[64] = {};
        size_t take = std::min<size_t>(64, n - std::min(n, b * 64));
        if (take) std::memcpy(buf, d + b * 64, take);
        u32 blk[16];
        for (int i = 0; i < 16; ++i) blk[i] = (u32)buf[4 * i] | (u32)buf[4 * i + 1] << 8 | (u32)buf[4 * i + 2] << 16 | (u32)buf[4 * i + 3] << 24;
        u32 flags = (b == 0 ? B3_CHUNK_START : 0) | (b + 1 == nblocks ? (B3_CHUNK_END | extra_end_flags) : 0);
        b3_compress(cv, blk, counter, (u32)take, flags);
    }
}
inline void b3_parent(const u32 l[8], const u32 r[8], u32 flags, u32 out[8]) {
    u32 blk[16];
    for (int i = 0; i < 8; ++i) { blk[i] = l[i]; blk[8 + i] = r[i]; }
    for (int i = 0; i < 8; ++i) out[i] = B3_IV[i];
    b3_compress(out, blk, 0, 64, B3_PARENT | flags);
}
// Multi-chunk messages (rows wider than 1024 bytes, the reference's
// blake3_hasher fallback in blake3_engine.hpp:186-196) follow the
// specification's tree: chunk i is hashed with counter i, completed subtrees
// are merged as soon as the chunk count has a trailing zero bit, and the last
// chunk's chaining value is merged with the remaining stack from the top, the
// final merge carrying the ROOT flag.
inline Hash blake3(const u8* d, size_t n) {
    const size_t nch = n <= 1024 ? 1 : (n + 1023) / 1024;
    u32 cv[8];
    if (nch == 1) {
        b3_chunk(d, n, 0, B3_ROOT, cv);
    } else {
        std::vector<std::array<u32, 8>> stack;
        for (size_t c = 0; c + 1 < nch; ++c) {
            std::array<u32, 8> cur;
            b3_chunk(d + c * 1024, 1024, c, 0, cur.data());
            for (u64 total = c + 1; (total & 1) == 0; total >>= 1) {
                std::array<u32, 8> m;
                b3_parent(stack.back().data(), cur.data(), 0, m.data());
                stack.pop_back();
                cur = m;
            }
            stack.push_back(cur);
        }
        b3_chunk(d + (nch - 1) * 1024, n - (nch - 1) * 1024, nch - 1, 0, cv);
        while (!stack.empty()) {
            u32 m[8];
            b3_parent(stack.back().data(), cv, stack.size() == 1 ? B3_ROOT : 0, m);
            stack.pop_back();
            std::memcpy(cv, m, 32);
        }
    }
    Hash h;
    for (int i = 0; i < 8; ++i) for (int j = 0; j < 4; ++j) h[4 * i + j] = (u8)(cv[i] >> (8 * j));
    return h;
}

// ---------------------------------------------------------------------------
// SHA-256 (FIPS 180-4), the reference's second hash engine
// (cpp/include/whir/hash/sha2_engine.hpp:47-81 over cpp/third_party/sha256).
// The round constants and the initial hash value are derived here from their
// definitions: the first 32 fractional bits of the cube roots of the first 64
// primes and of the square roots of the first 8 primes.
// ---------------------------------------------------------------------------
constexpr u64 sha_prime(int k) {
    u64 n = 1;
    for (int found = -1; found < k;) {
        ++n;
        bool prime = true;
        for (u64 d = 2; d * d <= n; ++d)
            if (n % d == 0) { prime = false; break; }
        if (prime) ++found;
    }
    return n;
}
// floor(root-th root of p, with 32 fractional bits) mod 2^32
constexpr u32 sha_root_frac(u64 p, int root) {
    using u128 = unsigned __int128;
    const u128 target = (u128)p << (32 * root);
    u64 lo = 0, hi = 1ull << 40;
    while (lo + 1 < hi) {
        const u64 mid = (lo + hi) / 2;
        u128 v = 1;
        for (int i = 0; i < root; ++i) v *= mid;
        if (v <= target) lo = mid;
        else hi = mid;
    }
    return (u32)lo;
}
struct Sha256Consts {
    u32 k[64], h0[8];
    constexpr Sha256Consts() : k(), h0() {
        for (int i = 0; i < 64; ++i) k[i] = sha_root_frac(sha_prime(i), 3);
        for (int i = 0; i < 8; ++i) h0[i] = sha_root_frac(sha_prime(i), 2);
    }
};
inline constexpr Sha256Consts SHA256_C{};
inline u32 ror32(u32 x, int s) { return (x >> s) | (x << (32 - s)); }
inline void sha256_compress(u32 h[8], const u8 blk[64]) {
    u32 w[64];
    for (int i = 0; i < 16; ++i) w[i] = (u32)blk[4 * i] << 24 | (u32)blk[4 * i + 1] << 16 | (u32)blk[4 * i + 2] << 8 | blk[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
        const u32 s0 = ror32(w[i - 15], 7) ^ ror32(w[i - 15], 18) ^ (w[i - 15] >> 3);
        const u32 s1 = ror32(w[i - 2], 17) ^ ror32(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    u32 a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; ++i) {
        const u32 t1 = hh + (ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25)) + ((e & f) ^ (~e & g)) + SHA256_C.k[i] + w[i];
        const u32 t2 = (ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}
inline Hash sha256(const u8* d, size_t n) {
    u32 h[8];
    for (int i = 0; i < 8; ++i) h[i] = SHA256_C.h0[i];
    size_t full = n / 64;
    for (size_t b = 0; b < full; ++b) sha256_compress(h, d + 64 * b);
    u8 tail[128] = {};
    const size_t rem = n - 64 * full;
    if (rem) std::memcpy(tail, d + 64 * full, rem);
    tail[rem] = 0x80;
    const size_t tl = rem + 9 <= 64 ? 64 : 128;
    const u64 bits = (u64)n * 8;
    for (int i = 0; i < 8; ++i) tail[tl - 1 - i] = (u8)(bits >> (8 * i));
    for (size_t b = 0; b < tl / 64; ++b) sha256_compress(h, tail + 64 * b);
    Hash out;
    for (int i = 0; i < 8; ++i) for (int j = 0; j < 4; ++j) out[4 * i + j] = (u8)(h[i] >> (24 - 8 * j));
    return out;
}

// The engine a configuration's hash_id selects (irs_commit.hpp:62-74): SHA-256
// for ENGINE_ID_SHA2, BLAKE3 otherwise.
enum class Engine { Blake3, Sha2 };
inline Hash hash_with(Engine e, const u8* d, size_t n) { return e == Engine::Sha2 ? sha256(d, n) : blake3(d, n); }

// ---------------------------------------------------------------------------
// Fiat-Shamir transcript (cpp/include/whir/transcript/transcript.hpp).
// absorb continues the SHAKE128 hasher; the first squeeze after an absorb
// finalises a clone of the hasher and later squeezes keep reading that XOF
// until the next absorb (:80-106).  prover_message = absorb + append raw LE
// bytes to narg (:623-629); prover_hint(vector) = u64 LE length + raw
// elements, prover_hint(Hash) = 32 raw bytes (:290-296, :633-635);
// field challenges decode 40 LE bytes per base coefficient mod p (:375-453).
// ---------------------------------------------------------------------------
struct Transcript {
    Sponge hasher{168};
    Sponge reader{168};
    bool has_reader = false;
    std::vector<u8> narg, hints;

    void absorb(const u8* d, size_t n) { has_reader = false; hasher.absorb(d, n); }
    void squeeze(u8* out, size_t n) {
        if (n == 0) return;
        if (!has_reader) { reader = hasher; reader.finalize(0x1F); has_reader = true; }
        reader.squeeze(out, n);
    }
    void message_bytes(const u8* d, size_t n) { absorb(d, n); narg.insert(narg.end(), d, d + n); }
    void message_e3(const E3& v) { u8 b[24]; std::memcpy(b, v.c, 24); message_bytes(b, 24); }
    void message_u64(u64 v) { u8 b[8]; std::memcpy(b, &v, 8); message_bytes(b, 8); }
    void message_hash(const Hash& h) { message_bytes(h.data(), 32); }
    void hint_bytes(const u8* d, size_t n) { hints.insert(hints.end(), d, d + n); }
    void hint_u64(u64 v) { u8 b[8]; std::memcpy(b, &v, 8); hint_bytes(b, 8); }
    static u64 decode40(const u8* b) {
        u64 acc = 0;  // big integer from LE bytes, reduced mod p; Horner from the top byte
        for (int i = 39; i >= 0; --i) acc = (u64)(((u128)acc * 256 + b[i]) % P);
        return acc;
    }
    u64 challenge_base() { u8 b[40]; squeeze(b, 40); return decode40(b); }
    E3 challenge_e3() {
        u8 b[120];
        squeeze(b, 120);
        E3 r;
        for (int i = 0; i < 3; ++i) r.c[i] = decode40(b + 40 * i);
        return r;
    }
    // The protocol's target field: Ext3 (Basefield<GoldilocksExt3>, deg 3) or the
    // base field itself (Identity<Goldilocks>, deg 1), whose elements are kept
    // here as Ext3 values (x, 0, 0) -- the base field is a subfield, so the
    // arithmetic is unchanged -- and cross the transcript as 8 bytes / 40-byte
    // challenges (transcript.hpp:375-453).
    int deg = 3;
    E3 challenge_t() { return deg == 1 ? E3::from_base(challenge_base()) : challenge_e3(); }
    void message_t(const E3& v) {
        if (deg == 1) {
            if (v.c[1] || v.c[2]) throw std::runtime_error("base-field message outside the subfield");
            message_u64(v.c[0]);
        } else {
            message_e3(v);
        }
    }
};

// ---------------------------------------------------------------------------
// Domain separator of the reference CLI (cpp/main.cpp:174-215): protocol_id =
// SHA3-512(CBOR map of ProtocolParameters), session_id = SHA3-256(CBOR text
// "Example at src/bin/main.rs:133"); absorbed as protocol_id || session_id ||
// instance bytes (transcript.hpp:533-539; instance Empty -> no bytes).
// ---------------------------------------------------------------------------
// Engine ids of the reference's hash engines (cpp/include/whir/hash/blake3_engine.hpp,
// sha2_engine.hpp:38-43), copied: they are identifiers, not computed here.
constexpr u8 SHA2_ENGINE_ID[32] = {0x01, 0x8e, 0xaa, 0x24, 0x7c, 0xb8, 0x95, 0x7a, 0xb1, 0xe9, 0xfd,
                                   0xac, 0x88, 0x54, 0x50, 0x40, 0x3c, 0x5e, 0x7b, 0xda, 0x1a, 0xca,
                                   0xaa, 0x50, 0x4e, 0x4c, 0xc8, 0xf2, 0xf7, 0x6b, 0xb0, 0x76};
constexpr u8 BLAKE3_ENGINE_ID[32] = {0x03, 0xe0, 0x17, 0x49, 0xeb, 0xcc, 0x04, 0x77, 0x92, 0x42, 0x54,
                                     0xeb, 0x48, 0x20, 0x66, 0xb8, 0x64, 0xa8, 0xdd, 0x4d, 0x77, 0x25,
                                     0x24, 0x64, 0xca, 0x6f, 0x5b, 0x6f, 0x5c, 0xc0, 0x5b, 0x4c};

struct Params {  // ProtocolParameters (cpp/include/whir/parameters.hpp:25-34)
    bool unique_decoding = false;
    u64 starting_log_inv_rate = 1, initial_folding_factor = 4, folding_factor = 4;
    u64 security_level = 100, pow_bits = 20, batch_size = 1;
    u8 hash_id[32];
    Params() { std::memcpy(hash_id, BLAKE3_ENGINE_ID, 32); }
};

inline void cbor_head(std::vector<u8>& o, u8 major, u64 v) {
    u8 m = (u8)(major << 5);
    if (v < 24) o.push_back(m | (u8)v);
    else if (v <= 0xFF) { o.push_back(m | 24); o.push_back((u8)v); }
    else if (v <= 0xFFFF) { o.push_back(m | 25); for (int s = 8; s >= 0; s -= 8) o.push_back((u8)(v >> s)); }
    else if (v <= 0xFFFFFFFFull) { o.push_back(m | 26); for (int s = 24; s >= 0; s -= 8) o.push_back((u8)(v >> s)); }
    else { o.push_back(m | 27); for (int s = 56; s >= 0; s -= 8) o.push_back((u8)(v >> s)); }
}
inline void cbor_text(std::vector<u8>& o, const char* s) { size_t n = std::strlen(s); cbor_head(o, 3, n); o.insert(o.end(), s, s + n); }

struct DomainSep { u8 protocol_id[64]; u8 session_id[32]; };
inline DomainSep cli_domain_separator(const Params& p) {
    std::vector<u8> c;
    cbor_head(c, 5, 8);
    cbor_text(c, "unique_decoding"); c.push_back(p.unique_decoding ? 0xF5 : 0xF4);
    cbor_text(c, "starting_log_inv_rate"); cbor_head(c, 0, p.starting_log_inv_rate);
    cbor_text(c, "initial_folding_factor"); cbor_head(c, 0, p.initial_folding_factor);
    cbor_text(c, "folding_factor"); cbor_head(c, 0, p.folding_factor);
    cbor_text(c, "security_level"); cbor_head(c, 0, p.security_level);
    cbor_text(c, "pow_bits"); cbor_head(c, 0, p.pow_bits);
    cbor_text(c, "batch_size"); cbor_head(c, 0, p.batch_size);
    cbor_text(c, "hash_id"); cbor_head(c, 4, 32);
    for (int i = 0; i < 32; ++i) cbor_head(c, 0, p.hash_id[i]);
    DomainSep ds;
    sha3_512(c.data(), c.size(), ds.protocol_id);
    std::vector<u8> s;
    cbor_text(s, "Example at src/bin/main.rs:133");
    sha3_256(s.data(), s.size(), ds.session_id);
    return ds;
}

// ---------------------------------------------------------------------------
// Parameter schedule (cpp/include/whir/protocols/whir/whir.hpp:118-224 and
// irs_commit.hpp:192-324).  Double-precision expressions kept operation for
// operation, since PoW thresholds and sample counts are derived from them.
// ---------------------------------------------------------------------------
struct IrsCfg {
    u64 num_vectors = 1, vector_size = 0, codeword_length = 0, depth = 0;
    double johnson_slack = 0;
    u64 in_domain = 0, out_domain = 0;
    u64 msg_len() const { return vector_size / depth; }
    double rate() const { return (double)msg_len() / (double)codeword_length; }
    bool unique() const { return out_domain == 0 && johnson_slack == 0.0; }
    double list_size() const { return unique() ? 1.0 : 1.0 / (2.0 * johnson_slack * std::sqrt(rate())); }
    double rbr_queries() const {
        double per = unique() ? ((1.0 + rate()) * 0.5) : (std::sqrt(rate()) + johnson_slack);
        return (double)in_domain * (-std::log2(per));
    }
    double fold_prox_gaps(double fbits) const {
        double lir = -std::log2(rate());
        double logk = std::log2((double)msg_len());
        double err;
        if (unique()) err = logk + lir;
        else { constexpr double L10 = 3.321928094887362; err = 7.0 * L10 + 3.5 * lir + 2.0 * logk; }
        return fbits - err;
    }
    static IrsCfg make(double sec, bool ud, u64 nvec, u64 vsize, u64 depth, double rate, double fbits) {
        IrsCfg c;
        c.num_vectors = nvec; c.vector_size = vsize; c.depth = depth;
        u64 ml = vsize / depth;
        c.codeword_length = (u64)std::ceil((double)ml / rate);
        double ar = (double)ml / (double)c.codeword_length;
        c.johnson_slack = ud ? 0.0 : std::sqrt(ar) / 20.0;
        if (ud) c.out_domain = 0;
        else {
            double L = 1.0 / (2.0 * c.johnson_slack * std::sqrt(ar));
            double lc2 = L * (L - 1.0) / 2.0;
            double lps = fbits - std::log2((double)(vsize - 1));
            c.out_domain = (u64)std::ceil((sec + std::log2(lc2)) / lps);
            if (c.out_domain < 1) c.out_domain = 1;
        }
        double per = ud ? ((1.0 + ar) * 0.5) : (std::sqrt(ar) + c.johnson_slack);
        c.in_domain = (u64)std::ceil(sec / (-std::log2(per)));
        return c;
    }
};
struct SumcheckCfg { u64 initial_size = 0, num_rounds = 0, pow_threshold = ~0ull; };
struct RoundCfg { IrsCfg irs; SumcheckCfg sumcheck; u64 pow_threshold = ~0ull; };
struct WhirCfg {
    IrsCfg initial;
    SumcheckCfg initial_sumcheck;
    u64 initial_skip_pow = ~0ull;
    std::vector<RoundCfg> rounds;
    SumcheckCfg final_sumcheck;
    u64 final_pow = ~0ull;
};
inline u64 pow_threshold_of(double diff) {
    return diff <= 0.0 ? ~0ull : (u64)std::ceil(std::exp2(64.0 - diff));
}
// fbits = Target::field_size_bits: 192 for Ext3, 64 for Identity<Goldilocks>.
inline WhirCfg whir_from_params(u64 size, const Params& p, double fbits = 192.0) {
    if (!size || (size & (size - 1))) throw std::runtime_error("size must be a power of two");
    WhirCfg c;
    const double sec = (double)p.security_level;
    const double psec = (double)(p.security_level - p.pow_bits);
    u64 lir = p.starting_log_inv_rate;
    u64 nv = 0;
    for (u64 s = size; s > 1; s >>= 1) ++nv;
    if (nv < p.initial_folding_factor) throw std::runtime_error("num_variables < folding factor");
    double irate = std::pow(0.5, (double)p.starting_log_inv_rate);
    c.initial = IrsCfg::make(psec, p.unique_decoding, p.batch_size, size, 1ull << p.initial_folding_factor, irate, fbits);
    double start_fold = std::max(sec - std::min(c.initial.fold_prox_gaps(fbits), fbits - std::log2(c.initial.list_size()) - 1.0), 0.0);
    double skip = std::max(sec - (c.initial.fold_prox_gaps(fbits) + std::log2((double)p.initial_folding_factor)), 0.0);
    c.initial_sumcheck = {size, p.initial_folding_factor, pow_threshold_of(start_fold)};
    c.initial_skip_pow = pow_threshold_of(skip);
    u64 rd = 0;
    u64 ids = c.initial.in_domain;
    double qe = c.initial.rbr_queries();
    nv -= p.initial_folding_factor;
    while (nv >= p.folding_factor) {
        u64 rff = rd == 0 ? p.initial_folding_factor : p.folding_factor;
        u64 nli = lir + (rff - 1);
        double rr = std::pow(0.5, (double)nli);
        RoundCfg rc;
        rc.irs = IrsCfg::make(psec, p.unique_decoding, 1, 1ull << nv, 1ull << p.folding_factor, rr, fbits);
        double ll = std::log2(rc.irs.list_size());
        u64 cnt = rc.irs.out_domain + ids;
        double cbe = fbits - (std::log2((double)cnt) + ll + 1.0);
        double pb = std::max(sec - std::min(qe, cbe), 0.0);
        double fpb = std::max(sec - std::min(rc.irs.fold_prox_gaps(fbits), fbits - ll - 1.0), 0.0);
        rc.sumcheck = {1ull << nv, p.folding_factor, pow_threshold_of(fpb)};
        rc.pow_threshold = pow_threshold_of(pb);
        ++rd;
        nv -= p.folding_factor;
        lir = nli;
        ids = rc.irs.in_domain;
        qe = rc.irs.rbr_queries();
        c.rounds.push_back(rc);
    }
    double rbr_e = c.rounds.empty() ? c.initial.rbr_queries() : c.rounds.back().irs.rbr_queries();
    double fpb2 = std::max(sec - rbr_e, 0.0);
    double ffpb = std::max(sec - fbits + 1.0, 0.0);
    c.final_sumcheck = {1ull << nv, nv, pow_threshold_of(ffpb)};
    c.final_pow = pow_threshold_of(fpb2);
    return c;
}

// ---------------------------------------------------------------------------
// NTT and interleaved RS encoding (mod_ntt.hpp:49-130, cooley_tukey.hpp:200-259):
// codeword_b[i] = sum_{j<m} v[b*m + j] * w_N^(i*j), natural order in i;
// matrix row i = (codeword_0[i], ..., codeword_{d-1}[i]).
// ---------------------------------------------------------------------------
inline void ntt_inplace(std::vector<u64>& a) {
    const size_t n = a.size();
    if (n <= 1) return;
    for (size_t i = 1, j = 0; i < n; ++i) {  // bit-reversal permutation
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        u64 w = root_of_unity(len);
        std::vector<u64> tw(len / 2);
        tw[0] = 1;
        for (size_t k = 1; k < len / 2; ++k) tw[k] = fmul(tw[k - 1], w);
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                u64 u = a[i + k], v = fmul(a[i + k + len / 2], tw[k]);
                a[i + k] = fadd(u, v);
                a[i + k + len / 2] = fsub(u, v);
            }
    }
}
// Base-field vector -> row-major N x depth matrix.
inline std::vector<u64> rs_encode_base(const std::vector<u64>& v, u64 N, u64 depth) {
    const u64 m = v.size() / depth;
    std::vector<u64> out(N * depth);
#pragma omp parallel for schedule(dynamic)
    for (long long b = 0; b < (long long)depth; ++b) {
        std::vector<u64> blk(N, 0);
        for (u64 j = 0; j < m; ++j) blk[j] = v[b * m + j];
        ntt_inplace(blk);
        for (u64 i = 0; i < N; ++i) out[i * depth + b] = blk[i];
    }
    return out;
}
// Ext3 vector -> row-major N x depth matrix (roots are in the base field, so
// the Ext3 NTT is three component NTTs).
inline std::vector<E3> rs_encode_e3(const std::vector<E3>& v, u64 N, u64 depth) {
    const u64 m = v.size() / depth;
    std::vector<E3> out(N * depth);
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (long long b = 0; b < (long long)depth; ++b)
        for (int comp = 0; comp < 3; ++comp) {
            std::vector<u64> blk(N, 0);
            for (u64 j = 0; j < m; ++j) blk[j] = v[b * m + j].c[comp];
            ntt_inplace(blk);
            for (u64 i = 0; i < N; ++i) out[i * depth + b].c[comp] = blk[i];
        }
    return out;
}

// ---------------------------------------------------------------------------
// Merkle tree (merkle_tree.hpp:79-211): leaves padded to 2^L with zero hashes,
// parent = BLAKE3(left || right), node array [leaves | level 1 | ... | root].
// ---------------------------------------------------------------------------
inline u64 layers_for(u64 n) { u64 k = 0; while ((1ull << k) < n) ++k; return n <= 1 ? 0 : k; }
inline std::vector<Hash> merkle_build(std::vector<Hash> leaves, Engine eng = Engine::Blake3) {
    u64 L = layers_for(leaves.size());
    u64 leaf_layer = 1ull << L;
    std::vector<Hash> nodes = std::move(leaves);
    nodes.resize((1ull << (L + 1)) - 1, Hash{});
    u64 prev_off = 0, prev_len = leaf_layer, cur = leaf_layer;
    for (u64 l = 0; l < L; ++l) {
        u64 cur_len = prev_len / 2;
#pragma omp parallel for if (cur_len >= 4096)
        for (long long i = 0; i < (long long)cur_len; ++i) {
            u8 buf[64];
            std::memcpy(buf, nodes[prev_off + 2 * i].data(), 32);
            std::memcpy(buf + 32, nodes[prev_off + 2 * i + 1].data(), 32);
            nodes[cur + i] = hash_with(eng, buf, 64);
        }
        prev_off = cur;
        prev_len = cur_len;
        cur += cur_len;
    }
    return nodes;
}
inline std::vector<Hash> merkle_open(const std::vector<Hash>& nodes, u64 L, std::vector<u64> idx) {
    std::sort(idx.begin(), idx.end());
    idx.erase(std::unique(idx.begin(), idx.end()), idx.end());
    std::vector<Hash> hints;
    u64 off = 0, len = 1ull << L;
    while (len > 1) {
        std::vector<u64> nxt;
        for (size_t k = 0; k < idx.size();) {
            u64 a = idx[k];
            if (k + 1 < idx.size() && idx[k + 1] == (a ^ 1)) { k += 2; }
            else { hints.push_back(nodes[off + (a ^ 1)]); k += 1; }
            nxt.push_back(a >> 1);
        }
        idx = std::move(nxt);
        off += len;
        len /= 2;
    }
    return hints;
}

// Leaf hashes of a row-major matrix, LE canonical bytes per element
// (matrix_commit.hpp:74-195).
inline std::vector<Hash> leaves_base(const std::vector<u64>& mat, u64 cols, Engine eng = Engine::Blake3) {
    u64 rows = mat.size() / cols;
    std::vector<Hash> out(rows);
#pragma omp parallel for if (rows >= 1024)
    for (long long r = 0; r < (long long)rows; ++r)
        out[r] = hash_with(eng, reinterpret_cast<const u8*>(&mat[r * cols]), cols * 8);
    return out;
}
inline std::vector<Hash> leaves_e3(const std::vector<E3>& mat, u64 cols, Engine eng = Engine::Blake3) {
    u64 rows = mat.size() / cols;
    std::vector<Hash> out(rows);
#pragma omp parallel for if (rows >= 1024)
    for (long long r = 0; r < (long long)rows; ++r)
        out[r] = hash_with(eng, reinterpret_cast<const u8*>(&mat[r * cols]), cols * 24);
    return out;
}

// ---------------------------------------------------------------------------
// Proof of work (proof_of_work.hpp:95-193, 236-257): smallest nonce n >= 0 with
// LE_u64(BLAKE3(challenge || n_le8 || 0^24)[0..8]) <= threshold.
// ---------------------------------------------------------------------------
inline u64 pow_hash_u64(const u8 ch[32], u64 nonce, Engine eng = Engine::Blake3) {
    u8 msg[64] = {};
    std::memcpy(msg, ch, 32);
    std::memcpy(msg + 32, &nonce, 8);
    Hash h = hash_with(eng, msg, 64);
    u64 v;
    std::memcpy(&v, h.data(), 8);
    return v;
}
inline u64 find_nonce(const u8 ch[32], u64 threshold, Engine eng = Engine::Blake3) {
    if (threshold == ~0ull) return 0;
    const u64 W = 1 << 14;
    for (u64 base = 0;; base += W * 64) {
        u64 best = ~0ull;
#pragma omp parallel for reduction(min : best) schedule(static)
        for (long long i = 0; i < (long long)(W * 64); ++i)
            if (pow_hash_u64(ch, base + (u64)i, eng) <= threshold) best = std::min(best, base + (u64)i);
        if (best != ~0ull) return best;
    }
}
inline void pow_prove(Transcript& t, u64 threshold, Engine eng = Engine::Blake3) {
    if (threshold == ~0ull) return;
    u8 ch[32];
    t.squeeze(ch, 32);
    t.message_u64(find_nonce(ch, threshold, eng));
}

// ---------------------------------------------------------------------------
// Field helpers (utilities.hpp, multilinear.hpp, multilinear_point.hpp).
// ---------------------------------------------------------------------------
inline std::vector<E3> geometric(const E3& x, size_t n) {  // utilities.hpp:85-95
    std::vector<E3> o(n);
    E3 c = E3::one();
    for (size_t i = 0; i < n; ++i) { o[i] = c; c = c * x; }
    return o;
}
inline std::vector<E3> geometric_challenge(Transcript& t, size_t n) {  // geometric_challenge.hpp:39-44
    if (n == 0) return {};
    if (n == 1) return {E3::one()};
    return geometric(t.challenge_t(), n);
}
// acc[i] += scalar * eq(point, i), point[0] <-> most significant bit of i (multilinear.hpp:121-133)
inline void eval_eq_acc(std::vector<E3>& acc, const std::vector<E3>& pt, const E3& scalar) {
    std::vector<E3> w{scalar};
    for (const E3& x : pt) {
        std::vector<E3> nw(w.size() * 2);
        for (size_t j = 0; j < w.size(); ++j) {
            E3 hi = w[j] * x;
            nw[2 * j] = w[j] - hi;
            nw[2 * j + 1] = hi;
        }
        w.swap(nw);
    }
    for (size_t i = 0; i < acc.size(); ++i) acc[i] = acc[i] + w[i];
}
inline std::vector<E3> eq_weights(const std::vector<E3>& pt) {  // multilinear_point.hpp:40-62
    std::vector<E3> w(1ull << pt.size());
    eval_eq_acc(w, pt, E3::one());
    return w;
}
// acc[i] += sum_j scal[j] * pts[j]^i (utilities.hpp:261-307)
inline void geometric_accumulate(std::vector<E3>& acc, const std::vector<E3>& scal, const std::vector<E3>& pts) {
    const long long n = (long long)acc.size();
    const long long chunk = 4096;
#pragma omp parallel for schedule(static)
    for (long long c0 = 0; c0 < n; c0 += chunk) {
        std::vector<E3> cur(scal.size());
        for (size_t j = 0; j < scal.size(); ++j) cur[j] = scal[j] * e3pow(pts[j], (u64)c0);
        for (long long i = c0; i < std::min(n, c0 + chunk); ++i) {
            E3 e = acc[i];
            for (size_t j = 0; j < scal.size(); ++j) { e = e + cur[j]; cur[j] = cur[j] * pts[j]; }
            acc[i] = e;
        }
    }
}
// sum_i v_i z^i, base coefficients (utilities.hpp:196-246)
inline E3 univariate_eval_base(const std::vector<u64>& v, const E3& z) {
    E3 acc;
    for (size_t i = v.size(); i-- > 0;) { acc = acc * z; acc.c[0] = fadd(acc.c[0], v[i]); }
    return acc;
}
inline E3 univariate_eval_e3(const std::vector<E3>& v, const E3& z) {
    E3 acc;
    for (size_t i = v.size(); i-- > 0;) acc = acc * z + v[i];
    return acc;
}
// multilinear extension of base evaluations at an Ext3 point (multilinear.hpp:42-110)
inline E3 mle_eval_base(const std::vector<u64>& v, const std::vector<E3>& pt) {
    std::vector<E3> w = eq_weights(pt);
    E3 acc;
    for (size_t i = 0; i < v.size(); ++i) acc = acc + smul(w[i], v[i]);
    return acc;
}

// ---------------------------------------------------------------------------
// Sumcheck (sumcheck.hpp:43-116, sumcheck_protocol.hpp:81-144).
// ---------------------------------------------------------------------------
inline void fold(std::vector<E3>& v, const E3& r) {
    size_t h = v.size() / 2;
    for (size_t i = 0; i < h; ++i) v[i] = v[i] + (v[h + i] - v[i]) * r;
    v.resize(h);
}
inline std::vector<E3> sumcheck_prove(Transcript& t, const SumcheckCfg& cfg, std::vector<E3>& a,
                                      std::vector<E3>& b, E3& sum, Engine eng = Engine::Blake3) {
    std::vector<E3> rs;
    for (u64 r = 0; r < cfg.num_rounds; ++r) {
        size_t h = a.size() / 2;
        E3 c0, c2;
        for (size_t i = 0; i < h; ++i) {
            c0 = c0 + a[i] * b[i];
            c2 = c2 + (a[h + i] - a[i]) * (b[h + i] - b[i]);
        }
        E3 c1 = sum - (c0 + c0) - c2;
        t.message_t(c0);
        t.message_t(c2);
        pow_prove(t, cfg.pow_threshold, eng);
        E3 rnd = t.challenge_t();
        rs.push_back(rnd);
        fold(a, rnd);
        fold(b, rnd);
        sum = (c2 * rnd + c1) * rnd + c0;
    }
    return rs;
}

// ---------------------------------------------------------------------------
// IRS commit / open (irs_commit.hpp:344-713), witness kept in the oracle.
// ---------------------------------------------------------------------------
// Codeword order.  The C++ reference stores codeword rows in natural order
// (row i = evaluation at w_N^i, mod_ntt.hpp:49-130).  The Rust crate without
// its `rs_in_order` feature stores them coset-major
// (rust/src/algebra/ntt/cooley_tukey.rs:375-480): with coset size m (the
// message length) and e = N / m cosets, row k holds the evaluation at
// w_N^transpose_permute(k, e, m), transpose_permute(k, rows, cols) =
// k / cols + (k % cols) * rows (rust/src/algebra/ntt/transpose.rs:10-15).
// Opened rows are addressed by k and their evaluation points follow the same
// permutation (evaluation_points, cooley_tukey.rs:375-402).  Process-wide
// switch of the oracle (test infrastructure): false = natural order.
inline bool& coset_major_order() {
    static bool on = false;
    return on;
}
inline u64 transpose_permute(u64 k, u64 rows, u64 cols) { return k / cols + (k % cols) * rows; }
// Natural row index of committed row k of an N-row codeword of message length m.
inline u64 codeword_row(u64 k, u64 N, u64 m) {
    if (!coset_major_order() || m == 0 || N % m != 0) return k;
    return transpose_permute(k, N / m, m);
}

struct Witness {
    bool base = true;
    std::vector<u64> mat_base;   // row-major N x (nvec * depth) (initial commitment)
    std::vector<E3> mat_e3;      // row-major N x depth (round commitments)
    std::vector<Hash> nodes;     // Merkle node array
    u64 layers = 0, depth = 0, N = 0, nvec = 1;
    std::vector<E3> ood_points;
    std::vector<E3> ood_values;  // point-major: ood_values[j * nvec + v]
    Hash root() const { return nodes.back(); }
    u64 cols() const { return nvec * depth; }
};

// irs_commit::Config::commit (irs_commit.hpp:344-561) of `vs.size()` base
// vectors: row i of the matrix is (codeword_0[i] .. codeword_{d-1}[i]) of
// vector 0, then of vector 1, ... (mod_ntt.hpp:49-130: plane v * depth + b);
// the OOD values are sent point-major, every vector at each point (:472-554).
inline Witness commit_base_multi(Transcript& t, const IrsCfg& c, const std::vector<const std::vector<u64>*>& vs,
                                 Engine eng = Engine::Blake3) {
    Witness w;
    w.base = true; w.N = c.codeword_length; w.depth = c.depth; w.layers = layers_for(w.N);
    w.nvec = vs.size();
    const u64 cols = w.cols();
    w.mat_base.assign(w.N * cols, 0);
    for (u64 v = 0; v < w.nvec; ++v) {
        auto m = rs_encode_base(*vs[v], w.N, w.depth);
        for (u64 i = 0; i < w.N; ++i) {
            const u64 nat = codeword_row(i, w.N, c.msg_len());
            for (u64 b = 0; b < w.depth; ++b) w.mat_base[i * cols + v * w.depth + b] = m[nat * w.depth + b];
        }
    }
    w.nodes = merkle_build(leaves_base(w.mat_base, cols, eng), eng);
    t.message_hash(w.root());
    for (u64 s = 0; s < c.out_domain; ++s) w.ood_points.push_back(t.challenge_t());
    for (const E3& z : w.ood_points)
        for (u64 v = 0; v < w.nvec; ++v) {
            E3 val = univariate_eval_base(*vs[v], z);
            t.message_t(val);
            w.ood_values.push_back(val);
        }
    return w;
}
inline Witness commit_base(Transcript& t, const IrsCfg& c, const std::vector<u64>& v, Engine eng = Engine::Blake3) {
    return commit_base_multi(t, c, {&v}, eng);
}
inline Witness commit_e3(Transcript& t, const IrsCfg& c, const std::vector<E3>& v, Engine eng = Engine::Blake3) {
    Witness w;
    w.base = false; w.N = c.codeword_length; w.depth = c.depth; w.layers = layers_for(w.N);
    w.mat_e3 = rs_encode_e3(v, w.N, w.depth);
    if (coset_major_order()) {
        std::vector<E3> nat = w.mat_e3;
        for (u64 i = 0; i < w.N; ++i)
            for (u64 b = 0; b < w.depth; ++b)
                w.mat_e3[i * w.depth + b] = nat[codeword_row(i, w.N, c.msg_len()) * w.depth + b];
    }
    w.nodes = merkle_build(leaves_e3(w.mat_e3, w.depth, eng), eng);
    t.message_hash(w.root());
    for (u64 s = 0; s < c.out_domain; ++s) w.ood_points.push_back(t.challenge_t());
    for (const E3& z : w.ood_points) {
        E3 val = univariate_eval_e3(v, z);
        t.message_t(val);
        w.ood_values.push_back(val);
    }
    return w;
}
// indices_from_entropy (challenge_indices.hpp:56-98): ceil(log2 N / 8) bytes
// per index, big-endian, mod N; optional sort + dedup.
inline std::vector<u64> indices_from_entropy(const u8* ent, u64 N, u64 count, bool dedup) {
    if (count == 0) return {};
    if (N == 1) return dedup ? std::vector<u64>{0} : std::vector<u64>(count, 0);
    u64 nbytes = (layers_for(N) + 7) / 8;
    std::vector<u64> out;
    for (u64 i = 0; i < count; ++i) {
        u64 acc = 0;
        for (u64 b = 0; b < nbytes; ++b) acc = (acc << 8) | ent[i * nbytes + b];
        out.push_back(acc % N);
    }
    if (dedup) {
        std::sort(out.begin(), out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
    }
    return out;
}
// challenge_indices (challenge_indices.hpp:100-119), no dedup on the WHIR path;
// the bytes come from byte-wise squeezes, which read the XOF sequentially.
inline std::vector<u64> challenge_indices(Transcript& t, u64 N, u64 count) {
    if (count == 0) return {};
    if (N == 1) return std::vector<u64>(count, 0);
    u64 nbytes = (layers_for(N) + 7) / 8;
    std::vector<u8> ent(count * nbytes);
    t.squeeze(ent.data(), ent.size());
    return indices_from_entropy(ent.data(), N, count, false);
}
// irs_commit::Config::open (irs_commit.hpp:637-713) of one or more witnesses
// at the same challenged rows: per witness the row hint then its Merkle hints;
// the returned rows are the witnesses' rows side by side (stride sum of cols).
struct Opening { std::vector<E3> points; std::vector<E3> rows; u64 stride = 0; };  // rows lifted to Ext3
inline Opening open_witnesses(Transcript& t, const IrsCfg& c, const std::vector<const Witness*>& ws) {
    auto idx = challenge_indices(t, c.codeword_length, c.in_domain);
    Opening o;
    u64 gen = root_of_unity(c.codeword_length);
    for (u64 i : idx) o.points.push_back(E3::from_base(fpow(gen, codeword_row(i, c.codeword_length, c.msg_len()))));
    for (const Witness* w : ws) o.stride += w->cols();
    o.rows.assign(idx.size() * o.stride, E3());
    u64 col0 = 0;
    for (const Witness* w : ws) {
        const u64 cols = w->cols();
        t.hint_u64(idx.size() * cols);
        for (size_t q = 0; q < idx.size(); ++q)
            for (u64 col = 0; col < cols; ++col) {
                const u64 i = idx[q];
                if (w->base) {
                    u64 x = w->mat_base[i * cols + col];
                    t.hint_bytes(reinterpret_cast<const u8*>(&x), 8);
                    o.rows[q * o.stride + col0 + col] = E3::from_base(x);
                } else {
                    const E3& x = w->mat_e3[i * cols + col];
                    t.hint_bytes(reinterpret_cast<const u8*>(x.c), 24);
                    o.rows[q * o.stride + col0 + col] = x;
                }
            }
        for (const Hash& h : merkle_open(w->nodes, w->layers, idx)) t.hint_bytes(h.data(), 32);
        col0 += cols;
    }
    return o;
}
inline Opening open_witness(Transcript& t, const IrsCfg& c, const Witness& w) { return open_witnesses(t, c, {&w}); }

// ---------------------------------------------------------------------------
// Whole prover: Config::commit (once per witness) then Config::prove
// (whir.hpp:303-309, whir_prover.hpp:56-407) over num_witnesses * batch_size
// base vectors, MLE-point and/or dense-covector forms.
// ---------------------------------------------------------------------------
// Linear forms of the statement (linear_form.hpp:54-138): a MultilinearExtension
// at a point (accumulate = scalar * eq(point, .)) or a dense Covector
// (accumulate = scalar * vector).  `dense[f]` tells form f's kind; the
// points and covectors are listed in form order within their own kind.
struct Statement {
    std::vector<std::vector<E3>> mle_points;   // MultilinearExtension forms
    std::vector<std::vector<E3>> covectors;    // Covector forms
    std::vector<bool> dense;                   // per form; empty = MLE forms, then covectors
    std::vector<E3> evaluations;               // form-major: evaluations[f * num_vectors + v]
    size_t num_forms() const { return mle_points.size() + covectors.size(); }
    bool is_dense(size_t f) const { return dense.empty() ? f >= mle_points.size() : (bool)dense[f]; }
};
struct ProofOut { std::vector<u8> narg, hints; std::vector<E3> evaluation_point; Hash initial_root{}; };

// Commit + prove for an explicit configuration (a Config built field by field,
// as the reference's golden dumper does, or from_params), target field of
// degree `deg` (3: Basefield<GoldilocksExt3>, 1: Identity<Goldilocks>).
inline ProofOut prove_cfg(const WhirCfg& cfg, Engine eng, int deg, u64 B, const std::vector<std::vector<u64>>& vs,
                          u64 num_witnesses, const Statement& st, const DomainSep& ds) {
    const u64 W = num_witnesses, V = vs.size();
    if (B == 0 || W == 0 || V != W * B) throw std::runtime_error("vectors != witnesses * batch_size");
    if (deg != 1 && deg != 3) throw std::runtime_error("target field degree must be 1 or 3");
    const u64 size = vs[0].size();
    for (const auto& v : vs) if (v.size() != size) throw std::runtime_error("vector sizes differ");
    if (cfg.initial.vector_size != size) throw std::runtime_error("config size != vector size");
    Transcript t;
    t.deg = deg;
    t.absorb(ds.protocol_id, 64);
    t.absorb(ds.session_id, 32);
    ProofOut out;
    // commit: one witness of B vectors at a time, on the same transcript
    std::vector<Witness> wits;
    for (u64 w = 0; w < W; ++w) {
        std::vector<const std::vector<u64>*> mine;
        for (u64 b = 0; b < B; ++b) mine.push_back(&vs[w * B + b]);
        wits.push_back(commit_base_multi(t, cfg.initial, mine, eng));
    }
    out.initial_root = wits[0].root();
    const size_t nforms = st.num_forms();
    if (!st.dense.empty() && st.dense.size() != nforms) throw std::runtime_error("form kinds != forms");
    if (st.evaluations.size() != nforms * V) throw std::runtime_error("evaluations != forms * vectors");
    // step 1: OOD completion (whir_prover.hpp:92-120): every vector at every
    // witness's OOD points; values of other witnesses' vectors are sent.
    std::vector<E3> oods_pts, oods_mat;  // oods_mat[i * V + j]
    for (u64 w = 0; w < W; ++w)
        for (size_t e = 0; e < wits[w].ood_points.size(); ++e) {
            const E3& z = wits[w].ood_points[e];
            for (u64 j = 0; j < V; ++j) {
                if (j >= w * B && j < (w + 1) * B) {
                    oods_mat.push_back(wits[w].ood_values[e * B + (j - w * B)]);
                } else {
                    E3 val = univariate_eval_base(vs[j], z);
                    t.message_t(val);
                    oods_mat.push_back(val);
                }
            }
            oods_pts.push_back(z);
        }
    // step 2: vector RLC (:131-140)
    auto vrlc = geometric_challenge(t, V);
    std::vector<E3> vec(size);
    for (size_t i = 0; i < size; ++i) vec[i] = E3::from_base(vs[0][i]);
    for (u64 j = 1; j < V; ++j)
        for (size_t i = 0; i < size; ++i) vec[i] = vec[i] + smul(vrlc[j], vs[j][i]);
    // step 3: constraint RLC (:150-170)
    auto crlc = geometric_challenge(t, nforms + oods_pts.size());
    bool has_constraints = !crlc.empty();
    std::vector<E3> cov;
    if (nforms > 0 || has_constraints) cov.assign(size, E3());
    for (size_t f = 0, fm = 0, fc = 0; f < nforms; ++f) {
        E3 s = f == 0 ? E3::one() : crlc[f];  // linear_forms[0] with ONE (whir_prover.hpp:161)
        if (!st.is_dense(f)) eval_eq_acc(cov, st.mle_points[fm++], s);
        else {
            const auto& cv = st.covectors[fc++];
            if (cv.size() != cov.size()) throw std::runtime_error("covector size != vector size");
            for (size_t i = 0; i < cov.size(); ++i) cov[i] = cov[i] + s * cv[i];  // scalar_mul_add
        }
    }
    // step 4: the sum, a double RLC of the evaluation and OOD matrices (:172-197)
    E3 sum;
    for (size_t f = 0; f < nforms; ++f) {
        E3 row;
        for (u64 j = 0; j < V; ++j) row = row + vrlc[j] * st.evaluations[f * V + j];
        sum = sum + crlc[f] * row;
    }
    std::vector<E3> ood_rlc(crlc.begin() + (long)std::min(nforms, crlc.size()), crlc.end());
    if (!ood_rlc.empty()) geometric_accumulate(cov, ood_rlc, oods_pts);
    for (size_t i = 0; i < ood_rlc.size(); ++i) {
        E3 row;
        for (u64 j = 0; j < V; ++j) row = row + vrlc[j] * oods_mat[i * V + j];
        sum = sum + ood_rlc[i] * row;
    }
    // step 5: initial sumcheck
    std::vector<E3> last_r;
    if (has_constraints) last_r = sumcheck_prove(t, cfg.initial_sumcheck, vec, cov, sum, eng);
    else {
        for (u64 r = 0; r < cfg.initial_sumcheck.num_rounds; ++r) last_r.push_back(t.challenge_t());
        pow_prove(t, cfg.initial_skip_pow, eng);
        for (const E3& r : last_r) fold(vec, r);
        cov.assign(cfg.initial_sumcheck.initial_size >> cfg.initial_sumcheck.num_rounds, E3());
    }
    out.evaluation_point = last_r;
    // step 6: rounds.  The first opening covers every initial witness and
    // weighs its rows by vector_rlc (x) eq(last folding randomness) (:283-310).
    std::vector<const Witness*> prev;
    for (const Witness& w : wits) prev.push_back(&w);
    const IrsCfg* prev_cfg = &cfg.initial;
    std::vector<E3> wrlc = vrlc;
    std::vector<Witness> stored;
    stored.reserve(cfg.rounds.size());
    for (size_t rd = 0; rd < cfg.rounds.size(); ++rd) {
        const RoundCfg& rc = cfg.rounds[rd];
        if (deg == 1) {  // base-field round vector: 8-byte row elements
            std::vector<u64> b(vec.size());
            for (size_t i = 0; i < vec.size(); ++i) b[i] = vec[i].c[0];
            stored.push_back(commit_base(t, rc.irs, b, eng));
        } else {
            stored.push_back(commit_e3(t, rc.irs, vec, eng));
        }
        const Witness& nw = stored.back();
        pow_prove(t, rc.pow_threshold, eng);
        Opening o = open_witnesses(t, *prev_cfg, prev);
        std::vector<E3> pts = nw.ood_points;
        pts.insert(pts.end(), o.points.begin(), o.points.end());
        std::vector<E3> vals = nw.ood_values;
        std::vector<E3> eqw = last_r.empty() ? std::vector<E3>{E3::one()} : eq_weights(last_r);
        std::vector<E3> tp;  // tensor_product(vector_rlc, eq_weights) (utilities.hpp:137-150)
        for (const E3& a : wrlc) for (const E3& b : eqw) tp.push_back(a * b);
        if (tp.size() != o.stride) throw std::runtime_error("opened row width != tensor product");
        for (size_t q = 0; q < o.points.size(); ++q) {
            E3 acc;
            for (size_t col = 0; col < o.stride; ++col) acc = acc + o.rows[q * o.stride + col] * tp[col];
            vals.push_back(acc);
        }
        auto srlc = geometric_challenge(t, pts.size());
        geometric_accumulate(cov, srlc, pts);
        for (size_t j = 0; j < srlc.size(); ++j) sum = sum + srlc[j] * vals[j];
        last_r = sumcheck_prove(t, rc.sumcheck, vec, cov, sum, eng);
        out.evaluation_point.insert(out.evaluation_point.end(), last_r.begin(), last_r.end());
        prev = {&nw};
        prev_cfg = &rc.irs;
        wrlc = {E3::one()};
    }
    // steps 7-10
    for (const E3& c : vec) t.message_t(c);
    pow_prove(t, cfg.final_pow, eng);
    open_witnesses(t, *prev_cfg, prev);
    auto fr = sumcheck_prove(t, cfg.final_sumcheck, vec, cov, sum, eng);
    out.evaluation_point.insert(out.evaluation_point.end(), fr.begin(), fr.end());
    out.narg = std::move(t.narg);
    out.hints = std::move(t.hints);
    return out;
}
inline ProofOut prove_multi(const Params& p, const std::vector<std::vector<u64>>& vs, u64 num_witnesses,
                            const Statement& st, const DomainSep& ds, int deg = 3) {
    if (vs.empty()) throw std::runtime_error("no vectors");
    const WhirCfg cfg = whir_from_params(vs[0].size(), p, deg == 1 ? 64.0 : 192.0);
    const Engine eng = std::memcmp(p.hash_id, SHA2_ENGINE_ID, 32) == 0 ? Engine::Sha2 : Engine::Blake3;
    return prove_cfg(cfg, eng, deg, p.batch_size, vs, num_witnesses, st, ds);
}
inline ProofOut prove(const Params& p, const std::vector<u64>& v, const Statement& st, const DomainSep& ds) {
    if (p.batch_size != 1) throw std::runtime_error("prove(): one vector; use prove_multi");
    return prove_multi(p, {v}, 1, st, ds);
}

}  // namespace oracle
