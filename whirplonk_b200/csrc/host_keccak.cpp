// host_keccak.cpp -- Keccak-f[1600] and SHAKE128 absorption on the host CPU
// (see host_keccak.h).  Constants are derived from their FIPS 202 definitions
// at compile time (round-constant LFSR x^8+x^6+x^5+x^4+1; rho offsets
// (t+1)(t+2)/2 along the (x,y) -> (y, 2x+3y) orbit), as for the device sponge.
#include "host_keccak.h"

#include <cstring>

namespace wg {
namespace {

constexpr int rc_bit(int t) {
    int r = 0x80;
    for (int i = 1; i <= t % 255; ++i) {
        const int r8 = r & 1;
        r >>= 1;
        if (r8) r ^= 0x8E;
    }
    return (t % 255 == 0) ? 1 : ((r >> 7) & 1);
}
constexpr uint64_t round_constant(int round) {
    uint64_t v = 0;
    for (int j = 0; j <= 6; ++j)
        if (rc_bit(j + 7 * round)) v |= 1ull << ((1 << j) - 1);
    return v;
}
constexpr int rho_offset(int x, int y) {
    if (x == 0 && y == 0) return 0;
    int cx = 1, cy = 0;
    for (int t = 0; t < 24; ++t) {
        if (cx == x && cy == y) return ((t + 1) * (t + 2) / 2) % 64;
        const int nx = cy, ny = (2 * cx + 3 * cy) % 5;
        cx = nx;
        cy = ny;
    }
    return 0;
}
struct Tables {
    int rho[25];
    uint64_t rc[24];
    constexpr Tables() : rho(), rc() {
        for (int i = 0; i < 25; ++i) rho[i] = rho_offset(i % 5, i / 5);
        for (int r = 0; r < 24; ++r) rc[r] = round_constant(r);
    }
};
constexpr Tables KT{};

inline uint64_t rotl(uint64_t v, int s) { return s ? (v << s) | (v >> (64 - s)) : v; }

constexpr unsigned RATE = 168;

}  // namespace

// The state is copied to a local array whose fully unrolled accesses the
// compiler keeps in registers.
void keccak_f1600_cpu(uint64_t s[25]) {
    uint64_t A[25];
#pragma GCC unroll 25
    for (int i = 0; i < 25; ++i) A[i] = s[i];
    for (int round = 0; round < 24; ++round) {
        uint64_t C[5], D[5], B[25];
#pragma GCC unroll 5
        for (int x = 0; x < 5; ++x) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
#pragma GCC unroll 5
        for (int x = 0; x < 5; ++x) D[x] = C[(x + 4) % 5] ^ rotl(C[(x + 1) % 5], 1);
#pragma GCC unroll 25
        for (int i = 0; i < 25; ++i) A[i] ^= D[i % 5];
#pragma GCC unroll 5
        for (int y = 0; y < 5; ++y)
#pragma GCC unroll 5
            for (int x = 0; x < 5; ++x) B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(A[x + 5 * y], KT.rho[x + 5 * y]);
#pragma GCC unroll 5
        for (int y = 0; y < 5; ++y)
#pragma GCC unroll 5
            for (int x = 0; x < 5; ++x) A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
        A[0] ^= KT.rc[round];
    }
#pragma GCC unroll 25
    for (int i = 0; i < 25; ++i) s[i] = A[i];
}

void host_absorb_message_words(uint64_t hasher[25], unsigned& hpos, const uint64_t* w, size_t nw, uint8_t* narg_out,
                               size_t& pos) {
    for (size_t i = 0; i < nw; ++i) {
        const uint64_t v = w[i];
        if ((hpos & 7) == 0) {
            hasher[hpos >> 3] ^= v;
            hpos += 8;
            if (hpos == RATE) {
                keccak_f1600_cpu(hasher);
                hpos = 0;
            }
        } else {
            for (int b = 0; b < 8; ++b) {
                hasher[hpos >> 3] ^= ((v >> (8 * b)) & 0xFF) << (8 * (hpos & 7));
                if (++hpos == RATE) {
                    keccak_f1600_cpu(hasher);
                    hpos = 0;
                }
            }
        }
        std::memcpy(narg_out + pos, &v, 8);  // LE host
        pos += 8;
    }
}

}  // namespace wg
