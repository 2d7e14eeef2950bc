// host_keccak.h -- Keccak-f[1600] and SHAKE128 absorption on the host CPU.
//
// Used where the transcript absorbs a long run of prover messages at once:
// the sponge is inherently sequential, and one CPU core runs a permutation
// several times faster than one GPU warp, so such a run is absorbed on the
// host between two device phases.  Byte semantics are those of the device
// transcript (transcript.cuh): absorb continues the hasher at byte position
// hpos of the 168-byte rate and permutes when it is full.
#pragma once
#include <cstddef>
#include <cstdint>

namespace wg {

// Keccak-f[1600] (FIPS 202), state lane x + 5 y at s[x + 5 y].
void keccak_f1600_cpu(uint64_t s[25]);

// Absorbs nw 64-bit LE words into (hasher, hpos) and appends their bytes at
// narg_out[pos ..]; pos advances by 8 nw.
void host_absorb_message_words(uint64_t hasher[25], unsigned& hpos, const uint64_t* w, size_t nw, uint8_t* narg_out,
                               size_t& pos);

}  // namespace wg
