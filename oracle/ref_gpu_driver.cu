// ref_gpu_driver.cu -- test infrastructure, NOT product code.
//
// Runs the reference's own CUDA side-car (hxd77/WhirPlonk cpp/cuda, compiled
// unmodified for sm_100a by oracle/Makefile with WHIR_CUDA and
// WHIR_CUDA_EXPERIMENTAL_NTT defined, as the reference CMake does for a CUDA
// build) on the kernel-level commitment, through the calls
// irs_commit::Config::commit makes (irs_commit.hpp:382-391, 440-455): per
// vector, the Goldilocks NTT engine's RS encode + BLAKE3 leaf hashes on the GPU
// (NttEngine::try_gpu_interleaved_rs_encode_blake3_matrix_leaves,
// cooley_tukey.hpp:560-612, which uploads its roots table and calls
// whir::cuda::gpu_interleaved_rs_encode_blake3_matrix_leaves), then the GPU
// Merkle root (whir::cuda::gpu_blake3_merkle_tree, cuda_integration.hpp:942-993).
// Host buffers in and out, as that API takes them.  bench.py uses it as the
// same-box reference GPU arm of the kernel-level workload and checks its roots
// against the library's.
//
// Input file (little endian): u32 magic 0x47505552 ('RUPG'), u32 version 1,
//   u64 count, log_len, log_expansion, log_depth, reps,
//   count * 2^log_len u64 coefficients (canonical, < p).
// Output file: count * 32 root bytes, then f64 ms of one pass over the count
//   vectors (the median of `reps` timed passes after one warm-up pass).
#include "whir/algebra/goldilocks.hpp"
#include "whir/algebra/ntt/cooley_tukey_goldilocks.hpp"
#include "whir/hash/hash_engine.hpp"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <span>
#include <vector>

namespace {

[[noreturn]] void die(const char* msg) {
    std::fprintf(stderr, "ref_gpu_driver: %s\n", msg);
    std::exit(2);
}

struct Header {
    uint32_t magic, version;
    uint64_t count, log_len, log_exp, log_depth, reps;
};

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) die("usage: ref_gpu_driver IN OUT");
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) die("cannot open input");
    Header h{};
    if (std::fread(&h, sizeof(h), 1, f) != 1 || h.magic != 0x47505552u || h.version != 1) die("bad header");
    if (h.log_len < h.log_depth || h.log_len > 26 || h.log_exp < 1 || h.log_exp > 4 || h.count == 0 || h.reps == 0)
        die("unsupported sizes");
    const uint64_t len = 1ull << h.log_len, depth = 1ull << h.log_depth;
    const uint64_t N = (len / depth) << h.log_exp;
    using G = ::whir::algebra::Goldilocks;
    std::vector<G> coeffs(h.count * len);
    {
        std::vector<uint64_t> raw(h.count * len);
        if (std::fread(raw.data(), 8, raw.size(), f) != raw.size()) die("short input");
        for (size_t i = 0; i < raw.size(); ++i) coeffs[i] = G::from_u64(raw[i]);
    }
    std::fclose(f);

    auto& engine = ::whir::algebra::ntt::goldilocks_engine();
    std::vector<G> matrix;
    std::vector<::whir::hash::Hash> leaves;
    std::vector<uint8_t> roots(h.count * 32);
    auto pass = [&]() {
        for (uint64_t v = 0; v < h.count; ++v) {
            const std::span<const G> vec(coeffs.data() + v * len, len);
            const std::span<const std::span<const G>> vecs(&vec, 1);
            if (!engine.try_gpu_interleaved_rs_encode_blake3_matrix_leaves(vecs, N, depth, matrix, leaves))
                die("the reference GPU path declined this shape");
            whir::cuda::gpu_blake3_merkle_tree(reinterpret_cast<const uint8_t*>(leaves.data()), leaves.size(),
                                               roots.data() + 32 * v);
        }
    };
    pass();  // warm-up: the reference's memory pool grows to this shape
    std::vector<double> ms;
    for (uint64_t r = 0; r < h.reps; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        pass();
        ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
    std::sort(ms.begin(), ms.end());
    const double med = ms[ms.size() / 2];

    FILE* o = std::fopen(argv[2], "wb");
    if (!o) die("cannot open output");
    std::fwrite(roots.data(), 1, roots.size(), o);
    std::fwrite(&med, sizeof(med), 1, o);
    std::fclose(o);
    return 0;
}
