// k_peaks.cu -- integer-pipe peaks of the GPU, measured: the roofline
// denominators of the kernel families that the integer pipes bound rather than
// HBM (NTT butterflies, BLAKE3 compressions, 192-bit multiply-accumulates).
//
// Each kernel runs the operation on registers only -- independent chains per
// thread, no memory traffic in the loop -- over a full grid of resident CTAs,
// timed with CUDA events.  The field and hash operations are the library's own
// (gl_mul / gl_add / gl_sub, b3_compress, acc_mac), so a family's fraction of
// its peak says how much of the issue rate its memory access, shuffles and
// addressing cost.  The raw per-instruction rates (32-bit multiply-add, wide
// multiply, three-input add, lop3, funnel shift) are reported beside them.
#include <cuda_runtime.h>

#include "../../include/whirgpu.h"
#include "blake3.cuh"
#include "gl.cuh"
#include "launch.h"

namespace wg {

constexpr int PK_THREADS = 256, PK_CHAINS = 8;

__device__ __forceinline__ u64 pk_seed(u64 s, u32 c) {
    const u64 v = (s + 0x9E3779B97F4A7C15ull * (threadIdx.x + 1 + 977ull * (blockIdx.x + 1))) ^ ((u64)c << 40);
    return v % GL_P;
}

// Radix-2 Goldilocks butterflies (x, y) <- (x + w y, x - w y).
__global__ void __launch_bounds__(PK_THREADS) k_peak_bfly(u64* sink, u32 iters, u64 seed) {
    u64 x[PK_CHAINS], y[PK_CHAINS], w[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) {
        x[c] = pk_seed(seed, c);
        y[c] = pk_seed(seed ^ 0x5555, c);
        w[c] = pk_seed(seed ^ 0xAAAA, c);
    }
    for (u32 it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) {
            const u64 t = gl_mul(y[c], w[c]);
            const u64 a = gl_add(x[c], t);
            y[c] = gl_sub(x[c], t);
            x[c] = a;
        }
    }
    u64 r = 0;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) r ^= x[c] ^ y[c];
    sink[(u64)blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// 64x64-bit products accumulated into 192-bit sums (acc_mac).
__global__ void __launch_bounds__(PK_THREADS) k_peak_mac(u64* sink, u32 iters, u64 seed) {
    Acc192 s[PK_CHAINS];
    u64 a[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) {
        s[c] = Acc192{0, 0, 0};
        a[c] = pk_seed(seed, c);
    }
    u64 b = pk_seed(seed ^ 0x1234, 99);
    for (u32 it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) acc_mac(s[c], a[c], b);
        b += 0x9E3779B97F4A7C15ull;
    }
    u64 r = 0;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) r ^= s[c].w0 ^ s[c].w1 ^ s[c].w2;
    sink[(u64)blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// BLAKE3 compressions, two independent chaining values per thread.
__global__ void __launch_bounds__(PK_THREADS) k_peak_b3(u64* sink, u32 iters, u64 seed) {
    unsigned cv0[8], cv1[8], m[16];
    b3_init(cv0);
    b3_init(cv1);
#pragma unroll
    for (int i = 0; i < 16; ++i) m[i] = (unsigned)pk_seed(seed, i);
    for (u32 it = 0; it < iters; ++it) {
        b3_compress(cv0, m, B3_CHUNK_START);
        b3_compress(cv1, m, B3_CHUNK_END);
#pragma unroll
        for (int i = 0; i < 8; ++i) m[i] ^= cv1[i];
    }
    u64 r = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) r ^= (u64)cv0[i] << 32 | cv1[i];
    sink[(u64)blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// Raw instruction rates: OP 0 mad.lo.u32, 1 mad.wide.u32, 2 three-input
// add.u32, 3 lop3.b32, 4 shf.l.wrap.b32; 8 independent chains, operands
// rotating between chains so no chain folds to a constant.
template <int OP>
__global__ void __launch_bounds__(PK_THREADS) k_peak_op(u64* sink, u32 iters, u64 seed) {
    unsigned a[PK_CHAINS];
    u64 w[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) {
        a[c] = (unsigned)pk_seed(seed, c) | 1u;
        w[c] = pk_seed(seed ^ 0x77, c);
    }
    for (u32 it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) {
            const unsigned b = a[(c + 1) % PK_CHAINS], d = a[(c + 3) % PK_CHAINS];
            if (OP == 0) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
            if (OP == 1) asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(w[c]) : "r"((unsigned)w[c]), "r"(b));
            if (OP == 2) asm volatile("add.u32 %0, %0, %1;\n\tadd.u32 %0, %0, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
            if (OP == 3) asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[c]) : "r"(b), "r"(d));
            if (OP == 4) asm volatile("shf.l.wrap.b32 %0, %0, %1, %2;" : "+r"(a[c]) : "r"(b), "r"(d));
        }
    }
    u64 r = 0;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) r ^= a[c] ^ w[c];
    sink[(u64)blockIdx.x * blockDim.x + threadIdx.x] = r;
}

}  // namespace wg

namespace {
using namespace wg;

// Operations per second of one kernel: a warm-up launch, then a launch timed
// with events on `st`.
template <typename K>
double measure(K kernel, unsigned grid, u64* sink, u32 iters, double ops_per_thread_iter, cudaStream_t st,
               whirgpu_status* status) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) { *status = WHIRGPU_E_CUDA; return 0; }
    if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); *status = WHIRGPU_E_CUDA; return 0; }
    kernel<<<grid, PK_THREADS, 0, st>>>(sink, iters / 8 + 1, 7);
    cudaEventRecord(a, st);
    kernel<<<grid, PK_THREADS, 0, st>>>(sink, iters, 11);
    cudaEventRecord(b, st);
    count_launches(2);
    float ms = 0;
    if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess || ms <= 0)
        *status = WHIRGPU_E_CUDA;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms > 0 ? (double)grid * PK_THREADS * iters * ops_per_thread_iter / (ms * 1e-3) : 0.0;
}
}  // namespace

extern "C" whirgpu_status whirgpu_measure_int_peaks(int device, double out[WHIRGPU_NUM_INT_PEAKS]) {
    using namespace wg;
    if (!out) return WHIRGPU_E_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return WHIRGPU_E_CUDA;
    const u32 sms = device_sms();
    const unsigned grid = sms * 8;  // 8 CTAs of 256 threads per SM: 64 warps, a full SM
    u64* sink = nullptr;
    if (cudaMalloc(&sink, (size_t)grid * PK_THREADS * 8) != cudaSuccess) return WHIRGPU_E_OOM;
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaFree(sink);
        return WHIRGPU_E_CUDA;
    }
    whirgpu_status s = WHIRGPU_OK;
    out[0] = measure(k_peak_bfly, grid, sink, 4096, PK_CHAINS, st, &s);
    out[1] = measure(k_peak_b3, grid, sink, 1024, 2, st, &s);
    out[2] = measure(k_peak_mac, grid, sink, 8192, PK_CHAINS, st, &s);
    out[3] = measure(k_peak_op<0>, grid, sink, 65536, PK_CHAINS, st, &s);
    out[4] = measure(k_peak_op<1>, grid, sink, 32768, PK_CHAINS, st, &s);
    out[5] = measure(k_peak_op<2>, grid, sink, 65536, PK_CHAINS, st, &s);
    out[6] = measure(k_peak_op<3>, grid, sink, 65536, PK_CHAINS, st, &s);
    out[7] = measure(k_peak_op<4>, grid, sink, 65536, PK_CHAINS, st, &s);
    cudaStreamDestroy(st);
    cudaFree(sink);
    return s;
}
