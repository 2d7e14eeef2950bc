// k_diag.cu -- diagnostics: runs the device field arithmetic on caller-supplied
// operands so tests can check it against exact integer arithmetic.
#include <cuda_runtime.h>

#include "../../include/whirgpu.h"
#include "gl.cuh"
#include "launch.h"

namespace wg {

// op 0: a+b  1: a-b  2: a*b  (base field, one word each)
// op 3: Ext3 a*b (three words each)
__global__ void k_field_ops(const u64* a, const u64* b, u64* out, u64 n, int op) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        if (op == 0) out[i] = gl_add(a[i], b[i]);
        else if (op == 1) out[i] = gl_sub(a[i], b[i]);
        else if (op == 2) out[i] = gl_mul(a[i], b[i]);
        else {
            const E3 r = e3_mul(E3{a[3 * i], a[3 * i + 1], a[3 * i + 2]}, E3{b[3 * i], b[3 * i + 1], b[3 * i + 2]});
            out[3 * i] = r.c0;
            out[3 * i + 1] = r.c1;
            out[3 * i + 2] = r.c2;
        }
    }
}

}  // namespace wg

extern "C" whirgpu_status whirgpu_debug_field_ops(const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t n,
                                                  int op) {
    using namespace wg;
    if (!a || !b || !out || op < 0 || op > 3) return WHIRGPU_E_INVALID;
    const u64 words = n * (op == 3 ? 3 : 1);
    u64 *da = nullptr, *db = nullptr, *dout = nullptr;
    if (cudaMalloc(&da, words * 8 + 8) != cudaSuccess) return WHIRGPU_E_OOM;
    if (cudaMalloc(&db, words * 8 + 8) != cudaSuccess) { cudaFree(da); return WHIRGPU_E_OOM; }
    if (cudaMalloc(&dout, words * 8 + 8) != cudaSuccess) { cudaFree(da); cudaFree(db); return WHIRGPU_E_OOM; }
    whirgpu_status st = WHIRGPU_OK;
    if (cudaMemcpy(da, a, words * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db, b, words * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
        st = WHIRGPU_E_CUDA;
    } else {
        const u64 blocks = (n + 255) / 256;
        k_field_ops<<<(unsigned)(blocks > 4096 ? 4096 : (blocks ? blocks : 1)), 256>>>(da, db, dout, n, op);
        count_launches(1);
        if (cudaMemcpy(out, dout, words * 8, cudaMemcpyDeviceToHost) != cudaSuccess) st = WHIRGPU_E_CUDA;
    }
    cudaFree(da);
    cudaFree(db);
    cudaFree(dout);
    return st;
}
