// k_noalloc.cu -- multilinear-extension evaluation that allocates nothing.
//
// Some callers cannot call cudaMalloc on the path where they need this value:
// code running inside a host callback or a driver hook, callers whose device
// memory is carved out by their own pool or arena and that must not take the
// runtime allocator's locks (or let it synchronise the device), and
// latency-critical loops where an allocation on the first call would stall.
// For them this entry point keeps its working memory in a fixed file-scope
// __device__ array instead of asking the runtime for it; inputs and the output
// are device buffers the caller already owns.
//
// The array lives on every GPU that loads this library, from load until the
// process exits (NOALLOC_SCRATCH_BYTES, under half a MiB).  All calls on one
// device share it and it keeps the previous call's contents: the ticket counter
// that must start at zero is cleared on the caller's stream before each launch,
// and two calls whose kernels overlap on the GPU (different streams, no
// ordering between them) race on the array and give wrong results.
#include <cuda_runtime.h>

#include "../../include/whirgpu.h"
#include "launch.h"

namespace wg {

// Layout used by launch_mle_eval: [ticket | 592 CTA partials | eq tables].
// 2^24 coefficients need (2^10 + 2^14) table entries of 24 B.
constexpr size_t NOALLOC_SCRATCH_BYTES = 448u * 1024u;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of g_noalloc_scratch on the current device.  The host-side
// symbol is only a stand-in and must never reach a kernel.  The address is
// looked up on every call (the lookup allocates nothing), so it stays right
// after a cudaDeviceReset reloads the module.  The first lookup on a device
// may load the library's module there, which is why the first call on a device
// must come before any stream capture.
cudaError_t scratch_for_current_device(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = p;
    return cudaSuccess;
}
}  // namespace

}  // namespace wg

extern "C" whirgpu_status whirgpu_mle_evaluate_noalloc(const uint64_t* d_coeffs, uint64_t num_variables,
                                                       const uint64_t* d_point, uint64_t* d_out, void* stream) {
    using namespace wg;
    if (!d_coeffs || !d_point || !d_out) return WHIRGPU_E_INVALID;
    if (num_variables > WHIRGPU_NOALLOC_MLE_MAX_VARS) return WHIRGPU_E_TOO_LARGE;
    if (mle_eval_scratch_bytes((u32)num_variables) > NOALLOC_SCRATCH_BYTES) return WHIRGPU_E_TOO_LARGE;
    // A launch error still pending on this thread belongs to the caller's
    // earlier work: leave it for its owner (cudaGetLastError would clear it)
    // and queue nothing.  With none pending, any error seen below is ours.
    if (cudaPeekAtLastError() != cudaSuccess) return WHIRGPU_E_CUDA;
    void* scratch = nullptr;
    if (scratch_for_current_device(&scratch) != cudaSuccess) {
        cudaGetLastError();  // clear this call's own lookup error
        return WHIRGPU_E_CUDA;
    }
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (launch_mle_eval(d_coeffs, (u32)num_variables, d_point, scratch, d_out, st) != 0) {
        cudaGetLastError();  // clear this call's own memset or launch error
        return WHIRGPU_E_CUDA;
    }
    return WHIRGPU_OK;
}
