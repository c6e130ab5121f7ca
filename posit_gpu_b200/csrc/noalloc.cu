// noalloc.cu -- posit_rgemm_dev_noalloc: the device GEMM for callers that cannot
// allocate device memory.
//
// Who needs it: a host program whose memory manager reserves the GPU's memory up front
// and hands out sub-buffers itself (a cudaMalloc from inside this library would fail or
// break its budget), or a latency-critical loop that must not call cudaMalloc/cudaFree
// because they can synchronise the whole device.  posit_rgemm_dev needs a scratch
// workspace for the decoded operand tiles and either allocates it or takes one from the
// caller; this entry point takes neither: its scratch is a fixed array compiled into the
// library.
//
// The array, g_noalloc_scratch, is a file-scope __device__ object of
// POSIT_NOALLOC_SCRATCH_BYTES (64 MiB).  Every GPU that loads this library holds those
// 64 MiB until the process exits.  Host code must not pass the symbol itself to a
// kernel (on the host it names a shadow object, not device memory): the first call on
// each device looks up the array's device address with cudaGetSymbolAddress, with that
// device current, and caches it.  Make that first call before any stream capture.  A
// cudaDeviceReset unloads the module and with it the array; the cached address is then
// stale, so do not call this entry point again in a process that has reset the device.
//
// All calls on a device share the one array and it keeps whatever the last call left in
// it.  Nothing in it has to start at zero from an earlier call: on every call the GEMM
// launch clears the region of per-row and per-column NaR flags (a stream-ordered memset)
// before the decode pre-pass sets the flags it finds, and the decode pre-pass writes every
// byte of the operand-tile region before the main kernel reads it.  Two calls whose work
// overlaps on the GPU (e.g. issued on different streams without ordering) race on the
// array.
#include "../../include/posit_gpu.h"
#include "gemm.cuh"

#include <cuda_runtime.h>
#include <mutex>

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[POSIT_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_dev_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch for the current device (looked up once per device).
int scratch_for_current_device(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return POSIT_E_NO_DEVICE;
    if (dev < 0 || dev >= kMaxDevices)
        return POSIT_E_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return POSIT_E_CUDA;
        g_scratch_dev_ptr[dev] = p;
    }
    *out = g_scratch_dev_ptr[dev];
    return 0;
}

} // namespace

extern "C" int posit_rgemm_dev_noalloc(char transa, char transb, int m, int n, int k, uint32_t alpha,
                                       const uint32_t *A, int lda, const uint32_t *B, int ldb, uint32_t beta,
                                       uint32_t *C, int ldc, void *stream)
{
    // The Rgemm argument checks come first, so a bad argument gets its info code whatever
    // the shape.
    bool nota, notb;
    const int info = pg::rgemm_check_args(transa, transb, m, n, k, lda, ldb, ldc, nota, notb);
    if (info)
        return info;
    // Only a call that runs the main GEMM (alpha != 0, k > 0, a non-empty C) uses scratch;
    // the quick returns and the calls that only scale C need none and are never refused.
    const bool uses_scratch = m > 0 && n > 0 && k > 0 && alpha != 0;
    if (uses_scratch &&
        posit_rgemm_workspace_size(transa, transb, m, n, k) > (size_t)POSIT_NOALLOC_SCRATCH_BYTES)
        return POSIT_E_NOALLOC_LIMIT;
    void *scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc)
        return rc;
    // With a caller-supplied workspace posit_rgemm_dev makes no allocation.
    return posit_rgemm_dev(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, scratch,
                           (size_t)POSIT_NOALLOC_SCRATCH_BYTES, stream);
}
