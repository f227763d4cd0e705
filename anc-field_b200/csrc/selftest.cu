// Self-test of the bounded device waits (afd_wait_selftest): one block
// waits on a shared-memory mbarrier with the streaming kernel's wait
// (fused.cuh, which = 0) or the GEMM kernels' wait (tc.cuh, which = 1).
// With `complete` = 0 nothing ever arrives on the barrier, so the wait gives
// up at its time limit; the kernel records that and the time it waited and
// returns normally, so the host reads a status and the context stays usable.
#include <cuda_runtime.h>

#include "afd.h"
#include "fused.cuh"
#include "tc.cuh"

namespace afd {
namespace {

__global__ void k_wait_selftest(int which, int complete, unsigned long long* out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (complete) mbar_arrive(&bar);
    const unsigned long long t0 = global_ns();
    const bool ok = which == 0 ? mbar_wait(&bar, 0) : tc::bar_wait(&bar, 0);
    out[0] = ok ? 0ull : 1ull;
    out[1] = global_ns() - t0;
}

}  // namespace
}  // namespace afd

extern "C" int afd_wait_selftest(int32_t device, int32_t which, int32_t complete, int32_t* timed_out,
                                 int64_t* waited_ns) {
    if ((which != 0 && which != 1) || !timed_out || !waited_ns) return AFD_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return AFD_ERR_CUDA;
    if (device < 0 || device >= ndev) return AFD_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return AFD_ERR_CUDA;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(unsigned long long)) != cudaSuccess) return AFD_ERR_CUDA;
    afd::k_wait_selftest<<<1, 32>>>(which, complete != 0, d);
    unsigned long long h[2] = {0ull, 0ull};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return AFD_ERR_CUDA;
    *timed_out = (int32_t)h[0];
    *waited_ns = (int64_t)h[1];
    return AFD_OK;
}
