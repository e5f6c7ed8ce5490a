// Self-check of the device's bounded waits.
//
// Every wait in this library's kernels has a cycle budget: a tensor-core
// kernel whose mbarrier phase never completes gives up, sets the context's
// device error word and returns, and the next synchronising call reports
// FS_ERR_DEVICE instead of hanging the GPU.  fs_gpu_check_bounded_wait runs
// that path on purpose, safely: one CTA waits, through the same wait routine
// and with the caller's (short) budget, on a freshly initialised mbarrier
// that nothing arrives at and no copy or MMA is bound to.
#include "internal.cuh"
#include "tc_common.cuh"

using namespace fsg;

namespace fsg {
namespace {

__global__ void bounded_wait_probe_kernel(long long budget, int32_t *__restrict__ err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  __syncthreads();
  // phase 0 of a barrier expecting one arrival, which never comes
  if (threadIdx.x == 0 && !tc::mbar_wait(&bar, 0, budget)) atomicExch(err, 1);
}

} // namespace
} // namespace fsg

extern "C" int fs_gpu_check_bounded_wait(fs_gpu *h, int64_t cycles) {
  if (!h) return FS_ERR_ARG;
  if (cycles < 1 || cycles > tc::kWaitCycles)
    return set_error(h, FS_ERR_ARG, "check_bounded_wait: cycles must be in [1, " + std::to_string(tc::kWaitCycles) + "]");
  cudaSetDevice(h->device);
  if (!h->d_err) {
    FS_CUDA(cudaMalloc(&h->d_err, sizeof(int32_t)));
    FS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int32_t), h->stream));
  }
  bounded_wait_probe_kernel<<<1, 32, 0, h->stream>>>(static_cast<long long>(cycles), h->d_err);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  return sync_checked(h);
}
