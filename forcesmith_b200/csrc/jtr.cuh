// Jᵀr for a column-major J (leading dimension ld, M rows, D columns) against
// the FP64 residual F, in two passes: CTA (chunk, column) sums its slice of
// the column's rows in FP64 into part[column][chunk], then one CTA per column
// adds its chunks in order (deterministic).  A CTA per column alone leaves
// most SMs idle when D is small.
#pragma once

#include "spline_dev.cuh"

#include <algorithm>

namespace fsg {
namespace {

constexpr int kJtrChunks = 128;

template <class T>
__global__ void jtr_chunk_kernel(const T *__restrict__ J, int64_t ld, int64_t M, const double *__restrict__ F,
                                 double *__restrict__ part) {
  __shared__ double r[32];
  const int64_t len = (M + gridDim.x - 1) / gridDim.x;
  const int64_t k0 = static_cast<int64_t>(blockIdx.x) * len, k1 = min(M, k0 + len);
  const T *Jc = J + static_cast<int64_t>(blockIdx.y) * ld;
  double s = 0.0;
  for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) s += static_cast<double>(Jc[k]) * F[k];
  s = block_sum(s, r);
  if (threadIdx.x == 0) part[static_cast<int64_t>(blockIdx.y) * gridDim.x + blockIdx.x] = s;
}

__global__ void jtr_chunk_reduce(const double *__restrict__ part, int n, double *__restrict__ Jtr) {
  __shared__ double r[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[static_cast<int64_t>(blockIdx.x) * n + k];
  s = block_sum(s, r);
  if (threadIdx.x == 0) Jtr[blockIdx.x] = s;
}

// Both passes on the context's stream; the partials live in h->d_jtr_part.
template <class T>
int launch_jtr(fs_gpu *h, const T *J, int64_t ld, int64_t M, int D, const double *F, double *Jtr) {
  if (D <= 0) return FS_OK;
  if (D > 65535) return set_error(h, FS_ERR_UNSUPPORTED, "Jacobian-transpose residual: more than 65535 columns");
  const size_t need = static_cast<size_t>(D) * kJtrChunks;
  if (h->jtr_part_alloc < need || !h->d_jtr_part) {
    if (h->d_jtr_part) cudaFree(h->d_jtr_part);
    h->d_jtr_part = nullptr;
    FS_CUDA(cudaMalloc(&h->d_jtr_part, need * sizeof(double)));
    h->jtr_part_alloc = need;
  }
  jtr_chunk_kernel<T><<<dim3(kJtrChunks, D), 256, 0, h->stream>>>(J, ld, M, F, h->d_jtr_part);
  jtr_chunk_reduce<<<D, 128, 0, h->stream>>>(h->d_jtr_part, kJtrChunks, Jtr);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

} // namespace
} // namespace fsg
