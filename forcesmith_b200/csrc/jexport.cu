// Jacobian export: a row block of the device Jacobian, as FP64 column-major,
// into host memory.
//
// The reference's solvers take J as Eigen's column-major FP64 `fjac`
// (values × inputs, include/forcesmith/optimization/solver.hpp:14-15), and a
// cached-Jacobian calculator writes its configuration's row block of it
// (ForceCalculator::eval_cached_jacobian, force_calculator.hpp:62-159, called
// per configuration from df_cached_analytic, forcesmith_functor.cpp:111-132).
// The device keeps J in its working precision: FP32 row-major for the EAM /
// pair Jacobians that feed the tensor-core JᵀJ, column-major otherwise.  The
// widening to FP64 and the transpose run on the device, into a staging
// buffer laid out exactly as the destination block, so the host sees one
// strided DMA per call.
#include "internal.cuh"

using namespace fsg;

namespace fsg {
namespace {

// Row-major source (rows × ld, row stride ld ≥ D): 32 × 32 tiles through
// shared memory so that both the read (along a row) and the write (along a
// column) are coalesced.  Block (32, 8).
template <class T>
__global__ void __launch_bounds__(256) export_rowmajor_kernel(const T *__restrict__ J, int64_t ld, int64_t row0,
                                                              int64_t nrows, int D, double *__restrict__ out) {
  __shared__ double tile[32][33];
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int64_t r = r0 + k;
    const int c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < nrows && c < D) ? static_cast<double>(J[(row0 + r) * ld + c]) : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int c = c0 + k;
    const int64_t r = r0 + threadIdx.x;
    if (c < D && r < nrows) out[static_cast<int64_t>(c) * nrows + r] = tile[threadIdx.x][k];
  }
}

// Column-major FP32 source (leading dimension ld): element-wise widening.
__global__ void __launch_bounds__(256) export_colmajor_kernel(const float *__restrict__ J, int64_t ld, int64_t row0,
                                                              int64_t nrows, int D, double *__restrict__ out) {
  const int64_t n = nrows * D;
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = q / nrows, r = q - c * nrows;
    out[q] = static_cast<double>(J[c * ld + row0 + r]);
  }
}

} // namespace
} // namespace fsg

extern "C" int fs_gpu_copy_jacobian_rows(fs_gpu *h, int64_t row0, int64_t nrows, double *J, int64_t ldJ) {
  if (!h) return FS_ERR_ARG;
  if (!h->jac_valid || !h->d_J) return set_error(h, FS_ERR_STATE, "copy_jacobian_rows: no Jacobian evaluated");
  const int64_t m = rows_of(h, h->last_ws);
  if (row0 < 0 || nrows < 0 || row0 + nrows > m)
    return set_error(h, FS_ERR_ARG, "copy_jacobian_rows: rows [" + std::to_string(row0) + ", " +
                                        std::to_string(row0 + nrows) + ") outside the " + std::to_string(m) +
                                        " residual rows");
  if (nrows == 0) return FS_OK;
  if (!J || ldJ < nrows) return set_error(h, FS_ERR_ARG, "copy_jacobian_rows: null J or ldJ < nrows");
  cudaSetDevice(h->device);
  const int D = h->D;
  if (h->precision == FS_PREC_FP64 && !h->j_rowmajor) {
    // already FP64 column-major: one strided DMA
    FS_CUDA(cudaMemcpy2DAsync(J, ldJ * sizeof(double), static_cast<const double *>(h->d_J) + row0,
                              h->ldj * sizeof(double), nrows * sizeof(double), D, cudaMemcpyDeviceToHost,
                              h->stream));
    return sync_checked(h);
  }
  const size_t need = static_cast<size_t>(nrows) * D;
  if (need > h->jx_alloc) {
    if (h->d_jx) cudaFree(h->d_jx);
    h->d_jx = nullptr;
    h->jx_alloc = 0;
    if (cudaMalloc(&h->d_jx, need * sizeof(double)) != cudaSuccess)
      return set_error(h, FS_ERR_NOMEM, "copy_jacobian_rows: staging buffer of " +
                                            std::to_string(need * sizeof(double)) + " bytes");
    h->jx_alloc = need;
  }
  if (h->j_rowmajor) {
    const dim3 grid(static_cast<unsigned>((nrows + 31) / 32), static_cast<unsigned>((D + 31) / 32));
    if (h->precision == FS_PREC_FP64)
      export_rowmajor_kernel<double><<<grid, dim3(32, 8), 0, h->stream>>>(static_cast<const double *>(h->d_J),
                                                                          h->ldj, row0, nrows, D, h->d_jx);
    else
      export_rowmajor_kernel<float><<<grid, dim3(32, 8), 0, h->stream>>>(static_cast<const float *>(h->d_J),
                                                                         h->ldj, row0, nrows, D, h->d_jx);
  } else {
    export_colmajor_kernel<<<4 * 148, 256, 0, h->stream>>>(static_cast<const float *>(h->d_J), h->ldj, row0, nrows,
                                                           D, h->d_jx);
  }
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  FS_CUDA(cudaMemcpy2DAsync(J, ldJ * sizeof(double), h->d_jx, nrows * sizeof(double), nrows * sizeof(double), D,
                            cudaMemcpyDeviceToHost, h->stream));
  return sync_checked(h);
}
