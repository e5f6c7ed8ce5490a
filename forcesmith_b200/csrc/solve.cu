// FP64 damped normal-equation solve on the device:
//   (JᵀJ + λ·diag) dx = −Jᵀr
// by a right-looking Cholesky factorisation in one CTA (the LM / lsq step
// consumers of EigenLMSolver and NormalEquationsSolver,
// src/optimization/solver.cpp:67-85,242-266; the reference factorises with
// MINPACK QR and LDLT respectively, this build with Cholesky).
#include "internal.cuh"

#include <algorithm>

namespace fsg {
namespace {

__global__ void __launch_bounds__(1024) chol_solve_kernel(const double *__restrict__ JtJ, const double *__restrict__ Jtr,
                                                          int D, double lambda, int mode, double *__restrict__ A,
                                                          double *__restrict__ x, int32_t *__restrict__ flag) {
  __shared__ double piv;
  __shared__ int bad;
  const int tid = threadIdx.x, nth = blockDim.x;
  if (tid == 0) bad = 0;
  for (int k = tid; k < D * D; k += nth) {
    const int i = k / D, j = k % D;
    double v = JtJ[k];
    if (i == j) v += lambda * (mode == 1 ? (JtJ[k] > 0.0 ? JtJ[k] : 1.0) : 1.0); // zero column → 1
    A[k] = v;
  }
  __syncthreads();
  for (int j = 0; j < D; ++j) {
    if (tid == 0) {
      const double d = A[j * D + j];
      if (!(d > 0.0) || !isfinite(d)) bad = 1;
      piv = bad ? 1.0 : sqrt(d);
      A[j * D + j] = piv;
    }
    __syncthreads();
    for (int i = j + 1 + tid; i < D; i += nth) A[i * D + j] /= piv;
    __syncthreads();
    const int rem = D - j - 1;
    for (int k = tid; k < rem * rem; k += nth) {
      const int i = j + 1 + k / rem, c = j + 1 + k % rem;
      if (c <= i) A[i * D + c] -= A[i * D + j] * A[c * D + j];
    }
    __syncthreads();
  }
  // forward L y = −Jᵀr, backward Lᵀ x = y (one warp, lane-parallel dots)
  if (tid < 32) {
    for (int i = 0; i < D; ++i) {
      double s = 0.0;
      for (int k = tid; k < i; k += 32) s += A[i * D + k] * x[k];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (tid == 0) x[i] = (-Jtr[i] - s) / A[i * D + i];
      __syncwarp();
    }
    for (int i = D - 1; i >= 0; --i) {
      double s = 0.0;
      for (int k = i + 1 + tid; k < D; k += 32) s += A[k * D + i] * x[k];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (tid == 0) x[i] = (x[i] - s) / A[i * D + i];
      __syncwarp();
    }
  }
  if (tid == 0) *flag = bad;
}

} // namespace

int lm_solve(fs_gpu *h, double lambda, int mode, double *dx_host) {
  const int D = h->D;
  if (!h->d_chol || h->chol_D != D) {
    if (h->d_chol) cudaFree(h->d_chol);
    if (h->d_dx) cudaFree(h->d_dx);
    if (h->d_flag) cudaFree(h->d_flag);
    h->chol_D = D;
    FS_CUDA(cudaMalloc(&h->d_chol, static_cast<size_t>(std::max(D, 1)) * std::max(D, 1) * sizeof(double)));
    FS_CUDA(cudaMalloc(&h->d_dx, std::max(D, 1) * sizeof(double)));
    FS_CUDA(cudaMalloc(&h->d_flag, sizeof(int32_t)));
  }
  chol_solve_kernel<<<1, 1024, 0, h->stream>>>(h->d_JtJ, h->d_Jtr, D, lambda, mode, h->d_chol, h->d_dx, h->d_flag);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  int32_t flag = 0;
  FS_CUDA(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaMemcpyAsync(dx_host, h->d_dx, D * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  if (flag) return set_error(h, FS_ERR_NUMERIC, "lm_step: matrix not positive definite");
  return FS_OK;
}

} // namespace fsg
