// Central-difference Jacobian on the device — the reference's own method
// (opt::fd_jacobian, include/forcesmith/optimization/fd_jacobian.hpp:37-49:
// h = 1e-5, x restored by the same add/subtract sequence), used for families
// without an analytic device Jacobian in this build (ADP, Tersoff, Angular).
// 2·D residual launches; FP64 contexts only (FP32 residuals are too coarse for
// h = 1e-5).
#include "internal.cuh"
#include "jtr.cuh"

#include <vector>

namespace fsg {
namespace {

__global__ void fd_column(const double *__restrict__ Fp, const double *__restrict__ Fm, int64_t M, double inv2h,
                          double *__restrict__ col) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < M;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    col[r] = (Fp[r] - Fm[r]) * inv2h;
}

} // namespace

int eval_jacobian_fd(fs_gpu *h, double w_e, double w_s) {
  if (h->precision != FS_PREC_FP64)
    return set_error(h, FS_ERR_UNSUPPORTED, "central-difference Jacobian needs an FP64 context");
  const int D = h->D;
  const int64_t M = rows_of(h, w_s);
  const int64_t ldj = (M + 31) / 32 * 32;
  const size_t jn = static_cast<size_t>(ldj) * D;
  if (static_cast<size_t>(h->jac_alloc) != jn || h->ldj != ldj || !h->d_J || h->j_rowmajor) {
    if (h->d_J) cudaFree(h->d_J);
    h->d_J = nullptr;
    FS_CUDA(cudaMalloc(&h->d_J, std::max<size_t>(jn, 1) * sizeof(double)));
    FS_CUDA(cudaMemsetAsync(h->d_J, 0, std::max<size_t>(jn, 1) * sizeof(double), h->stream));
    h->jac_alloc = static_cast<int64_t>(jn);
    h->ldj = ldj;
    h->j_rowmajor = false;
  }
  if (!h->d_JtJ) {
    FS_CUDA(cudaMalloc(&h->d_JtJ, std::max(D * D, 1) * sizeof(double)));
    FS_CUDA(cudaMalloc(&h->d_Jtr, std::max(D, 1) * sizeof(double)));
  }
  // the base residual and F(x + h e_j): scratch kept with the context
  if (h->fd_scratch_alloc < static_cast<size_t>(2 * M) || !h->d_fd_scratch) {
    if (h->d_fd_scratch) cudaFree(h->d_fd_scratch);
    h->d_fd_scratch = nullptr;
    FS_CUDA(cudaMalloc(&h->d_fd_scratch, 2 * M * sizeof(double)));
    h->fd_scratch_alloc = static_cast<size_t>(2 * M);
  }
  double *Fbase = h->d_fd_scratch, *Fp = h->d_fd_scratch + M;
  FS_CUDA(cudaMemcpyAsync(Fbase, h->d_F, M * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  std::vector<double> x(D), xp;
  FS_TRY(fs_gpu_gather_params(h, x.data()));
  xp = x;
  const double hh = 1e-5;
  int rc = FS_OK;
  for (int j = 0; j < D && rc == FS_OK; ++j) {
    xp[j] += hh;
    rc = fs_gpu_set_params(h, xp.data(), D);
    if (rc == FS_OK) rc = refresh_segments(h);
    if (rc == FS_OK) rc = eval_residual(h, w_e, w_s);
    if (rc != FS_OK) break;
    FS_CUDA(cudaMemcpyAsync(Fp, h->d_F, M * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    xp[j] -= 2.0 * hh;
    rc = fs_gpu_set_params(h, xp.data(), D);
    if (rc == FS_OK) rc = refresh_segments(h);
    if (rc == FS_OK) rc = eval_residual(h, w_e, w_s);
    if (rc != FS_OK) break;
    xp[j] += hh;
    fd_column<<<256, 256, 0, h->stream>>>(Fp, h->d_F, M, 1.0 / (2.0 * hh),
                                          static_cast<double *>(h->d_J) + static_cast<int64_t>(j) * ldj);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  const int rc2 = fs_gpu_set_params(h, x.data(), D);
  if (rc == FS_OK) rc = rc2;
  if (rc == FS_OK) rc = refresh_segments(h);
  h->params_dirty = false;
  FS_CUDA(cudaMemcpyAsync(h->d_F, Fbase, M * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  if (rc == FS_OK) rc = launch_jtr<double>(h, static_cast<const double *>(h->d_J), ldj, M, D, h->d_F, h->d_Jtr);
  return rc;
}

} // namespace fsg
