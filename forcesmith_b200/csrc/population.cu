// Batched objective evaluation: ‖F(x_k)‖² for a population of parameter
// vectors (the cost of BoostDESolver, src/optimization/solver.cpp:143-146).
#include "internal.cuh"

#include <algorithm>

namespace fsg {

int eval_population(fs_gpu *h, double w_e, double w_s, const double *xs, int NP, double *obj) {
  // Sequential reference schedule: one residual launch per trial vector.
  std::vector<double> x0(h->D);
  FS_TRY(fs_gpu_gather_params(h, x0.data()));
  for (int k = 0; k < NP; ++k) {
    FS_TRY(fs_gpu_set_params(h, xs + static_cast<size_t>(k) * h->D, h->D));
    FS_TRY(refresh_segments(h));
    h->params_dirty = false;
    FS_TRY(eval_residual(h, w_e, w_s));
    FS_CUDA(cudaMemcpyAsync(obj + k, h->d_obj, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  FS_CUDA(cudaStreamSynchronize(h->stream));
  FS_TRY(fs_gpu_set_params(h, x0.data(), h->D));
  return FS_OK;
}

} // namespace fsg
