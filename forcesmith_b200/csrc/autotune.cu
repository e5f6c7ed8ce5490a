// Schedule autotuner: times the launch shapes the kernels can take on the
// context's own configurations and model, with CUDA events on the context's
// stream, and keeps the fastest for later calls.
//   residual          lanes per atom 4, 8, 16, 32
//   Jacobian          warps per CTA of the force-row kernel 11, 10, 8, 6, 4 (FP64:
//                     at most 8; those that fit)
//   population (FP32) CTA waves 2, 4, 8 of the lanes-per-trial kernel
// Every candidate computes the same quantities; only summation order (and
// so the last bits of FP32/FP64 sums) differs between them.
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fsg {
namespace {

template <class F> float time_ms(fs_gpu *h, F &&run, int reps, int *rc) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  *rc = run(); // warm-up (also the first launch of a new template instance)
  cudaEventRecord(a, h->stream);
  for (int k = 0; k < reps && *rc == FS_OK; ++k) *rc = run();
  cudaEventRecord(b, h->stream);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return *rc == FS_OK ? ms / reps : INFINITY;
}

} // namespace
} // namespace fsg

extern "C" int fs_gpu_autotune(fs_gpu *h, double w_e, double w_s, fs_tune_report *rep) {
  using namespace fsg;
  if (!h) return FS_ERR_ARG;
  if (h->n_cfg == 0 || !h->have_model || h->rcut_built < 0)
    return set_error(h, FS_ERR_STATE, "autotune: configurations, model and neighbour lists first");
  cudaSetDevice(h->device);
  fs_tune_report r{};
  // buffers and segments for these weights (a full evaluation)
  FS_TRY(fs_gpu_eval(h, w_e, w_s, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
  const bool ep = h->family == FS_FAMILY_EAM || h->family == FS_FAMILY_PAIR;
  bool splines = true;
  for (const HostTable &t : h->tables) splines = splines && t.kind == FS_TABLE_SPLINE;
  int rc = FS_OK;
  if (ep && !h->lanes_per_atom) {
    static const int lpa[4] = {4, 8, 16, 32};
    int best = 0;
    for (int k = 0; k < 4; ++k) {
      h->tuned_lpa = lpa[k];
      r.residual_ms[k] = time_ms(h, [&] { return eval_residual(h, w_e, w_s); }, 3, &rc);
      FS_TRY(rc);
      if (r.residual_ms[k] < r.residual_ms[best]) best = k;
    }
    h->tuned_lpa = lpa[best];
  }
  r.lanes_per_atom = h->lanes_per_atom ? h->lanes_per_atom : h->tuned_lpa;
  if (ep && splines) {
    static const int k2w[5] = {11, 10, 8, 6, 4};
    const int max_wp = h->precision == FS_PREC_FP64 ? 8 : 11;
    int best = -1;
    for (int k = 0; k < 5; ++k) {
      r.jacobian_ms[k] = INFINITY;
      if (k2w[k] > max_wp) continue;
      h->tuned_k2_warps = k2w[k];
      r.jacobian_ms[k] = time_ms(h, [&] { return eval_jacobian(h, w_e, w_s); }, 2, &rc);
      FS_TRY(rc);
      if (best < 0 || r.jacobian_ms[k] < r.jacobian_ms[best]) best = k;
    }
    h->tuned_k2_warps = k2w[best];
    r.k2_warps = h->tuned_k2_warps;
    h->jac_valid = false;
  }
  if (ep && splines && h->precision == FS_PREC_FP32) {
    // a probe population of 64 vectors around the current parameters
    const int NP = 64, D = h->D;
    std::vector<double> x(D), xs(static_cast<size_t>(NP) * D);
    FS_TRY(fs_gpu_gather_params(h, x.data()));
    for (int k = 0; k < NP; ++k)
      for (int j = 0; j < D; ++j) xs[static_cast<size_t>(k) * D + j] = x[j] * (1.0 + 0.002 * ((k + j) % 9 - 4));
    double *d_xs = nullptr, *d_obj = nullptr;
    FS_CUDA(cudaMallocAsync(&d_xs, xs.size() * sizeof(double), h->stream));
    FS_CUDA(cudaMallocAsync(&d_obj, NP * sizeof(double), h->stream));
    FS_CUDA(cudaMemcpyAsync(d_xs, xs.data(), xs.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    static const int waves[3] = {2, 4, 8};
    int best = 0;
    for (int k = 0; k < 3 && rc == FS_OK; ++k) {
      h->tuned_pop_waves = waves[k];
      r.population_ms[k] = time_ms(h, [&] { return eval_population_device(h, w_e, w_s, d_xs, NP, d_obj); }, 3, &rc);
      if (r.population_ms[k] < r.population_ms[best]) best = k;
    }
    cudaFreeAsync(d_xs, h->stream);
    cudaFreeAsync(d_obj, h->stream);
    FS_TRY(rc);
    h->tuned_pop_waves = waves[best];
    r.pop_waves = h->tuned_pop_waves;
  }
  FS_CUDA(cudaStreamSynchronize(h->stream));
  if (rep) *rep = r;
  return FS_OK;
}
