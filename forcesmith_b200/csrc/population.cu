// Batched objective and differential evolution on the device.
//
// fs_gpu_eval_population: ‖F(x_k)‖² for NP parameter vectors in one pass —
//   per-trial spline segments + one CTA per (configuration, tile of trials),
//   the geometry staged once per CTA (eam.cu: pop_setup_kernel,
//   pop_eval_kernel).  This is the cost BoostDESolver evaluates one vector at
//   a time (src/optimization/solver.cpp:143-146).
//
// fs_gpu_de_*: DE/rand/1/bin with the reference's parameterisation
//   (mutation F, crossover CR, NP, seeded — solver.cpp:113-155): every member
//   i draws distinct r1, r2, r3 ≠ i, mutant v = x_r1 + F (x_r2 − x_r3) clamped
//   to the box, binomial crossover with one forced coordinate, and greedy
//   selection (trial replaces i when its cost is ≤).  One generation = trial
//   kernel → population objective → selection kernel, captured once as a
//   CUDA graph and replayed; the generation counter lives on the device so
//   the random streams advance without host involvement.  The random numbers
//   are a counter-based hash of (seed, generation, member, draw), so runs are
//   reproducible.  The reference's Boost.Math DE trajectory is not pinned
//   (third-party RNG consumption); the objective it minimises is.
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fsg {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double urand(uint64_t seed, uint64_t gen, uint64_t i, uint64_t draw) {
  const uint64_t z = mix64(seed ^ mix64(gen * 0x100000001B3ull ^ mix64(i * 0x9E3779B1ull + draw)));
  return (z >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void de_init_kernel(double *pop, const double *lo, const double *hi, const double *x0, int NP, int D,
                               uint64_t seed) {
  const int i = blockIdx.x;
  for (int j = threadIdx.x; j < D; j += blockDim.x) {
    double v;
    if (i == 0 && x0)
      v = fmin(fmax(x0[j], lo[j]), hi[j]);
    else
      v = __dadd_rn(lo[j], __dmul_rn(__dsub_rn(hi[j], lo[j]), urand(seed, 0xFFFFFFFFull, i, j)));
    pop[static_cast<int64_t>(i) * D + j] = v;
  }
}

// Member i builds its trial vector (one block per member).
__global__ void de_trial_kernel(const double *__restrict__ pop, double *__restrict__ trial,
                                const double *__restrict__ lo, const double *__restrict__ hi, int NP, int D, double F,
                                double CR, uint64_t seed, const int64_t *__restrict__ gen_ctr) {
  const int i = blockIdx.x;
  const uint64_t gen = static_cast<uint64_t>(*gen_ctr);
  __shared__ int r[3], jrand;
  if (threadIdx.x == 0) {
    uint64_t draw = 0;
    for (int q = 0; q < 3; ++q) {
      // up to 64 random draws, then the first free index (NP >= 4 leaves one)
      int c = -1;
      for (int t = 0; t < 64 && c < 0; ++t) {
        int v = static_cast<int>(urand(seed, gen, i, draw++) * NP);
        if (v >= NP) v = NP - 1;
        if (!(v == i || (q > 0 && v == r[0]) || (q > 1 && v == r[1]))) c = v;
      }
      for (int v = 0; v < NP && c < 0; ++v)
        if (!(v == i || (q > 0 && v == r[0]) || (q > 1 && v == r[1]))) c = v;
      r[q] = c;
    }
    jrand = static_cast<int>(urand(seed, gen, i, 1ull << 33) * D);
    if (jrand >= D) jrand = D - 1;
  }
  __syncthreads();
  const double *x1 = pop + static_cast<int64_t>(r[0]) * D, *x2 = pop + static_cast<int64_t>(r[1]) * D,
               *x3 = pop + static_cast<int64_t>(r[2]) * D, *xi = pop + static_cast<int64_t>(i) * D;
  double *t = trial + static_cast<int64_t>(i) * D;
  for (int j = threadIdx.x; j < D; j += blockDim.x) {
    const bool take = j == jrand || urand(seed, gen, i, (1ull << 32) + j) < CR;
    t[j] = take ? fmin(fmax(__dadd_rn(x1[j], __dmul_rn(F, __dsub_rn(x2[j], x3[j]))), lo[j]), hi[j]) : xi[j];
  }
}

// Greedy selection + best tracking; the last block advances the generation.
__global__ void de_select_kernel(double *__restrict__ pop, double *__restrict__ obj, const double *__restrict__ trial,
                                 const double *__restrict__ tobj, int NP, int D, int64_t *__restrict__ gen_ctr,
                                 int *__restrict__ accepted) {
  const int i = blockIdx.x;
  const bool take = tobj[i] <= obj[i];
  if (take)
    for (int j = threadIdx.x; j < D; j += blockDim.x)
      pop[static_cast<int64_t>(i) * D + j] = trial[static_cast<int64_t>(i) * D + j];
  __syncthreads();
  if (threadIdx.x == 0) {
    if (take) {
      obj[i] = tobj[i];
      atomicAdd(accepted, 1);
    }
  }
}

__global__ void de_advance_kernel(int64_t *gen_ctr) { *gen_ctr += 1; }

__global__ void argmin_kernel(const double *__restrict__ v, int n, int *__restrict__ out) {
  __shared__ double bv[1024];
  __shared__ int bi[1024];
  double best = INFINITY;
  int idx = 0;
  for (int k = threadIdx.x; k < n; k += blockDim.x)
    if (v[k] < best || (v[k] == best && k < idx)) {
      best = v[k];
      idx = k;
    }
  bv[threadIdx.x] = best;
  bi[threadIdx.x] = idx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double o = bv[threadIdx.x + s];
      const int oi = bi[threadIdx.x + s];
      if (o < bv[threadIdx.x] || (o == bv[threadIdx.x] && oi < bi[threadIdx.x])) {
        bv[threadIdx.x] = o;
        bi[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = bi[0];
}

} // namespace

// Device buffers of the DE state (owned by the context through DeState).
struct DeState {
  int NP = 0, D = 0;
  double F = 0.65, CR = 0.5, w_e = 1.0, w_s = 0.0;
  uint64_t seed = 42;
  double *pop = nullptr, *obj = nullptr, *trial = nullptr, *tobj = nullptr, *lo = nullptr, *hi = nullptr;
  int64_t *gen = nullptr;
  int *accepted = nullptr, *best = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t generations = 0;
  // device buffers the captured generation reads; a change forces a new capture
  std::vector<const void *> captured;
};

static std::vector<const void *> graph_inputs(const fs_gpu *h) {
  return {h->d_cfg, h->d_wpos, h->d_type, h->d_ref_force, h->d_nb_start, h->d_nb_pack, h->d_desc,
          h->d_cmap,  h->d_vals, h->d_seg_a, h->d_pop_seg_a, h->d_pop_spl};
}

void de_free(DeState *s) {
  if (!s) return;
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  cudaFree(s->pop);
  cudaFree(s->obj);
  cudaFree(s->trial);
  cudaFree(s->tobj);
  cudaFree(s->lo);
  cudaFree(s->hi);
  cudaFree(s->gen);
  cudaFree(s->accepted);
  cudaFree(s->best);
  delete s;
}

int eval_population(fs_gpu *h, double w_e, double w_s, const double *xs, int NP, double *obj) {
  const int D = h->D;
  FS_TRY(refresh_segments(h)); // base model values (fixed knots) current on the device
  h->params_dirty = false;
  const bool batched = (h->family == FS_FAMILY_EAM || h->family == FS_FAMILY_PAIR);
  bool splines = true;
  for (const HostTable &t : h->tables) splines = splines && t.kind == FS_TABLE_SPLINE;
  if (batched && splines) {
    double *d_xs = nullptr, *d_obj = nullptr;
    FS_CUDA(cudaMallocAsync(&d_xs, static_cast<size_t>(NP) * D * sizeof(double), h->stream));
    FS_CUDA(cudaMallocAsync(&d_obj, NP * sizeof(double), h->stream));
    FS_CUDA(cudaMemcpyAsync(d_xs, xs, static_cast<size_t>(NP) * D * sizeof(double), cudaMemcpyHostToDevice,
                            h->stream));
    int rc = eval_population_device(h, w_e, w_s, d_xs, NP, d_obj);
    if (rc == FS_OK)
      FS_CUDA(cudaMemcpyAsync(obj, d_obj, NP * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    cudaFreeAsync(d_xs, h->stream);
    cudaFreeAsync(d_obj, h->stream);
    FS_CUDA(cudaStreamSynchronize(h->stream));
    return rc;
  }
  // other families: one residual launch per trial vector; the normal
  // equations of the current parameters stay valid afterwards
  const bool jac_valid = h->jac_valid;
  std::vector<double> x0(D);
  FS_TRY(fs_gpu_gather_params(h, x0.data()));
  for (int k = 0; k < NP; ++k) {
    FS_TRY(fs_gpu_set_params(h, xs + static_cast<size_t>(k) * D, D));
    FS_TRY(refresh_segments(h));
    h->params_dirty = false;
    FS_TRY(eval_residual(h, w_e, w_s));
    FS_CUDA(cudaMemcpyAsync(obj + k, h->d_obj, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  FS_CUDA(cudaStreamSynchronize(h->stream));
  FS_TRY(fs_gpu_set_params(h, x0.data(), D));
  h->jac_valid = jac_valid;
  return FS_OK;
}

int de_init(fs_gpu *h, const fs_de_opts *o, const double *lo, const double *hi, const double *x0) {
  if (h->de) de_free(h->de);
  h->de = nullptr;
  DeState *s = new DeState();
  s->NP = o->NP;
  s->D = h->D;
  s->F = o->mutation;
  s->CR = o->crossover;
  s->seed = o->seed;
  s->w_e = o->w_e;
  s->w_s = o->w_s;
  const size_t pd = static_cast<size_t>(s->NP) * s->D;
  if (cudaMalloc(&s->pop, pd * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&s->trial, pd * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&s->obj, s->NP * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&s->tobj, s->NP * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&s->lo, s->D * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&s->hi, s->D * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&s->gen, sizeof(int64_t)) != cudaSuccess || cudaMalloc(&s->accepted, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&s->best, sizeof(int)) != cudaSuccess) {
    de_free(s);
    return set_error(h, FS_ERR_NOMEM, "de_init: cudaMalloc");
  }
  h->de = s;
  double *d_x0 = nullptr;
  FS_CUDA(cudaMemcpyAsync(s->lo, lo, s->D * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  FS_CUDA(cudaMemcpyAsync(s->hi, hi, s->D * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (x0) {
    FS_CUDA(cudaMallocAsync(&d_x0, s->D * sizeof(double), h->stream));
    FS_CUDA(cudaMemcpyAsync(d_x0, x0, s->D * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  FS_CUDA(cudaMemsetAsync(s->gen, 0, sizeof(int64_t), h->stream));
  FS_CUDA(cudaMemsetAsync(s->accepted, 0, sizeof(int), h->stream));
  de_init_kernel<<<s->NP, 128, 0, h->stream>>>(s->pop, s->lo, s->hi, d_x0, s->NP, s->D, s->seed);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  if (d_x0) cudaFreeAsync(d_x0, h->stream);
  FS_TRY(refresh_segments(h));
  h->params_dirty = false;
  FS_TRY(eval_population_device(h, s->w_e, s->w_s, s->pop, s->NP, s->obj));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  return FS_OK;
}

static int de_generation(fs_gpu *h, DeState *s) {
  de_trial_kernel<<<s->NP, 128, 0, h->stream>>>(s->pop, s->trial, s->lo, s->hi, s->NP, s->D, s->F, s->CR, s->seed,
                                                 s->gen);
  FS_CUDA(cudaGetLastError());
  FS_TRY(eval_population_device(h, s->w_e, s->w_s, s->trial, s->NP, s->tobj));
  de_select_kernel<<<s->NP, 128, 0, h->stream>>>(s->pop, s->obj, s->trial, s->tobj, s->NP, s->D, s->gen, s->accepted);
  FS_CUDA(cudaGetLastError());
  de_advance_kernel<<<1, 1, 0, h->stream>>>(s->gen);
  FS_CUDA(cudaGetLastError());
  h->launches += 3;
  return FS_OK;
}

int de_run(fs_gpu *h, int generations, int use_graph, double *best_obj, double *best_x, double *history) {
  DeState *s = h->de;
  if (!s) return set_error(h, FS_ERR_STATE, "de_run: fs_gpu_de_init first");
  if (use_graph && s->exec && s->captured != graph_inputs(h)) {
    cudaGraphExecDestroy(s->exec);
    cudaGraphDestroy(s->graph);
    s->exec = nullptr;
    s->graph = nullptr;
  }
  if (use_graph && !s->exec) {
    // capture one generation (trial → population objective → selection)
    FS_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int64_t l0 = h->launches;
    const int rc = de_generation(h, s);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->launches = l0;
    if (rc != FS_OK) return rc;
    if (e != cudaSuccess) return set_error(h, FS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    s->graph = g;
    FS_CUDA(cudaGraphInstantiate(&s->exec, g, 0));
    s->captured = graph_inputs(h);
  }
  int64_t per_gen = 0;
  if (use_graph) {
    size_t nn = 0;
    cudaGraphGetNodes(s->graph, nullptr, &nn);
    per_gen = static_cast<int64_t>(nn);
  }
  for (int g = 0; g < generations; ++g) {
    if (use_graph) {
      FS_CUDA(cudaGraphLaunch(s->exec, h->stream));
      h->launches += per_gen;
    } else {
      FS_TRY(de_generation(h, s));
    }
    if (history) {
      argmin_kernel<<<1, 1024, 0, h->stream>>>(s->obj, s->NP, s->best);
      int b = 0;
      FS_CUDA(cudaMemcpyAsync(&b, s->best, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      FS_CUDA(cudaStreamSynchronize(h->stream));
      FS_CUDA(cudaMemcpy(&history[g], s->obj + b, sizeof(double), cudaMemcpyDeviceToHost));
    }
  }
  s->generations += generations;
  argmin_kernel<<<1, 1024, 0, h->stream>>>(s->obj, s->NP, s->best);
  FS_CUDA(cudaGetLastError());
  int b = 0;
  FS_CUDA(cudaMemcpyAsync(&b, s->best, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  if (best_obj) FS_CUDA(cudaMemcpy(best_obj, s->obj + b, sizeof(double), cudaMemcpyDeviceToHost));
  if (best_x)
    FS_CUDA(cudaMemcpy(best_x, s->pop + static_cast<int64_t>(b) * s->D, s->D * sizeof(double), cudaMemcpyDeviceToHost));
  return FS_OK;
}

int de_population(fs_gpu *h, double *pop, double *obj) {
  DeState *s = h->de;
  if (!s) return set_error(h, FS_ERR_STATE, "de_population: fs_gpu_de_init first");
  if (pop)
    FS_CUDA(cudaMemcpyAsync(pop, s->pop, static_cast<size_t>(s->NP) * s->D * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream));
  if (obj) FS_CUDA(cudaMemcpyAsync(obj, s->obj, s->NP * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  return FS_OK;
}

} // namespace fsg

extern "C" {

int fs_gpu_de_init(fs_gpu *h, const fs_de_opts *opts, const double *lo, const double *hi, const double *x0) {
  if (!h || !opts || !lo || !hi) return FS_ERR_ARG;
  if (!h->have_model || h->rcut_built < 0) return fsg::set_error(h, FS_ERR_STATE, "de_init: model not prepared");
  if (opts->NP < 4 || !(opts->mutation > 0.0) || !(opts->crossover >= 0.0 && opts->crossover <= 1.0))
    return fsg::set_error(h, FS_ERR_ARG, "de_init: NP >= 4, F > 0, 0 <= CR <= 1");
  for (int j = 0; j < h->D; ++j)
    if (!(std::isfinite(lo[j]) && std::isfinite(hi[j]) && lo[j] <= hi[j]))
      return fsg::set_error(h, FS_ERR_ARG, "de_init: finite bounds lo <= hi required");
  cudaSetDevice(h->device);
  return fsg::de_init(h, opts, lo, hi, x0);
}

int fs_gpu_de_run(fs_gpu *h, int32_t generations, int32_t use_graph, double *best_obj, double *best_x,
                  double *history) {
  if (!h || generations < 0) return FS_ERR_ARG;
  cudaSetDevice(h->device);
  return fsg::de_run(h, generations, use_graph, best_obj, best_x, history);
}

int fs_gpu_de_population(fs_gpu *h, double *pop, double *obj) {
  if (!h) return FS_ERR_ARG;
  cudaSetDevice(h->device);
  return fsg::de_population(h, pop, obj);
}

} // extern "C"
