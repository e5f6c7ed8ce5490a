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

// Member i builds candidate k of its trial vector (block (i, k)); candidate
// k draws from the random stream of member i + k·2³², so k = 0 is the plain
// DE trial.  Optionally writes the candidate's model features
// 2(x − lo)/(hi − lo) − 1 in FP32.
__global__ void de_trial_kernel(const double *__restrict__ pop, double *__restrict__ trial,
                                float *__restrict__ feat, const double *__restrict__ lo,
                                const double *__restrict__ hi, int NP, int D, double F, double CR, uint64_t seed,
                                const int64_t *__restrict__ gen_ctr) {
  const int i = blockIdx.x;
  const uint64_t stream = static_cast<uint64_t>(i) + (static_cast<uint64_t>(blockIdx.y) << 32);
  const uint64_t gen = static_cast<uint64_t>(*gen_ctr);
  __shared__ int r[3], jrand;
  if (threadIdx.x == 0) {
    uint64_t draw = 0;
    for (int q = 0; q < 3; ++q) {
      // up to 64 random draws, then the first free index (NP >= 4 leaves one)
      int c = -1;
      for (int t = 0; t < 64 && c < 0; ++t) {
        int v = static_cast<int>(urand(seed, gen, stream, draw++) * NP);
        if (v >= NP) v = NP - 1;
        if (!(v == i || (q > 0 && v == r[0]) || (q > 1 && v == r[1]))) c = v;
      }
      for (int v = 0; v < NP && c < 0; ++v)
        if (!(v == i || (q > 0 && v == r[0]) || (q > 1 && v == r[1]))) c = v;
      r[q] = c;
    }
    jrand = static_cast<int>(urand(seed, gen, stream, 1ull << 33) * D);
    if (jrand >= D) jrand = D - 1;
  }
  __syncthreads();
  const double *x1 = pop + static_cast<int64_t>(r[0]) * D, *x2 = pop + static_cast<int64_t>(r[1]) * D,
               *x3 = pop + static_cast<int64_t>(r[2]) * D, *xi = pop + static_cast<int64_t>(i) * D;
  const int64_t row = static_cast<int64_t>(blockIdx.y) * NP + i;
  double *t = trial + row * D;
  for (int j = threadIdx.x; j < D; j += blockDim.x) {
    const bool take = j == jrand || urand(seed, gen, stream, (1ull << 32) + j) < CR;
    const double v =
        take ? fmin(fmax(__dadd_rn(x1[j], __dmul_rn(F, __dsub_rn(x2[j], x3[j]))), lo[j]), hi[j]) : xi[j];
    t[j] = v;
    if (feat) feat[row * D + j] = hi[j] > lo[j] ? static_cast<float>(2.0 * (v - lo[j]) / (hi[j] - lo[j]) - 1.0) : 0.f;
  }
}

// Per member: the candidate with the lowest predicted value (NaN last) is
// copied to the trial buffer and its features to the archive row.
__global__ void de_pick_kernel(const double *__restrict__ cand, const float *__restrict__ cfeat,
                               const float *__restrict__ y, int NP, int S, int D, double *__restrict__ trial,
                               float *__restrict__ feat_out) {
  const int i = blockIdx.x;
  __shared__ int best;
  if (threadIdx.x == 0) {
    int b = 0;
    float bv = INFINITY;
    for (int k = 0; k < S; ++k) {
      const float v = y[static_cast<int64_t>(k) * NP + i];
      if (v < bv) {
        bv = v;
        b = k;
      }
    }
    best = b;
  }
  __syncthreads();
  const int64_t src = static_cast<int64_t>(best) * NP + i;
  for (int j = threadIdx.x; j < D; j += blockDim.x) {
    trial[static_cast<int64_t>(i) * D + j] = cand[src * D + j];
    feat_out[static_cast<int64_t>(i) * D + j] = cfeat[src * D + j];
  }
}

// archive targets: log of the exact objective
__global__ void arch_target_kernel(const double *__restrict__ tobj, int NP, float *__restrict__ t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NP) t[i] = static_cast<float>(log(fmax(tobj[i], 1e-300)));
}

// Training batch: uniform rows of the archive outside the held-out slice
// (every P-th row, index ≡ P−1 mod P), targets standardised.
__global__ void arch_batch_kernel(const float *__restrict__ ax, const float *__restrict__ at, int64_t n, int P, int D,
                                  int rows, uint64_t seed, uint64_t ctr, float mu, float inv_sigma,
                                  float *__restrict__ xs, float *__restrict__ t) {
  const int r = blockIdx.x;
  __shared__ int64_t idx;
  if (threadIdx.x == 0) {
    int64_t k = static_cast<int64_t>(urand(seed, ctr, static_cast<uint64_t>(r), 7) * static_cast<double>(n));
    if (k >= n) k = n - 1;
    if (P > 1 && k % P == P - 1) k -= 1;
    idx = k;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < D; j += blockDim.x) xs[static_cast<int64_t>(r) * D + j] = ax[idx * D + j];
  if (threadIdx.x == 0) t[r] = (at[idx] - mu) * inv_sigma;
}

// The most recent `rows` held-out archive rows.
__global__ void arch_holdout_kernel(const float *__restrict__ ax, const float *__restrict__ at, int64_t n_held, int P,
                                    int D, float *__restrict__ xs, float *__restrict__ t) {
  const int r = blockIdx.x;
  const int64_t idx = (n_held - 1 - r) * P + (P - 1);
  for (int j = threadIdx.x; j < D; j += blockDim.x) xs[static_cast<int64_t>(r) * D + j] = ax[idx * D + j];
  if (threadIdx.x == 0) t[r] = at[idx];
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

// Index of the smallest of v[0..n) (lowest index on ties) into *out, and,
// when rec is not null, that value into *rec.
__global__ void argmin_kernel(const double *__restrict__ v, int n, int *__restrict__ out,
                              double *__restrict__ rec = nullptr) {
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
  if (threadIdx.x == 0) {
    *out = bi[0];
    if (rec) *rec = bv[0];
  }
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
  double *hist = nullptr; // best objective after each generation of a de_run call
  int hist_n = 0;
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
  cudaFree(s->hist);
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
  de_trial_kernel<<<s->NP, 128, 0, h->stream>>>(s->pop, s->trial, nullptr, s->lo, s->hi, s->NP, s->D, s->F, s->CR,
                                                 s->seed, s->gen);
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
  if (history && generations > s->hist_n) {
    cudaFree(s->hist);
    s->hist = nullptr;
    s->hist_n = 0;
    FS_CUDA(cudaMalloc(&s->hist, generations * sizeof(double)));
    s->hist_n = generations;
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
    if (history) { // the generation's best into a device slot: no host wait per generation
      argmin_kernel<<<1, 1024, 0, h->stream>>>(s->obj, s->NP, s->best, s->hist + g);
      FS_CUDA(cudaGetLastError());
      ++h->launches;
    }
  }
  if (history && generations > 0)
    FS_CUDA(cudaMemcpyAsync(history, s->hist, generations * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
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

// ---------------------------------------------------------------------------
// surrogate-screened DE

struct Surrogate {
  fs_surrogate_opts o{};
  int D = 0;
  int P = 10;                     // held-out period: every P-th archive row
  float *ax = nullptr, *at = nullptr;
  int64_t cap = 0, n = 0;         // archive rows (FP32 features, log objective)
  double *cand = nullptr;         // S·NP candidate vectors
  int64_t cand_cap = 0;
  float mu = 0.f, inv_sigma = 1.f;
  int64_t generations = 0;
  bool gate_open = false;
  double last_rho = 0.0;
  uint64_t ctr = 0;
};

void surrogate_free(Surrogate *s) {
  if (!s) return;
  cudaFree(s->ax);
  cudaFree(s->at);
  cudaFree(s->cand);
  delete s;
}

// Spearman rank correlation (average ranks for ties).
static double spearman(const std::vector<float> &a, const std::vector<float> &b) {
  const size_t n = a.size();
  if (n < 3) return 0.0;
  auto ranks = [n](const std::vector<float> &v) {
    std::vector<int> ix(n);
    for (size_t k = 0; k < n; ++k) ix[k] = static_cast<int>(k);
    std::sort(ix.begin(), ix.end(), [&](int p, int q) { return v[p] < v[q]; });
    std::vector<double> r(n);
    for (size_t k = 0; k < n;) {
      size_t e = k;
      while (e + 1 < n && v[ix[e + 1]] == v[ix[k]]) ++e;
      const double avg = 0.5 * static_cast<double>(k + e);
      for (size_t q = k; q <= e; ++q) r[ix[q]] = avg;
      k = e + 1;
    }
    return r;
  };
  const std::vector<double> ra = ranks(a), rb = ranks(b);
  double ma = 0, mb = 0;
  for (size_t k = 0; k < n; ++k) {
    ma += ra[k];
    mb += rb[k];
  }
  ma /= n;
  mb /= n;
  double sab = 0, saa = 0, sbb = 0;
  for (size_t k = 0; k < n; ++k) {
    sab += (ra[k] - ma) * (rb[k] - mb);
    saa += (ra[k] - ma) * (ra[k] - ma);
    sbb += (rb[k] - mb) * (rb[k] - mb);
  }
  return (saa > 0 && sbb > 0) ? sab / std::sqrt(saa * sbb) : 0.0;
}

static int surrogate_train(fs_gpu *h, Surrogate *sv, int steps) {
  const int B = sv->o.batch;
  FS_TRY(mlp_reserve(h, h->mlp, B));
  for (int k = 0; k < steps; ++k) {
    arch_batch_kernel<<<B, 64, 0, h->stream>>>(sv->ax, sv->at, sv->n, sv->P, sv->D, B, sv->o.seed ^ 0x5EEDull,
                                               sv->ctr++, sv->mu, sv->inv_sigma, mlp_rows_x(h->mlp),
                                               mlp_rows_t(h->mlp));
    FS_CUDA(cudaGetLastError());
    ++h->launches;
    FS_TRY(mlp_gradient_dev(h, h->mlp, B));
    FS_TRY(mlp_adam_dev(h, h->mlp));
  }
  return FS_OK;
}

// Rank correlation of the model on the newest held-out rows (≤ 2048).
static int surrogate_gate(fs_gpu *h, Surrogate *sv, double *rho) {
  const int64_t n_held = sv->P > 1 ? sv->n / sv->P : 0;
  const int rows = static_cast<int>(std::min<int64_t>(n_held, 2048));
  *rho = 0.0;
  if (rows < 8) return FS_OK;
  FS_TRY(mlp_reserve(h, h->mlp, rows));
  arch_holdout_kernel<<<rows, 64, 0, h->stream>>>(sv->ax, sv->at, n_held, sv->P, sv->D, mlp_rows_x(h->mlp),
                                                   mlp_rows_t(h->mlp));
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  FS_TRY(mlp_forward_dev(h, h->mlp, rows));
  std::vector<float> y(rows), t(rows);
  FS_CUDA(cudaMemcpyAsync(y.data(), mlp_rows_y(h->mlp), rows * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaMemcpyAsync(t.data(), mlp_rows_t(h->mlp), rows * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  *rho = spearman(y, t);
  return FS_OK;
}

int de_run_screened(fs_gpu *h, int generations, double *best_obj, double *best_x, double *history, double *rho_out,
                    int32_t *screened_out) {
  DeState *s = h->de;
  Surrogate *sv = h->sur;
  if (!s || !sv || !h->mlp) return set_error(h, FS_ERR_STATE, "de_run_screened: fs_gpu_de_init and fs_gpu_surrogate_init first");
  if (sv->D != s->D) return set_error(h, FS_ERR_STATE, "de_run_screened: surrogate and DE sizes differ");
  const int NP = s->NP, D = s->D, S = std::max(1, sv->o.screen);
  if (sv->o.archive_rows > 0 && sv->o.archive_rows < 2 * static_cast<int64_t>(NP))
    return set_error(h, FS_ERR_ARG, "de_run_screened: archive_rows must hold at least two generations (2 NP)");
  // archive: grows in whole generations (ring once the capacity is reached)
  const int64_t want = sv->n + static_cast<int64_t>(generations) * NP;
  if (want > sv->cap) {
    // grow geometrically so that runs made of many short calls copy little
    const int64_t grown = std::max<int64_t>(std::max<int64_t>(want, 2 * sv->cap), 16 * NP);
    const int64_t cap = sv->o.archive_rows > 0 ? std::min<int64_t>(grown, sv->o.archive_rows) : grown;
    float *ax = nullptr, *at = nullptr;
    if (cudaMalloc(&ax, cap * D * sizeof(float)) != cudaSuccess || cudaMalloc(&at, cap * sizeof(float)) != cudaSuccess) {
      cudaFree(ax);
      return set_error(h, FS_ERR_NOMEM, "de_run_screened: archive");
    }
    const int64_t keep = std::min(sv->n, cap);
    if (keep > 0) {
      FS_CUDA(cudaMemcpyAsync(ax, sv->ax, keep * D * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
      FS_CUDA(cudaMemcpyAsync(at, sv->at, keep * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    }
    FS_CUDA(cudaStreamSynchronize(h->stream));
    cudaFree(sv->ax);
    cudaFree(sv->at);
    sv->ax = ax;
    sv->at = at;
    sv->cap = cap;
    sv->n = keep;
  }
  if (sv->cand_cap < static_cast<int64_t>(S) * NP) {
    cudaFree(sv->cand);
    sv->cand = nullptr;
    FS_CUDA(cudaMalloc(&sv->cand, static_cast<size_t>(S) * NP * D * sizeof(double)));
    sv->cand_cap = static_cast<int64_t>(S) * NP;
  }
  FS_TRY(mlp_reserve(h, h->mlp, std::max(S * NP, sv->o.batch)));
  for (int g = 0; g < generations; ++g) {
    if (sv->n + NP > sv->cap) sv->n = 0; // ring: start over at the front
    float *frow = sv->ax + sv->n * D;
    const bool screen = sv->generations >= sv->o.warm_generations && sv->gate_open && S > 1;
    if (screen) {
      de_trial_kernel<<<dim3(NP, S), 128, 0, h->stream>>>(s->pop, sv->cand, mlp_rows_x(h->mlp), s->lo, s->hi, NP, D,
                                                           s->F, s->CR, s->seed, s->gen);
      FS_CUDA(cudaGetLastError());
      FS_TRY(mlp_forward_dev(h, h->mlp, S * NP));
      de_pick_kernel<<<NP, 128, 0, h->stream>>>(sv->cand, mlp_rows_x(h->mlp), mlp_rows_y(h->mlp), NP, S, D, s->trial,
                                                frow);
      FS_CUDA(cudaGetLastError());
      h->launches += 2;
    } else {
      de_trial_kernel<<<NP, 128, 0, h->stream>>>(s->pop, s->trial, frow, s->lo, s->hi, NP, D, s->F, s->CR, s->seed,
                                                 s->gen);
      FS_CUDA(cudaGetLastError());
      ++h->launches;
    }
    FS_TRY(eval_population_device(h, s->w_e, s->w_s, s->trial, NP, s->tobj));
    arch_target_kernel<<<(NP + 255) / 256, 256, 0, h->stream>>>(s->tobj, NP, sv->at + sv->n);
    de_select_kernel<<<NP, 128, 0, h->stream>>>(s->pop, s->obj, s->trial, s->tobj, NP, D, s->gen, s->accepted);
    de_advance_kernel<<<1, 1, 0, h->stream>>>(s->gen);
    FS_CUDA(cudaGetLastError());
    h->launches += 3;
    sv->n += NP;
    sv->generations += 1;
    s->generations += 1;
    if (sv->generations == sv->o.warm_generations) {
      // fix the target standardisation from the warm-start archive
      std::vector<float> t(sv->n);
      FS_CUDA(cudaMemcpyAsync(t.data(), sv->at, sv->n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
      FS_CUDA(cudaStreamSynchronize(h->stream));
      double m = 0, q = 0;
      for (float v : t) m += v;
      m /= std::max<size_t>(t.size(), 1);
      for (float v : t) q += (v - m) * (v - m);
      const double sd = std::sqrt(q / std::max<size_t>(t.size(), 1));
      sv->mu = static_cast<float>(m);
      sv->inv_sigma = static_cast<float>(sd > 0 ? 1.0 / sd : 1.0);
      FS_TRY(surrogate_train(h, sv, sv->o.steps_per_generation * std::max(1, sv->o.warm_generations)));
    } else if (sv->generations > sv->o.warm_generations) {
      FS_TRY(surrogate_train(h, sv, sv->o.steps_per_generation));
    }
    double rho = 0.0;
    if (sv->generations >= sv->o.warm_generations) {
      FS_TRY(surrogate_gate(h, sv, &rho));
      sv->gate_open = rho >= sv->o.gate;
    }
    sv->last_rho = rho;
    if (rho_out) rho_out[g] = rho;
    if (screened_out) screened_out[g] = screen ? 1 : 0;
    if (history) {
      argmin_kernel<<<1, 1024, 0, h->stream>>>(s->obj, NP, s->best);
      int b = 0;
      FS_CUDA(cudaMemcpyAsync(&b, s->best, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      FS_CUDA(cudaStreamSynchronize(h->stream));
      FS_CUDA(cudaMemcpy(&history[g], s->obj + b, sizeof(double), cudaMemcpyDeviceToHost));
    }
  }
  argmin_kernel<<<1, 1024, 0, h->stream>>>(s->obj, NP, s->best);
  FS_CUDA(cudaGetLastError());
  int b = 0;
  FS_CUDA(cudaMemcpyAsync(&b, s->best, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  if (best_obj) FS_CUDA(cudaMemcpy(best_obj, s->obj + b, sizeof(double), cudaMemcpyDeviceToHost));
  if (best_x)
    FS_CUDA(cudaMemcpy(best_x, s->pop + static_cast<int64_t>(b) * D, D * sizeof(double), cudaMemcpyDeviceToHost));
  return FS_OK;
}

int surrogate_init(fs_gpu *h, const fs_surrogate_opts *o) {
  surrogate_free(h->sur);
  h->sur = nullptr;
  mlp_free(h->mlp);
  h->mlp = nullptr;
  FS_TRY(mlp_create(h, h->D, o->seed, static_cast<float>(o->lr), &h->mlp));
  Surrogate *sv = new Surrogate();
  sv->o = *o;
  sv->D = h->D;
  sv->P = o->holdout > 0.0 ? std::max(2, static_cast<int>(std::lround(1.0 / o->holdout))) : 1;
  h->sur = sv;
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

int fs_gpu_surrogate_init(fs_gpu *h, const fs_surrogate_opts *opts) {
  if (!h || !opts) return FS_ERR_ARG;
  if (!h->have_model) return fsg::set_error(h, FS_ERR_STATE, "surrogate_init: no model");
  if (opts->batch < 8 || opts->batch % 8 || opts->screen < 1 || opts->warm_generations < 0 ||
      opts->steps_per_generation < 0 || !(opts->lr > 0.0) || opts->holdout < 0.0 || opts->holdout >= 1.0)
    return fsg::set_error(h, FS_ERR_ARG, "surrogate_init: bad options");
  cudaSetDevice(h->device);
  return fsg::surrogate_init(h, opts);
}

int fs_gpu_surrogate_param_count(fs_gpu *h, int64_t *n) {
  if (!h || !n) return FS_ERR_ARG;
  if (!h->mlp) return fsg::set_error(h, FS_ERR_STATE, "surrogate: not initialised");
  *n = fsg::mlp_param_count(h->D);
  return FS_OK;
}

int fs_gpu_surrogate_get_params(fs_gpu *h, float *params) {
  if (!h || !params) return FS_ERR_ARG;
  if (!h->mlp) return fsg::set_error(h, FS_ERR_STATE, "surrogate: not initialised");
  cudaSetDevice(h->device);
  return fsg::mlp_get(h, h->mlp, fsg::mlp_param_ptr(h->mlp), params);
}

int fs_gpu_surrogate_set_params(fs_gpu *h, const float *params) {
  if (!h || !params) return FS_ERR_ARG;
  if (!h->mlp) return fsg::set_error(h, FS_ERR_STATE, "surrogate: not initialised");
  cudaSetDevice(h->device);
  return fsg::mlp_set_params(h, h->mlp, params);
}

static int load_rows(fs_gpu *h, const float *x, const float *t, int32_t rows) {
  FS_TRY(fsg::mlp_reserve(h, h->mlp, rows));
  FS_CUDA(cudaMemcpyAsync(fsg::mlp_rows_x(h->mlp), x, static_cast<size_t>(rows) * h->D * sizeof(float),
                          cudaMemcpyHostToDevice, h->stream));
  if (t)
    FS_CUDA(cudaMemcpyAsync(fsg::mlp_rows_t(h->mlp), t, rows * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  return FS_OK;
}

int fs_gpu_surrogate_predict(fs_gpu *h, const float *x, int32_t rows, float *y) {
  if (!h || !x || !y || rows < 1) return FS_ERR_ARG;
  if (!h->mlp) return fsg::set_error(h, FS_ERR_STATE, "surrogate: not initialised");
  cudaSetDevice(h->device);
  FS_TRY(load_rows(h, x, nullptr, rows));
  FS_TRY(fsg::mlp_forward_dev(h, h->mlp, rows));
  FS_CUDA(cudaMemcpyAsync(y, fsg::mlp_rows_y(h->mlp), rows * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  return fsg::sync_checked(h);
}

int fs_gpu_surrogate_gradient(fs_gpu *h, const float *x, const float *t, int32_t rows, float *grad, float *loss) {
  if (!h || !x || !t || rows < 8) return FS_ERR_ARG;
  if (!h->mlp) return fsg::set_error(h, FS_ERR_STATE, "surrogate: not initialised");
  cudaSetDevice(h->device);
  FS_TRY(load_rows(h, x, t, rows));
  FS_TRY(fsg::mlp_gradient_dev(h, h->mlp, rows));
  if (loss) FS_CUDA(cudaMemcpyAsync(loss, fsg::mlp_loss_ptr(h->mlp), sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  FS_TRY(fsg::sync_checked(h));
  if (grad) FS_TRY(fsg::mlp_get(h, h->mlp, fsg::mlp_grad_ptr(h->mlp), grad));
  if (loss) *loss /= static_cast<float>(rows);
  return FS_OK;
}

int fs_gpu_surrogate_train(fs_gpu *h, const float *x, const float *t, int32_t rows, int32_t steps, float *loss) {
  if (!h || !x || !t || rows < 8 || steps < 0) return FS_ERR_ARG;
  if (!h->mlp) return fsg::set_error(h, FS_ERR_STATE, "surrogate: not initialised");
  cudaSetDevice(h->device);
  FS_TRY(load_rows(h, x, t, rows));
  for (int k = 0; k < steps; ++k) {
    FS_TRY(fsg::mlp_gradient_dev(h, h->mlp, rows));
    FS_TRY(fsg::mlp_adam_dev(h, h->mlp));
  }
  if (loss) FS_CUDA(cudaMemcpyAsync(loss, fsg::mlp_loss_ptr(h->mlp), sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  FS_TRY(fsg::sync_checked(h));
  if (loss) *loss /= static_cast<float>(rows);
  return FS_OK;
}

int fs_gpu_de_run_screened(fs_gpu *h, int32_t generations, double *best_obj, double *best_x, double *history,
                           double *rho, int32_t *screened) {
  if (!h || generations < 0) return FS_ERR_ARG;
  cudaSetDevice(h->device);
  return fsg::de_run_screened(h, generations, best_obj, best_x, history, rho, screened);
}

} // extern "C"
