// Pair runs: each atom's neighbour pairs sorted by (neighbour species,
// spline segment), for models whose pair and density tables share one knot
// grid (a setfl-style EAM model: every r-function on x_k = x0 + k·h).
//
// On a shared grid a pair's segment e and local coordinate t are the same in
// every radial table and depend only on the geometry, so they are found once
// per neighbour list.  Sorted by key = (t_j << 8) | e, consecutive pairs of
// an atom with one key (a run; 1.8 pairs on average in the ternary
// benchmark) use the same segment of φ_{t_i t_j}, ρ_{t_j} and ρ_{t_i}: the
// population kernel loads each trial's coefficients once per run instead of
// once per pair.  (u, t) come from the FP64 pair vector, t as seg_of64 forms
// it, so the segment and coordinate are the ones the FP32 kernels use.
#include "kern_common.cuh"

#include <algorithm>

namespace fsg {
namespace {

// Each atom's in-gate pairs (closed gate [x0, x_{n−1}], decided on the FP64
// length), sorted by key (stable within a key), into the atom's slots of the
// neighbour list: ra = (u, t), rb = (packed entry, key), rr = length;
// rcnt = their count.
// One CTA per configuration, a warp per atom; keys go through keys_tmp.
__global__ void __launch_bounds__(256) run_pairs_kernel(Common C, RunGrid G, int32_t *__restrict__ keys_tmp,
                                                        float4 *__restrict__ ra, int2 *__restrict__ rb,
                                                        float *__restrict__ rr, int32_t *__restrict__ rcnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const CfgDev &cd = C.cfg[blockIdx.x];
  const int N = cd.natoms;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  Smem S(smem_raw);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  stage_geometry(cd, C, wpos, shift, typ);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  constexpr int kOut = 0x7fffffff;
  // segment and local coordinate on the grid, as seg_of64 forms them
  auto locate = [&](double r64, int &e, float &t) {
    if (r64 <= G.x0) {
      e = 0;
      t = static_cast<float>((r64 - G.x0) * G.inv_h);
    } else if (r64 >= G.xmax) {
      e = G.n;
      t = static_cast<float>((r64 - G.xmax) * G.inv_h);
    } else {
      const double u = (r64 - G.x0) * G.inv_h;
      int k = static_cast<int>(u);
      k = min(max(k, 0), G.n - 2);
      t = static_cast<float>(u - static_cast<double>(k));
      e = 1 + k;
    }
  };
  auto vec = [&](int i, uint32_t pk, int &j, double &x, double &y, double &z) {
    j = static_cast<int>(pk & 0xFFFFFu);
    const int img = static_cast<int>(pk >> 20);
    x = (wpos[3 * j] - wpos[3 * i]) + shift[3 * img];
    y = (wpos[3 * j + 1] - wpos[3 * i + 1]) + shift[3 * img + 1];
    z = (wpos[3 * j + 2] - wpos[3 * i + 2]) + shift[3 * img + 2];
  };
  for (int i = w; i < N; i += nw) {
    const int64_t gi = static_cast<int64_t>(cd.atom0) + i;
    const int s0 = C.nb_start[gi], cnt = C.nb_start[gi + 1] - s0;
    int in_gate = 0;
    for (int q = lane; q < cnt; q += 32) {
      int j;
      double x, y, z;
      vec(i, C.nb_pack[s0 + q], j, x, y, z);
      const double r64 = sqrt(x * x + y * y + z * z);
      int key = kOut;
      if (r64 >= G.x0 && r64 <= G.xmax) {
        int e;
        float t;
        locate(r64, e, t);
        key = (typ[j] << kRunKeyBits) | e;
        ++in_gate;
      }
      keys_tmp[s0 + q] = key;
    }
    for (int o = 16; o > 0; o >>= 1) in_gate += __shfl_xor_sync(0xffffffffu, in_gate, o);
    __syncwarp();
    for (int q = lane; q < cnt; q += 32) {
      const int key = keys_tmp[s0 + q];
      if (key == kOut) continue;
      int rank = 0;
      for (int o = 0; o < cnt; ++o) {
        const int k2 = keys_tmp[s0 + o];
        rank += (k2 < key) || (k2 == key && o < q);
      }
      const uint32_t pk = C.nb_pack[s0 + q];
      int j;
      double x, y, z;
      vec(i, pk, j, x, y, z);
      const double r64 = sqrt(x * x + y * y + z * z);
      int e;
      float t;
      locate(r64, e, t);
      float4 a = make_float4(0.f, 0.f, 0.f, t);
      if (r64 >= 1e-14) {
        a.x = static_cast<float>(x / r64);
        a.y = static_cast<float>(y / r64);
        a.z = static_cast<float>(z / r64);
      }
      ra[s0 + rank] = a;
      rb[s0 + rank] = make_int2(static_cast<int>(pk), key);
      rr[s0 + rank] = r64 >= 1e-14 ? static_cast<float>(r64) : -1.f; // −1: coincident atoms, no pair force
    }
    if (lane == 0) rcnt[gi] = in_gate;
  }
}

} // namespace

// The shared knot grid of the pair and density tables, when the model has
// one and the population kernel can use it (FP32 EAM, spline tables, at most
// kRunMaxN knots on the grid, at most kRunMaxT species).
bool pair_runs_grid(const fs_gpu *h, RunGrid *g) {
  if (h->precision != FS_PREC_FP32 || h->family != FS_FAMILY_EAM || !h->have_model) return false;
  const int nt = h->ntypes, np = npair_of(nt);
  if (nt > kRunMaxT || static_cast<int>(h->desc.size()) != np + 2 * nt) return false;
  const TableDesc &d0 = h->desc[0];
  for (int t = 0; t < np + 2 * nt; ++t) {
    const TableDesc &d = h->desc[t];
    if (d.kind != FS_TABLE_SPLINE || d.n < 2) return false;
    if (t < np + nt && (d.n != d0.n || d.x0 != d0.x0 || d.h != d0.h || d.xmax != d0.xmax)) return false;
  }
  if (d0.n > kRunMaxN) return false;
  g->x0 = d0.x0;
  g->xmax = d0.xmax;
  g->inv_h = d0.inv_h;
  g->n = d0.n;
  return true;
}

// Builds the pair runs for the current neighbour lists when the model has a
// shared grid (else leaves them invalid); called after every neighbour build.
int build_pair_runs(fs_gpu *h) {
  h->runs_valid = false;
  RunGrid g;
  if (h->n_pairs == 0 || !pair_runs_grid(h, &g)) return FS_OK;
  const size_t sm = align16(3 * static_cast<size_t>(h->max_natoms) * sizeof(double)) +
                    align16(3 * max_images(h) * sizeof(double)) + align16(h->max_natoms) + 64;
  if (sm > 227 * 1024) return FS_OK; // the population kernel then walks pairs unsorted
  for (void *p : {static_cast<void *>(h->d_run_a), static_cast<void *>(h->d_run_b), static_cast<void *>(h->d_run_cnt),
                  static_cast<void *>(h->d_run_r)})
    if (p) cudaFree(p);
  h->d_run_a = nullptr;
  h->d_run_b = nullptr;
  h->d_run_cnt = nullptr;
  h->d_run_r = nullptr;
  const size_t np = static_cast<size_t>(h->n_pairs);
  int32_t *keys = nullptr;
  FS_CUDA(cudaMalloc(&h->d_run_a, np * sizeof(float4)));
  FS_CUDA(cudaMalloc(&h->d_run_b, np * sizeof(int2)));
  FS_CUDA(cudaMalloc(&h->d_run_r, np * sizeof(float)));
  FS_CUDA(cudaMalloc(&h->d_run_cnt, std::max<int64_t>(h->n_atoms, 1) * sizeof(int32_t)));
  FS_CUDA(cudaMalloc(&keys, np * sizeof(int32_t)));
  cudaError_t e = cudaFuncSetAttribute(run_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(sm));
  if (e == cudaSuccess) {
    run_pairs_kernel<<<h->n_cfg, 256, sm, h->stream>>>(make_common<float>(h), g, keys, h->d_run_a, h->d_run_b,
                                                       h->d_run_r, h->d_run_cnt);
    e = cudaGetLastError();
    ++h->launches;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(keys);
  if (e != cudaSuccess) return set_error(h, FS_ERR_CUDA, std::string("pair runs: ") + cudaGetErrorString(e));
  h->runs_valid = true;
  return FS_OK;
}

} // namespace fsg
