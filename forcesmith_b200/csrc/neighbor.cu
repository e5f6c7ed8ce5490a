// Device neighbour lists, bit-exact against the reference's build_periodic
// (src/core/neighbor_list.cpp:59-92).
//
// The integer set {(i, j, image)} is decided by an FP64 comparison
//   ‖((base + ix·a) + iy·b) + iz·c‖² ≤ rc²,  base = wrap(p_j) − wrap(p_i),
// so every operation is written with explicit __dadd_rn / __dmul_rn (no FMA
// contraction) in the reference's association order, and wrap() follows
// PeriodicBC::wrap (boundary_conditions.hpp:11-17,38-40):
// box·(f − floor f) with f = inv·r, each 3×3 product as (a0·v0 + a1·v1) + a2·v2.
//
// Order of a list: i, then j ascending, then image (ix, iy, iz)
// lexicographic, exactly as the reference's loops emit them.  Each warp owns
// an atom i; lanes take consecutive j, count their in-range images, and a
// warp exclusive scan places every lane's pairs behind those of lower j.
#include "internal.cuh"

#include <algorithm>
#include <cmath>

namespace fsg {
namespace {

__device__ __forceinline__ double dot3_rn(double a0, double a1, double a2, double v0, double v1,
                                          double v2) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a0, v0), __dmul_rn(a1, v1)), __dmul_rn(a2, v2));
}

__global__ void wrap_kernel(const CfgDev *__restrict__ cfg, int n_cfg, const double *__restrict__ pos,
                            double *__restrict__ wpos) {
  const int c = blockIdx.x;
  if (c >= n_cfg) return;
  const CfgDev &cd = cfg[c];
  for (int i = threadIdx.x; i < cd.natoms; i += blockDim.x) {
    const int64_t g = static_cast<int64_t>(cd.atom0) + i;
    const double r0 = pos[3 * g], r1 = pos[3 * g + 1], r2 = pos[3 * g + 2];
    double f[3];
    for (int k = 0; k < 3; ++k) {
      const double v = dot3_rn(cd.inv[3 * k], cd.inv[3 * k + 1], cd.inv[3 * k + 2], r0, r1, r2);
      f[k] = __dsub_rn(v, floor(v));
    }
    for (int k = 0; k < 3; ++k)
      wpos[3 * g + k] = dot3_rn(cd.box[3 * k], cd.box[3 * k + 1], cd.box[3 * k + 2], f[0], f[1], f[2]);
  }
}

// Number of in-range images of (i, j), and optionally their packed codes.
template <bool WRITE>
__device__ __forceinline__ int scan_images(const CfgDev &cd, int i, int j, double bx, double by,
                                           double bz, double rcut2, uint32_t *out) {
  const int wy = 2 * cd.sy + 1, wz = 2 * cd.sz + 1;
  int cnt = 0;
  for (int ix = -cd.sx; ix <= cd.sx; ++ix) {
    const double fx = static_cast<double>(ix);
    const double x1 = __dadd_rn(bx, __dmul_rn(fx, cd.box[0]));
    const double y1 = __dadd_rn(by, __dmul_rn(fx, cd.box[3]));
    const double z1 = __dadd_rn(bz, __dmul_rn(fx, cd.box[6]));
    for (int iy = -cd.sy; iy <= cd.sy; ++iy) {
      const double fy = static_cast<double>(iy);
      const double x2 = __dadd_rn(x1, __dmul_rn(fy, cd.box[1]));
      const double y2 = __dadd_rn(y1, __dmul_rn(fy, cd.box[4]));
      const double z2 = __dadd_rn(z1, __dmul_rn(fy, cd.box[7]));
      for (int iz = -cd.sz; iz <= cd.sz; ++iz) {
        if (i == j && ix == 0 && iy == 0 && iz == 0) continue;
        const double fz = static_cast<double>(iz);
        const double x3 = __dadd_rn(x2, __dmul_rn(fz, cd.box[2]));
        const double y3 = __dadd_rn(y2, __dmul_rn(fz, cd.box[5]));
        const double z3 = __dadd_rn(z2, __dmul_rn(fz, cd.box[8]));
        const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(x3, x3), __dmul_rn(y3, y3)), __dmul_rn(z3, z3));
        if (d2 > rcut2) continue;
        if (WRITE) {
          const uint32_t img = static_cast<uint32_t>(((ix + cd.sx) * wy + (iy + cd.sy)) * wz + (iz + cd.sz));
          out[cnt] = static_cast<uint32_t>(j) | (img << 20);
        }
        ++cnt;
      }
    }
  }
  return cnt;
}

template <bool WRITE>
__global__ void __launch_bounds__(256) neighbor_kernel(const CfgDev *__restrict__ cfg, int n_cfg,
                                                       const double *__restrict__ wpos, double rcut2,
                                                       int32_t *__restrict__ count,
                                                       const int32_t *__restrict__ start,
                                                       uint32_t *__restrict__ pack) {
  const int c = blockIdx.x;
  if (c >= n_cfg) return;
  const CfgDev &cd = cfg[c];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int i = warp; i < cd.natoms; i += nwarp) {
    const int64_t gi = static_cast<int64_t>(cd.atom0) + i;
    const double xi = wpos[3 * gi], yi = wpos[3 * gi + 1], zi = wpos[3 * gi + 2];
    int base = 0;
    const int64_t o0 = WRITE ? start[gi] : 0;
    for (int j0 = 0; j0 < cd.natoms; j0 += 32) {
      const int j = j0 + lane;
      int cnt = 0;
      double bx = 0, by = 0, bz = 0;
      if (j < cd.natoms) {
        const int64_t gj = static_cast<int64_t>(cd.atom0) + j;
        bx = __dsub_rn(wpos[3 * gj], xi);
        by = __dsub_rn(wpos[3 * gj + 1], yi);
        bz = __dsub_rn(wpos[3 * gj + 2], zi);
        cnt = scan_images<false>(cd, i, j, bx, by, bz, rcut2, nullptr);
      }
      // exclusive scan of the lanes' counts keeps the j-ascending order
      int incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      if (WRITE && cnt > 0) scan_images<true>(cd, i, j, bx, by, bz, rcut2, pack + o0 + base + incl - cnt);
      base += total;
    }
    if (!WRITE && lane == 0) count[gi] = base;
  }
}

} // namespace

int build_neighbors(fs_gpu *h, double rcut) {
  const int n_cfg = h->n_cfg;
  // image shells sx = ceil(rc·‖row_k(inv_box)‖) (neighbor_list.cpp:65-71)
  int64_t max_img = 0;
  for (int c = 0; c < n_cfg; ++c) {
    CfgDev &cd = h->cfg_host[c];
    int s[3];
    for (int k = 0; k < 3; ++k) {
      const double *r = cd.inv + 3 * k;
      const double w = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      s[k] = (!std::isfinite(w) || w <= 0.0 || !(rcut > 0.0 && std::isfinite(rcut)))
                 ? 0
                 : static_cast<int>(std::ceil(rcut * w));
    }
    cd.sx = s[0];
    cd.sy = s[1];
    cd.sz = s[2];
    const int64_t ni = static_cast<int64_t>(2 * s[0] + 1) * (2 * s[1] + 1) * (2 * s[2] + 1);
    max_img = std::max(max_img, ni);
  }
  if (max_img > 4096)
    return set_error(h, FS_ERR_UNSUPPORTED, "neighbour list: more than 4096 periodic images (box far smaller than the cutoff)");
  const bool none = !(rcut > 0.0 && std::isfinite(rcut));
  const double rcut2 = none ? -1.0 : rcut * rcut;
  FS_CUDA(cudaMemcpyAsync(h->d_cfg, h->cfg_host.data(), n_cfg * sizeof(CfgDev), cudaMemcpyHostToDevice,
                          h->stream));
  wrap_kernel<<<n_cfg, 128, 0, h->stream>>>(h->d_cfg, n_cfg, h->d_pos, h->d_wpos);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  if (h->d_nb_count) cudaFree(h->d_nb_count);
  if (h->d_nb_start) cudaFree(h->d_nb_start);
  h->d_nb_count = nullptr;
  h->d_nb_start = nullptr;
  FS_CUDA(cudaMalloc(&h->d_nb_count, h->n_atoms * sizeof(int32_t)));
  FS_CUDA(cudaMalloc(&h->d_nb_start, (h->n_atoms + 1) * sizeof(int32_t)));
  FS_CUDA(cudaMemsetAsync(h->d_nb_count, 0, h->n_atoms * sizeof(int32_t), h->stream));
  if (!none) {
    neighbor_kernel<false><<<n_cfg, 256, 0, h->stream>>>(h->d_cfg, n_cfg, h->d_wpos, rcut2, h->d_nb_count,
                                                         nullptr, nullptr);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  std::vector<int32_t> cnt(h->n_atoms);
  FS_CUDA(cudaMemcpyAsync(cnt.data(), h->d_nb_count, h->n_atoms * sizeof(int32_t), cudaMemcpyDeviceToHost,
                          h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  std::vector<int32_t> start(h->n_atoms + 1, 0);
  int64_t total = 0;
  for (int64_t i = 0; i < h->n_atoms; ++i) {
    start[i] = static_cast<int32_t>(total);
    total += cnt[i];
    if (total > (int64_t(1) << 31) - 1)
      return set_error(h, FS_ERR_UNSUPPORTED, "neighbour list: more than 2^31 pairs");
  }
  start[h->n_atoms] = static_cast<int32_t>(total);
  for (int c = 0; c < n_cfg; ++c) h->cfg_host[c].pair0 = start[h->atom0[c]];
  h->n_pairs = total;
  std::vector<int32_t> order(n_cfg); // outlives the asynchronous upload below (synchronised at the end)
  {
    std::vector<int64_t> work(n_cfg, 0);
    h->max_cfg_work = 0;
    for (int c = 0; c < n_cfg; ++c) {
      const int64_t a0 = h->atom0[c];
      for (int64_t i = a0; i < a0 + h->cfg_host[c].natoms; ++i)
        work[c] += cnt[i] + static_cast<int64_t>(cnt[i]) * (cnt[i] - 1) / 2;
      h->max_cfg_work = std::max(h->max_cfg_work, work[c]);
    }
    for (int c = 0; c < n_cfg; ++c) order[c] = c;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return work[x] > work[y]; });
    if (h->d_cfg_by_work) cudaFree(h->d_cfg_by_work);
    h->d_cfg_by_work = nullptr;
    FS_CUDA(cudaMalloc(&h->d_cfg_by_work, std::max(n_cfg, 1) * sizeof(int32_t)));
    FS_CUDA(cudaMemcpyAsync(h->d_cfg_by_work, order.data(), n_cfg * sizeof(int32_t), cudaMemcpyHostToDevice,
                            h->stream));
  }
  FS_CUDA(cudaMemcpyAsync(h->d_nb_start, start.data(), (h->n_atoms + 1) * sizeof(int32_t),
                          cudaMemcpyHostToDevice, h->stream));
  FS_CUDA(cudaMemcpyAsync(h->d_cfg, h->cfg_host.data(), n_cfg * sizeof(CfgDev), cudaMemcpyHostToDevice,
                          h->stream));
  if (h->d_nb_pack) cudaFree(h->d_nb_pack);
  h->d_nb_pack = nullptr;
  FS_CUDA(cudaMalloc(&h->d_nb_pack, std::max<int64_t>(total, 1) * sizeof(uint32_t)));
  if (!none && total > 0) {
    neighbor_kernel<true><<<n_cfg, 256, 0, h->stream>>>(h->d_cfg, n_cfg, h->d_wpos, rcut2, nullptr,
                                                        h->d_nb_start, h->d_nb_pack);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  FS_CUDA(cudaStreamSynchronize(h->stream));
  h->rcut_built = none ? 0.0 : rcut;
  return FS_OK;
}

} // namespace fsg
