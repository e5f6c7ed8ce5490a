// Device neighbour lists from device cell lists, bit-exact against the
// reference's build_periodic (src/core/neighbor_list.cpp:59-92).
//
// The integer set {(i, j, image)} is decided by an FP64 comparison
//   ‖((base + ix·a) + iy·b) + iz·c‖² ≤ rc²,  base = wrap(p_j) − wrap(p_i),
// so every operation is written with explicit __dadd_rn / __dmul_rn (no FMA
// contraction) in the reference's association order, and wrap() follows
// PeriodicBC::wrap (boundary_conditions.hpp:11-17,38-40):
// box·(f − floor f) with f = inv·r, each 3×3 product as (a0·v0 + a1·v1) + a2·v2.
//
// The reference tests every j against every image in [−s, s]³,
// s_k = ceil(rc·‖row_k(inv_box)‖): O(N²·images).  Here the candidates come
// from a cell list.  Along lattice direction k a configuration is cut into
// nc_k slabs of fractional width 1/nc_k ≥ rc·‖row_k(inv_box)‖·(1 + 1e-6); a
// pair within rc has |Δf_k| ≤ rc·‖row_k(inv_box)‖ (the fractional difference
// is row_k(inv_box)·d), so the slab of j's image differs from i's by at most
// one.  Cells of the periodic extension are "extended cells" e = c + δ; an
// extended cell is home cell e mod nc under image floor(e / nc).  When the
// box is narrower than the cutoff (nc_k = 1 and s_k > 1) the extended cells
// run over δ ∈ [−s_k, s_k], which is the reference's own image loop.  Each
// candidate (j, image) then takes the reference's exact test, so the set is
// the reference's.
//
// Order of a list: i, then j ascending, then image (ix, iy, iz)
// lexicographic, as the reference's loops emit them.  The cell walk finds
// the pairs in another order; a third pass sorts each atom's entries by the
// key (j << 12) | image, whose numeric order is exactly that order (the image
// code is ((ix + sx)·(2sy + 1) + (iy + sy))·(2sz + 1) + (iz + sz)).
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

// Cell grid of one configuration: slabs per lattice direction, the first
// entry of its cell offsets, and the extended-cell reach per direction.
struct CellGrid {
  int nc[3];
  int reach[3];
  int cell0; // first entry of this configuration's offsets in cell_start (ncells + 1 entries)
  int pad;
};

__device__ __forceinline__ int cell_coord(double f, int n) {
  const int c = static_cast<int>(floor(f * static_cast<double>(n)));
  return min(max(c, 0), n - 1);
}

// Bin one configuration's atoms (one CTA per configuration): cell of every
// atom, counts, offsets by a block scan, then the atoms of each cell (their
// order inside a cell is arbitrary; the lists are sorted afterwards).
// count holds zeros on entry.
__global__ void __launch_bounds__(256) cell_bin_kernel(const CfgDev *__restrict__ cfg, const CellGrid *__restrict__ grid,
                                                       const double *__restrict__ wpos, int32_t *__restrict__ cell_of,
                                                       int32_t *__restrict__ count, int32_t *__restrict__ cell_start,
                                                       int32_t *__restrict__ cell_atoms) {
  __shared__ int32_t carry;
  __shared__ int32_t wsum[8];
  const int c = blockIdx.x;
  const CfgDev &cd = cfg[c];
  const CellGrid G = grid[c];
  const int ncells = G.nc[0] * G.nc[1] * G.nc[2];
  int32_t *cnt = count + G.cell0;
  int32_t *cst = cell_start + G.cell0;
  for (int i = threadIdx.x; i < cd.natoms; i += blockDim.x) {
    const int64_t g = static_cast<int64_t>(cd.atom0) + i;
    const double r0 = wpos[3 * g], r1 = wpos[3 * g + 1], r2 = wpos[3 * g + 2];
    int cc[3];
    for (int k = 0; k < 3; ++k)
      cc[k] = cell_coord(dot3_rn(cd.inv[3 * k], cd.inv[3 * k + 1], cd.inv[3 * k + 2], r0, r1, r2), G.nc[k]);
    const int id = (cc[0] * G.nc[1] + cc[1]) * G.nc[2] + cc[2];
    cell_of[g] = id;
    atomicAdd(&cnt[id], 1);
  }
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  // exclusive scan of the counts, 256 cells per round
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int b = 0; b < ncells; b += blockDim.x) {
    const int k = b + threadIdx.x;
    const int v = k < ncells ? __ldcg(&cnt[k]) : 0; // (the counts were made by atomics)
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    int before = carry;
    for (int q = 0; q < w; ++q) before += wsum[q];
    if (k < ncells) cst[k] = before + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) cst[ncells] = carry;
  for (int k = threadIdx.x; k < ncells; k += blockDim.x) cnt[k] = 0; // reused as fill counters
  __syncthreads();
  for (int i = threadIdx.x; i < cd.natoms; i += blockDim.x) {
    const int id = cell_of[static_cast<int64_t>(cd.atom0) + i];
    const int slot = atomicAdd(&cnt[id], 1);
    cell_atoms[cd.atom0 + cst[id] + slot] = i;
  }
}

// The reference's test of one (i, j, image): d² of
// ((base + ix·a) + iy·b) + iz·c, in its association order.
__device__ __forceinline__ bool in_range(const CfgDev &cd, double bx, double by, double bz, int ix, int iy, int iz,
                                         double rcut2) {
  const double fx = static_cast<double>(ix), fy = static_cast<double>(iy), fz = static_cast<double>(iz);
  const double x1 = __dadd_rn(bx, __dmul_rn(fx, cd.box[0]));
  const double y1 = __dadd_rn(by, __dmul_rn(fx, cd.box[3]));
  const double z1 = __dadd_rn(bz, __dmul_rn(fx, cd.box[6]));
  const double x2 = __dadd_rn(x1, __dmul_rn(fy, cd.box[1]));
  const double y2 = __dadd_rn(y1, __dmul_rn(fy, cd.box[4]));
  const double z2 = __dadd_rn(z1, __dmul_rn(fy, cd.box[7]));
  const double x3 = __dadd_rn(x2, __dmul_rn(fz, cd.box[2]));
  const double y3 = __dadd_rn(y2, __dmul_rn(fz, cd.box[5]));
  const double z3 = __dadd_rn(z2, __dmul_rn(fz, cd.box[8]));
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(x3, x3), __dmul_rn(y3, y3)), __dmul_rn(z3, z3));
  return d2 <= rcut2;
}

__device__ __forceinline__ int floor_div(int a, int n) { return a >= 0 ? a / n : -((-a + n - 1) / n); }

// Walk atom i's extended cells.  WRITE = false: count the in-range entries;
// WRITE = true: write them (unsorted) at out.  Warp-wide; every lane returns
// the total.
template <bool WRITE>
__device__ int walk_cells(const CfgDev &cd, const CellGrid &G, const double *__restrict__ wpos,
                          const int32_t *__restrict__ cell_start, const int32_t *__restrict__ cell_atoms, int i,
                          int ci, double rcut2, uint32_t *out) {
  const int lane = threadIdx.x & 31;
  const int64_t gi = static_cast<int64_t>(cd.atom0) + i;
  const double xi = wpos[3 * gi], yi = wpos[3 * gi + 1], zi = wpos[3 * gi + 2];
  const int c0 = ci / (G.nc[1] * G.nc[2]), c1 = (ci / G.nc[2]) % G.nc[1], c2 = ci % G.nc[2];
  const int wy = 2 * cd.sy + 1, wz = 2 * cd.sz + 1;
  const int32_t *cst = cell_start + G.cell0;
  const int32_t *catoms = cell_atoms + cd.atom0;
  int total = 0;
  for (int d0 = -G.reach[0]; d0 <= G.reach[0]; ++d0) {
    const int e0 = c0 + d0, ix = floor_div(e0, G.nc[0]), h0 = e0 - ix * G.nc[0];
    if (ix < -cd.sx || ix > cd.sx) continue;
    for (int d1 = -G.reach[1]; d1 <= G.reach[1]; ++d1) {
      const int e1 = c1 + d1, iy = floor_div(e1, G.nc[1]), h1 = e1 - iy * G.nc[1];
      if (iy < -cd.sy || iy > cd.sy) continue;
      for (int d2 = -G.reach[2]; d2 <= G.reach[2]; ++d2) {
        const int e2 = c2 + d2, iz = floor_div(e2, G.nc[2]), h2 = e2 - iz * G.nc[2];
        if (iz < -cd.sz || iz > cd.sz) continue;
        const int home = (h0 * G.nc[1] + h1) * G.nc[2] + h2;
        const bool zero_img = ix == 0 && iy == 0 && iz == 0;
        const uint32_t img = static_cast<uint32_t>(((ix + cd.sx) * wy + (iy + cd.sy)) * wz + (iz + cd.sz));
        const int a0 = cst[home], a1 = cst[home + 1];
        for (int k0 = a0; k0 < a1; k0 += 32) {
          bool hit = false;
          int j = 0;
          if (k0 + lane < a1) {
            j = catoms[k0 + lane];
            if (!(zero_img && j == i)) {
              const int64_t gj = static_cast<int64_t>(cd.atom0) + j;
              const double bx = __dsub_rn(wpos[3 * gj], xi);
              const double by = __dsub_rn(wpos[3 * gj + 1], yi);
              const double bz = __dsub_rn(wpos[3 * gj + 2], zi);
              hit = in_range(cd, bx, by, bz, ix, iy, iz, rcut2);
            }
          }
          const unsigned m = __ballot_sync(0xffffffffu, hit);
          if (WRITE && hit) out[total + __popc(m & ((1u << lane) - 1u))] = static_cast<uint32_t>(j) | (img << 20);
          total += __popc(m);
        }
      }
    }
  }
  return total;
}

template <bool WRITE>
__global__ void __launch_bounds__(256) neighbor_cell_kernel(const CfgDev *__restrict__ cfg, const CellGrid *__restrict__ grid,
                                                            const double *__restrict__ wpos, double rcut2,
                                                            const int32_t *__restrict__ cell_of,
                                                            const int32_t *__restrict__ cell_start,
                                                            const int32_t *__restrict__ cell_atoms,
                                                            int32_t *__restrict__ count, const int32_t *__restrict__ start,
                                                            uint32_t *__restrict__ tmp) {
  const int c = blockIdx.x;
  const CfgDev &cd = cfg[c];
  const CellGrid G = grid[c];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int i = warp; i < cd.natoms; i += nwarp) {
    const int64_t gi = static_cast<int64_t>(cd.atom0) + i;
    const int n = walk_cells<WRITE>(cd, G, wpos, cell_start, cell_atoms, i, cell_of[gi], rcut2,
                                    WRITE ? tmp + start[gi] : nullptr);
    if (!WRITE && lane == 0) count[gi] = n;
  }
}

// Sort each atom's entries into the reference's order (warp per atom): the
// rank of an entry is the number of smaller keys (keys are distinct).  Lists
// of up to kSortStage entries are ranked from shared memory, longer ones
// from the unsorted copy in global memory.
constexpr int kSortStage = 512;
__device__ __forceinline__ uint32_t sort_key(uint32_t pk) { return ((pk & 0xFFFFFu) << 12) | (pk >> 20); }

__global__ void __launch_bounds__(256) neighbor_sort_kernel(int64_t n_atoms, const int32_t *__restrict__ start,
                                                            const uint32_t *__restrict__ tmp,
                                                            uint32_t *__restrict__ pack) {
  __shared__ uint32_t keys[8][kSortStage];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t gi = static_cast<int64_t>(blockIdx.x) * 8 + w;
  if (gi >= n_atoms) return;
  const int s = start[gi], n = start[gi + 1] - s;
  const uint32_t *src = tmp + s;
  const bool staged = n <= kSortStage;
  if (staged)
    for (int k = lane; k < n; k += 32) keys[w][k] = sort_key(src[k]);
  __syncwarp();
  for (int k = lane; k < n; k += 32) {
    const uint32_t pk = src[k], key = sort_key(pk);
    int rank = 0;
    if (staged)
      for (int q = 0; q < n; ++q) rank += keys[w][q] < key;
    else
      for (int q = 0; q < n; ++q) rank += sort_key(src[q]) < key;
    pack[s + rank] = pk;
  }
}

// Slabs per lattice direction: the most whose width is at least the cutoff
// (with a 1e-6 relative margin that covers the rounding of the fractional
// coordinates), at most 256, and at most about two cells per atom.
void cell_grid(const CfgDev &cd, double rcut, CellGrid &G) {
  int s[3] = {cd.sx, cd.sy, cd.sz};
  for (int k = 0; k < 3; ++k) {
    const double *r = cd.inv + 3 * k;
    const double w = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double slabs = 1.0 / (rcut * w * (1.0 + 1e-6));
    const int n = std::isfinite(slabs) ? static_cast<int>(std::min(256.0, std::floor(slabs))) : 1;
    G.nc[k] = std::max(1, n);
  }
  const int64_t cap = std::max<int64_t>(64, 2 * static_cast<int64_t>(cd.natoms));
  while (static_cast<int64_t>(G.nc[0]) * G.nc[1] * G.nc[2] > cap) {
    int k = 0;
    for (int q = 1; q < 3; ++q)
      if (G.nc[q] > G.nc[k]) k = q;
    --G.nc[k];
  }
  // slabs at least rc wide: neighbouring cells suffice; one slab narrower
  // than the cutoff (nc = 1): the reference's images [−s, s]
  for (int k = 0; k < 3; ++k) G.reach[k] = G.nc[k] > 1 ? 1 : s[k];
  G.pad = 0;
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
  h->runs_valid = false; // pair runs index the neighbour lists
  h->max_list = -1;
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

  // cell lists (build-time buffers, freed at the end)
  std::vector<CellGrid> grid(n_cfg);
  int64_t cell_entries = 0;
  if (!none)
    for (int c = 0; c < n_cfg; ++c) {
      cell_grid(h->cfg_host[c], rcut, grid[c]);
      grid[c].cell0 = static_cast<int>(cell_entries);
      cell_entries += static_cast<int64_t>(grid[c].nc[0]) * grid[c].nc[1] * grid[c].nc[2] + 1;
    }
  if (cell_entries > (int64_t(1) << 31) - 1) return set_error(h, FS_ERR_UNSUPPORTED, "neighbour list: too many cells");
  CellGrid *d_grid = nullptr;
  int32_t *d_cell_of = nullptr, *d_cell_cnt = nullptr, *d_cell_start = nullptr, *d_cell_atoms = nullptr;
  uint32_t *d_tmp = nullptr;
  auto release = [&] {
    cudaFree(d_grid);
    cudaFree(d_cell_of);
    cudaFree(d_cell_cnt);
    cudaFree(d_cell_start);
    cudaFree(d_cell_atoms);
    cudaFree(d_tmp);
  };
  auto fail = [&](cudaError_t e, const char *what) {
    cudaStreamSynchronize(h->stream);
    release();
    h->err = std::string(what) + ": " + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  };
#define FS_NB(call)                                                                                                    \
  do {                                                                                                                 \
    const cudaError_t e_ = (call);                                                                                     \
    if (e_ != cudaSuccess) return fail(e_, #call);                                                                     \
  } while (0)
  if (!none && n_cfg > 0) {
    const size_t na = static_cast<size_t>(std::max<int64_t>(h->n_atoms, 1));
    FS_NB(cudaMalloc(&d_grid, n_cfg * sizeof(CellGrid)));
    FS_NB(cudaMalloc(&d_cell_of, na * sizeof(int32_t)));
    FS_NB(cudaMalloc(&d_cell_atoms, na * sizeof(int32_t)));
    FS_NB(cudaMalloc(&d_cell_cnt, cell_entries * sizeof(int32_t)));
    FS_NB(cudaMalloc(&d_cell_start, cell_entries * sizeof(int32_t)));
    FS_NB(cudaMemcpyAsync(d_grid, grid.data(), n_cfg * sizeof(CellGrid), cudaMemcpyHostToDevice, h->stream));
    FS_NB(cudaMemsetAsync(d_cell_cnt, 0, cell_entries * sizeof(int32_t), h->stream));
    cell_bin_kernel<<<n_cfg, 256, 0, h->stream>>>(h->d_cfg, d_grid, h->d_wpos, d_cell_of, d_cell_cnt, d_cell_start,
                                                  d_cell_atoms);
    FS_NB(cudaGetLastError());
    neighbor_cell_kernel<false><<<n_cfg, 256, 0, h->stream>>>(h->d_cfg, d_grid, h->d_wpos, rcut2, d_cell_of,
                                                              d_cell_start, d_cell_atoms, h->d_nb_count, nullptr,
                                                              nullptr);
    FS_NB(cudaGetLastError());
    h->launches += 2;
  }
  std::vector<int32_t> cnt(h->n_atoms);
  FS_NB(cudaMemcpyAsync(cnt.data(), h->d_nb_count, h->n_atoms * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  FS_NB(cudaStreamSynchronize(h->stream));
  std::vector<int32_t> start(h->n_atoms + 1, 0);
  int64_t total = 0;
  int longest = 0; // the longest list (the LMBTR kernel's per-warp neighbour slices)
  for (int64_t i = 0; i < h->n_atoms; ++i) {
    start[i] = static_cast<int32_t>(total);
    total += cnt[i];
    longest = std::max(longest, cnt[i]);
    if (total > (int64_t(1) << 31) - 1) {
      release();
      return set_error(h, FS_ERR_UNSUPPORTED, "neighbour list: more than 2^31 pairs");
    }
  }
  start[h->n_atoms] = static_cast<int32_t>(total);
  for (int c = 0; c < n_cfg; ++c) h->cfg_host[c].pair0 = start[h->atom0[c]];
  h->n_pairs = total;
  h->max_list = longest;
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
    FS_NB(cudaMalloc(&h->d_cfg_by_work, std::max(n_cfg, 1) * sizeof(int32_t)));
    FS_NB(cudaMemcpyAsync(h->d_cfg_by_work, order.data(), n_cfg * sizeof(int32_t), cudaMemcpyHostToDevice,
                          h->stream));
  }
  FS_NB(cudaMemcpyAsync(h->d_nb_start, start.data(), (h->n_atoms + 1) * sizeof(int32_t), cudaMemcpyHostToDevice,
                        h->stream));
  FS_NB(cudaMemcpyAsync(h->d_cfg, h->cfg_host.data(), n_cfg * sizeof(CfgDev), cudaMemcpyHostToDevice, h->stream));
  if (h->d_nb_pack) cudaFree(h->d_nb_pack);
  h->d_nb_pack = nullptr;
  FS_NB(cudaMalloc(&h->d_nb_pack, std::max<int64_t>(total, 1) * sizeof(uint32_t)));
  if (!none && total > 0) {
    FS_NB(cudaMalloc(&d_tmp, total * sizeof(uint32_t)));
    neighbor_cell_kernel<true><<<n_cfg, 256, 0, h->stream>>>(h->d_cfg, d_grid, h->d_wpos, rcut2, d_cell_of,
                                                             d_cell_start, d_cell_atoms, nullptr, h->d_nb_start,
                                                             d_tmp);
    FS_NB(cudaGetLastError());
    const unsigned blocks = static_cast<unsigned>((h->n_atoms + 7) / 8);
    neighbor_sort_kernel<<<blocks, 256, 0, h->stream>>>(h->n_atoms, h->d_nb_start, d_tmp, h->d_nb_pack);
    FS_NB(cudaGetLastError());
    h->launches += 2;
  }
  FS_NB(cudaStreamSynchronize(h->stream));
#undef FS_NB
  release();
  h->rcut_built = none ? 0.0 : rcut;
  return build_pair_runs(h);
}

} // namespace fsg
