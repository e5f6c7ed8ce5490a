// Device helpers shared by the configuration kernels (one CTA per
// configuration): shared-memory carving, geometry staging, pair vectors.
#pragma once

#include "spline_dev.cuh"

namespace fsg {
namespace {

// Bump allocator over the dynamic shared-memory block.  Offsets are aligned
// as integers and added to the block's base pointer, so every carved pointer
// stays a pointer into the shared window (no round trip through an integer
// address, which would turn its loads into generic ones).  The block itself
// is declared 16-byte aligned.
struct Smem {
  unsigned char *base;
  size_t off = 0;
  __device__ explicit Smem(unsigned char *b) : base(b) {}
  template <class X> __device__ X *take(size_t n, size_t align = 16) {
    off = (off + align - 1) & ~(align - 1);
    X *r = reinterpret_cast<X *>(base + off);
    off += n * sizeof(X);
    return r;
  }
};

inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

struct Common {
  const CfgDev *cfg;
  const double *wpos;
  const int32_t *type;
  const double *ref_force;
  const int32_t *nb_start;
  const uint32_t *nb_pack;
  const TableDesc *desc;
  const int32_t *cmap;
  const double *vals; // table values / analytic parameters (FP64, table order)
  int n_tables, n_segs, n_cmap, ntypes;
  int family; // FS_FAMILY_EAM or FS_FAMILY_PAIR
  int cfg_count;
};

// Stage the configuration geometry: wrapped positions (FP64), species, and
// the image shift table ix·a + iy·b + iz·c.
__device__ void stage_geometry(const CfgDev &cd, const Common &A, double *wpos, double *shift, uint8_t *typ) {
  const int N = cd.natoms;
  for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) wpos[k] = A.wpos[3 * static_cast<int64_t>(cd.atom0) + k];
  for (int k = threadIdx.x; k < N; k += blockDim.x) typ[k] = static_cast<uint8_t>(A.type[cd.atom0 + k]);
  const int wx = 2 * cd.sx + 1, wy = 2 * cd.sy + 1, wz = 2 * cd.sz + 1;
  for (int k = threadIdx.x; k < wx * wy * wz; k += blockDim.x) {
    const double ix = k / (wy * wz) - cd.sx, iy = (k / wz) % wy - cd.sy, iz = k % wz - cd.sz;
    for (int a = 0; a < 3; ++a) shift[3 * k + a] = ix * cd.box[3 * a] + iy * cd.box[3 * a + 1] + iz * cd.box[3 * a + 2];
  }
}

template <class T>
__device__ __forceinline__ void pair_vec(const double *wpos, const double *shift, int i, uint32_t pk, int &j,
                                         T &dx, T &dy, T &dz) {
  j = static_cast<int>(pk & 0xFFFFFu);
  const int img = static_cast<int>(pk >> 20);
  dx = static_cast<T>((wpos[3 * j] - wpos[3 * i]) + shift[3 * img]);
  dy = static_cast<T>((wpos[3 * j + 1] - wpos[3 * i + 1]) + shift[3 * img + 1]);
  dz = static_cast<T>((wpos[3 * j + 2] - wpos[3 * i + 2]) + shift[3 * img + 2]);
}

template <class T> __device__ __forceinline__ T sqrt_t(T x) { return sqrt(x); }

// pair_vec, also returning the pair's FP64 length (the FP64 path's r).
template <class T>
__device__ __forceinline__ double pair_vec_len(const double *wpos, const double *shift, int i, uint32_t pk, int &j,
                                               T &dx, T &dy, T &dz) {
  j = static_cast<int>(pk & 0xFFFFFu);
  const int img = static_cast<int>(pk >> 20);
  const double x = (wpos[3 * j] - wpos[3 * i]) + shift[3 * img];
  const double y = (wpos[3 * j + 1] - wpos[3 * i + 1]) + shift[3 * img + 1];
  const double z = (wpos[3 * j + 2] - wpos[3 * i + 2]) + shift[3 * img + 2];
  dx = static_cast<T>(x);
  dy = static_cast<T>(y);
  dz = static_cast<T>(z);
  return sqrt(x * x + y * y + z * z);
}

// FP64 length of pair_vec's pair vector, computed as the FP64 path computes
// it; the FP32 kernels use it only to decide a distance within a few ulps
// of a gate bound (gate_seg).
__device__ __forceinline__ double pair_len64(const double *wpos, const double *shift, int i, uint32_t pk) {
  const int j = static_cast<int>(pk & 0xFFFFFu);
  const int img = static_cast<int>(pk >> 20);
  const double dx = (wpos[3 * j] - wpos[3 * i]) + shift[3 * img];
  const double dy = (wpos[3 * j + 1] - wpos[3 * i + 1]) + shift[3 * img + 1];
  const double dz = (wpos[3 * j + 2] - wpos[3 * i + 2]) + shift[3 * img + 2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}


// Block sums of K values at once (one pair of barriers); valid on thread 0.
// red holds K × 32 doubles.
template <int K> __device__ void block_sum_k(double (&v)[K], double *red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * 32 + w] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double t = 0.0;
      for (int q = 0; q < nw; ++q) t += red[k * 32 + q];
      v[k] = t;
    }
}

// Runs of lanes with the same key, for keys that do not decrease across the
// warp (flat work items are ordered by central atom, then by neighbour): bit s of
// the links is set when lane + 2^s has this lane's key; head: the run's first
// lane.  All 32 lanes call these together.
__device__ __forceinline__ unsigned run_links(int key, int lane, bool &head) {
  unsigned nx = 0;
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int kk = __shfl_down_sync(0xffffffffu, key, 1 << s);
    if (lane + (1 << s) < 32 && kk == key) nx |= 1u << s;
  }
  const int kp = __shfl_up_sync(0xffffffffu, key, 1);
  head = lane == 0 || kp != key;
  return nx;
}
// Sum of v over this lane and the later lanes of its run (the whole run at its head).
template <class T> __device__ __forceinline__ T run_sum(T v, unsigned nx) {
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const T t = __shfl_down_sync(0xffffffffu, v, 1 << s);
    if (nx >> s & 1) v += t;
  }
  return v;
}

// Warp sums of NV values (NV = 4 or 8) by halving exchanges: at each of the
// first log2(NV) levels a lane keeps half of its values and trades the other
// half with its partner, then the last levels sum one value.  Lane l ends
// with the warp sum of value (l >> (5 − log2 NV)) & (NV − 1); every lane calls
// this together.  NV − 1 + 5 − log2(NV) shuffles (8 values: 9, not 40).
template <int NV, class T> __device__ __forceinline__ T warp_sum_tr(const T (&v)[NV], int lane) {
  static_assert(NV == 4 || NV == 8, "NV is 4 or 8");
  T a[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) a[q] = v[q];
  int h = NV / 2, bit = 16;
#pragma unroll
  for (; h >= 1; h >>= 1, bit >>= 1) {
    const bool up = lane & bit;
#pragma unroll
    for (int q = 0; q < h; ++q) {
      const T send = up ? a[q] : a[q + h];
      const T keep = up ? a[q + h] : a[q];
      a[q] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
    }
  }
  T s = a[0];
#pragma unroll
  for (; bit >= 1; bit >>= 1) s += __shfl_xor_sync(0xffffffffu, s, bit);
  return s;
}

// An atom with n neighbours has n(n − 1)/2 neighbour pairs (j < k) in rows
// a = 0 .. n − 2 of n − 1 − a pairs each, row a starting at a(2n − a − 1)/2.
// For pair offset u: the row a (from the quadratic's root, then a one-step
// integer correction either way) and u's offset within that row.
__device__ __forceinline__ void pair_row(int n, int &u, int &a) {
  const float b = 2.f * static_cast<float>(n) - 1.f;
  int r = static_cast<int>((b - sqrtf(fmaxf(b * b - 8.f * static_cast<float>(u), 0.f))) * 0.5f);
  r = max(0, min(r, n - 2));
  while (r > 0 && r * (2 * n - r - 1) / 2 > u) --r;
  while (r + 1 <= n - 2 && (r + 1) * (2 * n - r - 2) / 2 <= u) ++r;
  u -= r * (2 * n - r - 1) / 2;
  a = r;
}

// Largest i in [0, N) with first[i] <= w, for non-decreasing first[] with
// first[0] = 0 <= w < first[N]: the atom that owns work item w.
__device__ __forceinline__ int owner_of(const int *first, int N, int w) {
  int lo = 0, hi = N;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= w) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Work-item offsets of one configuration: pfirst[i] = first directed pair of
// atom i (relative to atom 0's), tfirst[i] = first neighbour pair (j < k) of
// atom i, n_i (n_i − 1)/2 per atom; both with the totals at [N].  One block
// scan; blockDim.x a multiple of 32, at most 1024.
__device__ void stage_work(const int32_t *nb, int N, int *pfirst, int *tfirst, int *wsum) {
  for (int k = threadIdx.x; k <= N; k += blockDim.x) pfirst[k] = nb[k] - nb[0];
  const int per = (N + blockDim.x - 1) / blockDim.x;
  const int b = min(N, static_cast<int>(threadIdx.x) * per), e = min(N, b + per);
  int s = 0;
  for (int k = b; k < e; ++k) {
    const int n = nb[k + 1] - nb[k];
    s += n * (n - 1) / 2;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = s;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int v = lane < nw ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    __syncwarp();
    if (lane < nw) wsum[lane] = v;
  }
  __syncthreads();
  int base = x - s + (w > 0 ? wsum[w - 1] : 0);
  for (int k = b; k < e; ++k) {
    tfirst[k] = base;
    const int n = nb[k + 1] - nb[k];
    base += n * (n - 1) / 2;
  }
  if (threadIdx.x == blockDim.x - 1) tfirst[N] = base;
}

} // namespace

// Kernel-argument view of a context's configurations, neighbour lists and
// tables.
template <class T> inline Common make_common(fs_gpu *h) {
  Common c;
  c.cfg = h->d_cfg;
  c.wpos = h->d_wpos;
  c.type = h->d_type;
  c.ref_force = h->d_ref_force;
  c.nb_start = h->d_nb_start;
  c.vals = h->d_vals;
  c.nb_pack = h->d_nb_pack;
  c.desc = h->d_desc;
  c.cmap = h->d_cmap;
  c.n_tables = static_cast<int>(h->desc.size());
  c.n_segs = h->n_segs;
  c.n_cmap = h->n_cmap;
  c.ntypes = h->ntypes;
  c.family = h->family;
  c.cfg_count = h->n_cfg;
  return c;
}

// The largest periodic-image count of the context's configurations.
inline int max_images(const fs_gpu *h) {
  int m = 1;
  for (const CfgDev &cd : h->cfg_host) {
    const int n = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
    m = n > m ? n : m;
  }
  return m;
}

} // namespace fsg
