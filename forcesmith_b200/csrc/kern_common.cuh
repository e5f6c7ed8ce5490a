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


} // namespace
} // namespace fsg
