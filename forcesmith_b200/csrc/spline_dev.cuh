// Device-side spline evaluation shared by the evaluation kernels.
#pragma once

#include "internal.cuh"

#include <type_traits>

namespace fsg {

// Compact per-table record staged in shared memory.
template <class T> struct STab {
  T x0, inv_h, xmax, h;
  double x0d, hd; // FP64 grid for the exact interval search
  int n, seg0, cmap0, kind;
};

template <class T> __device__ __forceinline__ void load_stab(STab<T> &s, const TableDesc &d) {
  s.x0 = static_cast<T>(d.x0);
  s.inv_h = static_cast<T>(d.inv_h);
  s.xmax = static_cast<T>(d.xmax);
  s.h = static_cast<T>(d.h);
  s.x0d = d.x0;
  s.hd = d.h;
  s.n = d.n;
  s.seg0 = d.seg0;
  s.cmap0 = d.cmap0;
  s.kind = d.kind;
}

// Closed gate [x0, x_{n-1}] (force_calculator_concept.hpp:94-98).
template <class T> __device__ __forceinline__ bool in_span(const STab<T> &tb, T r) {
  return r >= tb.x0 && r <= tb.xmax;
}

// Extended segment of r and its local coordinate t = (r - origin)/h, with the
// reference's branch order (spline.cpp:215-252): r <= x0 → lower linear,
// r >= x_{n-1} → upper linear, else the interval of upper_bound − 1
// (spline.cpp:18-30).  In FP64 the interval is corrected against the exact
// knots x_k = x0 + k·h so that a distance exactly on a knot lands in the
// same interval as the reference.
template <class T> __device__ __forceinline__ int seg_of(const STab<T> &tb, T r, T &t) {
  if (r <= tb.x0) {
    t = (r - tb.x0) * tb.inv_h;
    return tb.seg0;
  }
  if (r >= tb.xmax) {
    t = (r - tb.xmax) * tb.inv_h;
    return tb.seg0 + tb.n;
  }
  if constexpr (std::is_same_v<T, double>) {
    int i = static_cast<int>((r - tb.x0d) * (1.0 / tb.hd));
    i = min(max(i, 0), tb.n - 2);
    while (i < tb.n - 2 && r >= __dadd_rn(tb.x0d, __dmul_rn(static_cast<double>(i + 1), tb.hd))) ++i;
    while (i > 0 && r < __dadd_rn(tb.x0d, __dmul_rn(static_cast<double>(i), tb.hd))) --i;
    const double xi = __dadd_rn(tb.x0d, __dmul_rn(static_cast<double>(i), tb.hd));
    t = (r - xi) / tb.hd;
    return tb.seg0 + 1 + i;
  } else {
    const T u = (r - tb.x0) * tb.inv_h;
    int i = static_cast<int>(u);
    i = min(max(i, 0), tb.n - 2);
    t = u - static_cast<T>(i);
    return tb.seg0 + 1 + i;
  }
}

template <class T> struct Vec4T;
template <> struct Vec4T<float> { using type = float4; };
template <> struct Vec4T<double> { using type = double4; };

template <class T>
__device__ __forceinline__ T seg_val(const typename Vec4T<T>::type &a, T t) {
  return a.x + t * (a.y + t * (a.z + t * a.w));
}
template <class T>
__device__ __forceinline__ T seg_der(const typename Vec4T<T>::type &a, T t, T inv_h) {
  return (a.y + t * (T(2) * a.z + T(3) * t * a.w)) * inv_h;
}
template <class T>
__device__ __forceinline__ T seg_der2(const typename Vec4T<T>::type &a, T t, T inv_h) {
  return (T(2) * a.z + T(6) * t * a.w) * inv_h * inv_h;
}

// pair_ordinal (include/forcesmith/force/potential_table.hpp:31-37)
__device__ __forceinline__ int pair_ord(int a, int b, int nt) {
  if (a > b) {
    const int t = a;
    a = b;
    b = t;
  }
  return a * nt - a * (a - 1) / 2 + (b - a);
}

template <class T> __device__ __forceinline__ T warp_sum_group(T v, int lpa) {
  for (int o = lpa >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < nw; ++k) s += red[k];
  return s; // valid on thread 0
}

} // namespace fsg
