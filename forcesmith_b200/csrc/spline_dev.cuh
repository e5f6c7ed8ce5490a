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
  int form, pv0; // analytic tables: fs_form and first parameter in the value array
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
  s.form = d.form;
  s.pv0 = d.pv0;
}

// Analytic radial forms (include/forcesmith/potentials/analytic_potential.hpp),
// value and d/dr, parameters p[] as in the header's fs_form list.
template <class T> struct VD {
  T v, d;
};
template <class T> __device__ __forceinline__ VD<T> form_vd(int form, const double *pp, int n, T r) {
  T p[5];
  for (int k = 0; k < 5; ++k) p[k] = k < n ? static_cast<T>(pp[k]) : T(0);
  VD<T> o{T(0), T(0)};
  switch (form) {
  case 0: { // LJ 4ε((σ/r)^12 − (σ/r)^6)
    const T sr = p[1] / r, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2;
    o.v = T(4) * p[0] * (sr6 * sr6 - sr6);
    o.d = T(4) * p[0] * (T(-12) * sr6 * sr6 + T(6) * sr6) / r;
    break;
  }
  case 1: { // Morse De(1 − e^{−a(r−re)})² − De
    const T e = exp(-p[1] * (r - p[2]));
    o.v = p[0] * (T(1) - e) * (T(1) - e) - p[0];
    o.d = T(2) * p[0] * (T(1) - e) * p[1] * e;
    break;
  }
  case 2: { // A e^{−Br}
    o.v = p[0] * exp(-p[1] * r);
    o.d = -p[1] * o.v;
    break;
  }
  case 3: { // A √(r/B)
    o.v = p[0] * sqrt(r / p[1]);
    o.d = o.v / (T(2) * r);
    break;
  }
  case 4: { // A / r^n
    o.v = p[0] / pow(r, p[1]);
    o.d = -p[1] * o.v / r;
    break;
  }
  case 5: { // A e^{−B(r−r0)}
    o.v = p[0] * exp(-p[1] * (r - p[2]));
    o.d = -p[1] * o.v;
    break;
  }
  case 6: { // k (r − r0)²
    o.v = p[0] * (r - p[1]) * (r - p[1]);
    o.d = T(2) * p[0] * (r - p[1]);
    break;
  }
  case 7: { // A e^{−Br} + C
    const T e = p[0] * exp(-p[1] * r);
    o.v = e + p[2];
    o.d = -p[1] * e;
    break;
  }
  case 8: { // A r² + B r + C
    o.v = p[0] * r * r + p[1] * r + p[2];
    o.d = T(2) * p[0] * r + p[1];
    break;
  }
  case 9: { // C
    o.v = p[0];
    break;
  }
  case 10: { // A e^{−r/ρ} − C (ρ²/r²)³
    const T x = (p[1] * p[1]) / (r * r), e = p[0] * exp(-r / p[1]);
    o.v = e - p[2] * x * x * x;
    o.d = -e / p[1] + T(6) * p[2] * x * x * x / r;
    break;
  }
  case 11: { // A e^{(C−r)/B} − D/r⁶ + E/r⁸
    const T r2 = r * r, r6 = r2 * r2 * r2, e = p[0] * exp((p[2] - r) / p[1]);
    o.v = e - p[3] / r6 + p[4] / (r6 * r2);
    o.d = -e / p[1] + T(6) * p[3] / (r6 * r) - T(8) * p[4] / (r6 * r2 * r);
    break;
  }
  }
  return o;
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

// Value and d/dr of a table at r (inside its gate): the makima segment, or,
// when AN and the table is analytic, its closed form.
template <class T, bool AN>
__device__ __forceinline__ VD<T> tab_vd(const STab<T> &tb, const typename Vec4T<T>::type *seg, const double *vals,
                                        T r) {
  if constexpr (AN) {
    if (tb.kind == FS_TABLE_ANALYTIC) return form_vd<T>(tb.form, vals + tb.pv0, tb.n, r);
  }
  T t;
  const int e = seg_of(tb, r, t);
  return VD<T>{seg_val<T>(seg[e], t), seg_der<T>(seg[e], t, tb.inv_h)};
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
