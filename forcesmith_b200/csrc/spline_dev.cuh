// Device-side spline evaluation shared by the evaluation kernels.
#pragma once

#include "forms_dev.cuh"
#include "internal.cuh"

#include <type_traits>

namespace fsg {

// Compact per-table record staged in shared memory.
template <class T> struct STab {
  T x0, inv_h, xmax, h;
  double x0d, hd; // FP64 grid for the exact interval search
  double xmaxd;   // FP64 upper gate bound
  double inv_hd;  // FP64 1/h
  // Gate bands of the working precision: r in (lo_in, hi_in) is inside the
  // gate, r below lo_out or above hi_out is outside it, and a distance
  // between is decided from its FP64 length (gate_seg below).
  T lo_in, hi_in, lo_out, hi_out;
  int n, seg0, cmap0, kind;
  int form, pv0; // analytic tables: fs_form and first parameter in the value array
};

// Relative width of the band around a gate bound inside which a length
// computed in FP32 (from an FP64 pair vector rounded per component) may fall
// on the other side of the bound than the FP64 length: a few FP32 ulps.
constexpr double kGateBand = 4e-6;

template <class T> __device__ __forceinline__ void load_stab(STab<T> &s, const TableDesc &d) {
  s.x0 = static_cast<T>(d.x0);
  s.inv_h = static_cast<T>(d.inv_h);
  s.xmax = static_cast<T>(d.xmax);
  s.h = static_cast<T>(d.h);
  s.x0d = d.x0;
  s.hd = d.h;
  s.xmaxd = d.xmax;
  s.inv_hd = d.inv_h;
  const double b0 = kGateBand * fabs(d.x0), b1 = kGateBand * fabs(d.xmax);
  s.lo_in = static_cast<T>(d.x0 + b0);
  s.lo_out = static_cast<T>(d.x0 - b0);
  s.hi_in = static_cast<T>(d.xmax - b1);
  s.hi_out = static_cast<T>(d.xmax + b1);
  s.n = d.n;
  s.seg0 = d.seg0;
  s.cmap0 = d.cmap0;
  s.kind = d.kind;
  s.form = d.form;
  s.pv0 = d.pv0;
}

// Analytic radial forms: value and d/dr at r (forms_dev.cuh).  rmax is the
// table's upper gate bound.
template <class T> struct VD {
  T v, d;
};
template <class T> __device__ __forceinline__ VD<T> form_vd(int form, const double *pp, int n, T r, T rmax) {
  if (form_outside<T>(form, pp, r)) return VD<T>{T(0), T(0)};
  const Hd<T> f = form_seeded<T>(form, pp, n, r, rmax, T(0), -1);
  return VD<T>{f.a, f.b};
}

// form_vd out of line, for the table helpers below that kernels taking both
// spline and analytic tables call at every pair: the 34 forms' code then
// stays out of those kernels' register allocation (a call only where a table
// is analytic).
template <class T> __device__ __noinline__ VD<T> form_vd_call(int form, const double *pp, int n, T r, T rmax) {
  return form_vd<T>(form, pp, n, r, rmax);
}

// Closed gate [x0, x_{n-1}] (force_calculator_concept.hpp:94-98), for
// values that are not pair distances (ρ against the embedding span).
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

// Gate and segment of a pair distance whose FP64 length r64 is at hand (the
// residual and population kernels).  The gate and the branch are decided in
// FP64, as the FP64 path decides them; in FP32 the local coordinate
// t = (r − x_e)/h is also formed in FP64 and then rounded, which keeps t
// accurate to an FP32 ulp of t rather than of r/h: on the steep repulsive
// wall of a pair table (φ'' of a few hundred eV/Å²) an FP32 r alone would
// put ~1e-5 eV/Å into each pair force.
template <bool CLOSED = true, class T> __device__ __forceinline__ bool gate64(const STab<T> &tb, double r64) {
  return CLOSED ? (r64 >= tb.x0d && r64 <= tb.xmaxd) : (r64 >= tb.x0d && r64 < tb.xmaxd);
}
template <class T> __device__ __forceinline__ int seg_of64(const STab<T> &tb, T r, double r64, T &t) {
  if constexpr (std::is_same_v<T, double>) {
    return seg_of(tb, r, t);
  } else {
    if (r64 <= tb.x0d) {
      t = static_cast<T>((r64 - tb.x0d) * tb.inv_hd);
      return tb.seg0;
    }
    if (r64 >= tb.xmaxd) {
      t = static_cast<T>((r64 - tb.xmaxd) * tb.inv_hd);
      return tb.seg0 + tb.n;
    }
    const double u = (r64 - tb.x0d) * tb.inv_hd;
    int i = static_cast<int>(u);
    i = min(max(i, 0), tb.n - 2);
    t = static_cast<T>(u - static_cast<double>(i));
    return tb.seg0 + 1 + i;
  }
}

// Gate and segment of a pair distance in one step, for kernels without the
// FP64 length at hand: the extended segment of r (and t), or −1 when r is
// outside the gate (closed [x0, x_{n-1}] for EAM, ADP and angular radial
// tables, force_calculator_concept.hpp:94-118; half-open [x0, x_{n-1}) for
// the pair calculator when !CLOSED, pair_force.cpp:28).  An FP32 distance
// carries a few ulps of rounding, so one within kGateBand of either end is
// decided by its FP64 length r64(): the gate as the FP64 path decides it,
// and the branch too, since the reference's derivative jumps at both end
// knots (makima end slope inside, the end interval's secant slope outside,
// spline.cpp:236-241).  Distances away from the ends take the direct path.
// Outside the gate t is set to 0.
template <bool CLOSED, class T, class R64>
__device__ __noinline__ int gate_seg_edge(const STab<T> &tb, T r, T &t, R64 r64) {
  t = T(0);
  if (r < tb.lo_out || r > tb.hi_out) return -1;
  const double q = r64();
  if (q < tb.x0d || (CLOSED ? q > tb.xmaxd : q >= tb.xmaxd)) return -1;
  if (q <= tb.x0d) {
    t = (r - tb.x0) * tb.inv_h;
    return tb.seg0;
  }
  if (q >= tb.xmaxd) {
    t = (r - tb.xmax) * tb.inv_h;
    return tb.seg0 + tb.n;
  }
  const T u = (r - tb.x0) * tb.inv_h;
  int i = static_cast<int>(u);
  i = min(max(i, 0), tb.n - 2);
  t = u - static_cast<T>(i);
  return tb.seg0 + 1 + i;
}

template <bool CLOSED = true, class T, class R64>
__device__ __forceinline__ int gate_seg(const STab<T> &tb, T r, T &t, R64 &&r64) {
  if constexpr (std::is_same_v<T, double>) {
    if (!(CLOSED ? (r >= tb.x0 && r <= tb.xmax) : (r >= tb.x0 && r < tb.xmax))) {
      t = T(0);
      return -1;
    }
    return seg_of(tb, r, t);
  } else {
    if (r > tb.lo_in && r < tb.hi_in) {
      const T u = (r - tb.x0) * tb.inv_h;
      int i = static_cast<int>(u);
      i = min(max(i, 0), tb.n - 2);
      t = u - static_cast<T>(i);
      return tb.seg0 + 1 + i;
    }
    return gate_seg_edge<CLOSED>(tb, r, t, r64);
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
    if (tb.kind == FS_TABLE_ANALYTIC) return form_vd_call<T>(tb.form, vals + tb.pv0, tb.n, r, tb.xmax);
  }
  T t;
  const int e = seg_of(tb, r, t);
  return VD<T>{seg_val<T>(seg[e], t), seg_der<T>(seg[e], t, tb.inv_h)};
}

// tab_vd at a pair distance with its FP64 length (seg_of64).
template <class T, bool AN>
__device__ __forceinline__ VD<T> tab_vd64(const STab<T> &tb, const typename Vec4T<T>::type *seg, const double *vals,
                                          T r, double r64) {
  if constexpr (AN) {
    if (tb.kind == FS_TABLE_ANALYTIC) return form_vd_call<T>(tb.form, vals + tb.pv0, tb.n, r, tb.xmax);
  }
  T t;
  const int e = seg_of64(tb, r, r64, t);
  return VD<T>{seg_val<T>(seg[e], t), seg_der<T>(seg[e], t, tb.inv_h)};
}

// Value and d/dr at r from gate_seg's segment e and t (analytic tables,
// when AN, from their closed form).
template <class T, bool AN>
__device__ __forceinline__ VD<T> tab_vd_at(const STab<T> &tb, const typename Vec4T<T>::type *seg,
                                           const double *vals, T r, int e, T t) {
  if constexpr (AN) {
    if (tb.kind == FS_TABLE_ANALYTIC) return form_vd_call<T>(tb.form, vals + tb.pv0, tb.n, r, tb.xmax);
  }
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
