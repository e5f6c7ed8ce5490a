// Stillinger–Weber on the device: residual and analytic parameter Jacobian.
//
//   StiwebForceCalculator::eval_forces (src/force/stiweb_force.cpp:241-271):
//     2-body v₂ = (A r⁻ᵖ − B r⁻ᵠ)·exp(δ/(r − a1)) for r < a1 (v2_dv2, :24-41),
//     ½ v₂ per directed pair (accumulate_pair, kernels.hpp:33-38);
//     3-body per central atom i and neighbour pair jj < kk:
//     h(r1) h(r2) λ_{i;jk} (cos θ + ⅓)² with h = exp(γ/(r − a2)) (h_dh,
//     :43-54; add_angular :138-144; three_body_forces kernels.hpp:44-58;
//     accumulate_triplet :60-68).
//   The reference has no analytic SW Jacobian (its Jacobian is central
//   differences); here every partial ∂/∂{A,B,p,q,δ,a1,γ,a2,λ} is carried
//   exactly by forward-mode dual numbers through the same expressions.
//
// One CTA per configuration.  A block scan lays out the configuration's work
// items, and threads take them flat: first one directed pair each (2-body),
// then one neighbour pair (j < k) of a central atom each (3-body), so atoms
// with few or many neighbours cost the same lanes.  Forces and the Jacobian
// block of the configuration ((3N + rows) × D, D = the few free SW parameters)
// accumulate in shared memory with atomics, then stream out; the energy and
// stress rows, which every item hits, are summed in registers first.
#include "kern_common.cuh"

#include <algorithm>

namespace fsg {
namespace {

// Reciprocal, exp and log: the hardware approximations in FP32 (a few ulp,
// inside the FP32 path's stated tolerances), IEEE in FP64.
__device__ __forceinline__ float rcp_t(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double rcp_t(double x) { return 1.0 / x; }
__device__ __forceinline__ float exp_t(float x) { return __expf(x); }
__device__ __forceinline__ double exp_t(double x) { return exp(x); }
__device__ __forceinline__ float log_t(float x) { return __logf(x); }
__device__ __forceinline__ double log_t(double x) { return log(x); }

template <class T, int N> struct Dual {
  T v;
  T d[N];
  __device__ Dual() : v(0) {
#pragma unroll
    for (int k = 0; k < N; ++k) d[k] = T(0);
  }
  __device__ explicit Dual(T x) : v(x) {
#pragma unroll
    for (int k = 0; k < N; ++k) d[k] = T(0);
  }
  __device__ static Dual var(T x, int k) {
    Dual r(x);
    if (k >= 0) r.d[k] = T(1);
    return r;
  }
};
template <class T, int N> __device__ Dual<T, N> operator+(const Dual<T, N> &a, const Dual<T, N> &b) {
  Dual<T, N> r(a.v + b.v);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <class T, int N> __device__ Dual<T, N> operator-(const Dual<T, N> &a, const Dual<T, N> &b) {
  Dual<T, N> r(a.v - b.v);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <class T, int N> __device__ Dual<T, N> operator*(const Dual<T, N> &a, const Dual<T, N> &b) {
  Dual<T, N> r(a.v * b.v);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <class T, int N> __device__ Dual<T, N> operator*(T s, const Dual<T, N> &a) {
  Dual<T, N> r(s * a.v);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
  return r;
}
template <class T, int N> __device__ Dual<T, N> operator/(const Dual<T, N> &a, const Dual<T, N> &b) {
  const T ib = rcp_t(b.v);
  Dual<T, N> r(a.v * ib);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
template <class T, int N> __device__ Dual<T, N> dexp(const Dual<T, N> &a) {
  Dual<T, N> r(exp_t(a.v));
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = r.v * a.d[k];
  return r;
}

// v₂ and dv₂/dr (stiweb_force.cpp:24-41) with partials over the 6 two-body
// parameters (A, B, p, q, δ, a1) of the pair slot.
template <class T>
__device__ void v2_dual(T r, const T *P, Dual<T, 6> &v2, Dual<T, 6> &dv2) {
  v2 = Dual<T, 6>();
  dv2 = Dual<T, 6>();
  if (r >= P[5]) return;
  using D6 = Dual<T, 6>;
  const D6 A = D6::var(P[0], 0), B = D6::var(P[1], 1), p = D6::var(P[2], 2), q = D6::var(P[3], 3);
  const D6 delta = D6::var(P[4], 4), a1 = D6::var(P[5], 5);
  const D6 rr(r);
  const D6 d = rr - a1;
  const D6 e = dexp(delta / d);
  if (e.v == T(0)) return;
  const T lr = log_t(r);
  const D6 rp = dexp(T(-1) * (p * D6(lr)));
  const D6 rq = dexp(T(-1) * (q * D6(lr)));
  const D6 rp1 = rp / rr, rq1 = rq / rr; // r^{-p-1}, r^{-q-1}
  const D6 poly = A * rp - B * rq;
  const D6 dpoly = T(-1) * (A * p * rp1) + B * q * rq1;
  v2 = poly * e;
  dv2 = dpoly * e + poly * e * (T(-1) * (delta / (d * d)));
}

template <class T> __device__ void v2_plain(T r, const T *P, T &v2, T &dv2) {
  v2 = dv2 = T(0);
  if (r >= P[5]) return;
  const T d = r - P[5];
  const T e = exp(P[4] / d);
  if (e == T(0)) return;
  const T rp = pow(r, -P[2]), rq = pow(r, -P[3]);
  const T poly = P[0] * rp - P[1] * rq;
  const T dpoly = -P[0] * P[2] * pow(r, -P[2] - T(1)) + P[1] * P[3] * pow(r, -P[3] - T(1));
  v2 = poly * e;
  dv2 = dpoly * e + poly * e * (-P[4] / (d * d));
}

// h and dh/dr (stiweb_force.cpp:43-54) with partials over (γ, a2) placed at
// dual slots kg, ka.
template <class T, int N>
__device__ void h_dual(T r, T gamma, T a2, int kg, int ka, Dual<T, N> &h, Dual<T, N> &dh) {
  h = Dual<T, N>();
  dh = Dual<T, N>();
  if (r >= a2) return;
  using DN = Dual<T, N>;
  const DN g = DN::var(gamma, kg), a = DN::var(a2, ka);
  const DN d = DN(r) - a;
  h = dexp(g / d);
  if (h.v == T(0)) {
    h = DN();
    return;
  }
  dh = h * (T(-1) * (g / (d * d)));
}

template <class T> struct SwArgs {
  Common c;
  const double *vals;  // all model values (FP64)
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
  // Jacobian (nullptr: residual only)
  T *J;
  int64_t ld;
  int D;
  double *jtr_part;
  const int32_t *order; // configurations by work, heaviest first (CTA b runs order[b])
  int use_own;          // work-item owner table in shared memory (else binary search)
};

constexpr int kSwThreads = 256;
constexpr int kSwChunk = 4; // consecutive 2-body and 3-body items per thread


template <class T>
__device__ __forceinline__ void add_row(T *Jb, int D, int row, int col, T v) {
  if (col >= 0 && v != T(0)) atomicAdd(&Jb[row * D + col], v); // the block is < 227 KB: int offsets
}

// The energy and six stress rows of the Jacobian block for NQ dual slots,
// summed in registers while a thread's consecutive work items map their slots
// to the same columns, and added to shared memory when the columns change
// (with one species: once, at the end of the phase).
template <class T, int NQ> struct RowAcc {
  T a[NQ][7];
  int col[NQ];
  __device__ RowAcc() {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      col[q] = -1;
#pragma unroll
      for (int r = 0; r < 7; ++r) a[q][r] = T(0);
    }
  }
  __device__ __forceinline__ void flush(T *Jb, int D, int rowE) {
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
      for (int r = 0; r < 7; ++r) {
        add_row(Jb, D, rowE + r, col[q], a[q][r]);
        a[q][r] = T(0);
      }
  }
  __device__ __forceinline__ void use(const int (&cols)[NQ], T *Jb, int D, int rowE) {
    bool same = true;
#pragma unroll
    for (int q = 0; q < NQ; ++q) same &= cols[q] == col[q];
    if (!same) {
      flush(Jb, D, rowE);
#pragma unroll
      for (int q = 0; q < NQ; ++q) col[q] = cols[q];
    }
  }
};


// The force and Jacobian rows of one central atom i, summed in registers over
// a thread's consecutive work items while i and the items' columns stay the
// same, and added to shared memory when they change.
template <class T, int NQ, bool JAC> struct AtomAcc {
  T f[3];
  T g[NQ][3];
  int col[NQ];
  int i = -1;
  __device__ AtomAcc() {
#pragma unroll
    for (int a = 0; a < 3; ++a) f[a] = T(0);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      col[q] = -1;
      g[q][0] = g[q][1] = g[q][2] = T(0);
    }
  }
  __device__ __forceinline__ void flush(T *Fs, T *Jb, int D) {
    if (i < 0) return;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicAdd(&Fs[3 * i + a], f[a]);
      f[a] = T(0);
    }
    if constexpr (JAC)
#pragma unroll
      for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          add_row(Jb, D, 3 * i + a, col[q], g[q][a]);
          g[q][a] = T(0);
        }
    i = -1;
  }
  // start summing for atom ii with columns cols (flushing what was summed)
  __device__ __forceinline__ void use(int ii, const int (&cols)[NQ], T *Fs, T *Jb, int D) {
    bool same = ii == i;
    if constexpr (JAC)
#pragma unroll
      for (int q = 0; q < NQ; ++q) same = same && cols[q] == col[q];
    if (!same) {
      flush(Fs, Jb, D);
      i = ii;
#pragma unroll
      for (int q = 0; q < NQ; ++q) col[q] = cols[q];
    }
  }
};

template <class T, bool JAC>
__global__ void __launch_bounds__(kSwThreads, sizeof(T) == 4 ? 2 : 1) sw_kernel(SwArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = A.order ? A.order[blockIdx.x] : blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  const int D = JAC ? A.D : 0;
  Smem S(smem_raw);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  T *Fs = S.take<T>(3 * N);
  T *par = S.take<T>(8 * np);
  T *lam = S.take<T>(nt * np);
  int *pcol = S.take<int>(8 * np);
  int *lcol = S.take<int>(nt * np);
  double *red = S.take<double>(8 * 32);
  int *pfirst = S.take<int>(N + 1);
  int *tfirst = S.take<int>(N + 1);
  int *wsum = S.take<int>(32);
  T *Jb = JAC ? S.take<T>(static_cast<size_t>(3 * N + 7) * D) : nullptr; // force rows, E, 6 stress
  double *jpart = JAC ? S.take<double>(static_cast<size_t>(D) * (blockDim.x >> 5)) : nullptr;
  for (int k = threadIdx.x; k < 8 * np; k += blockDim.x) {
    const TableDesc &td = A.c.desc[k / 8];
    par[k] = static_cast<T>(A.vals[td.pv0 + k % 8]);
    pcol[k] = A.c.cmap[td.cmap0 + k % 8];
  }
  for (int k = threadIdx.x; k < nt * np; k += blockDim.x) {
    const TableDesc &td = A.c.desc[np];
    lam[k] = static_cast<T>(A.vals[td.pv0 + k]);
    lcol[k] = A.c.cmap[td.cmap0 + k];
  }
  for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) Fs[k] = T(0);
  if constexpr (JAC)
    for (int k = threadIdx.x; k < (3 * N + 7) * D; k += blockDim.x) Jb[k] = T(0);
  stage_geometry(cd, A.c, wpos, shift, typ);
  const int32_t *start = A.c.nb_start + cd.atom0;
  stage_work(start, N, pfirst, tfirst, wsum);
  __syncthreads();
  const uint32_t *nbp = A.c.nb_pack + start[0];
  const int npair = pfirst[N], ntri = tfirst[N];
  // owner of each work item: pair p → i; neighbour pair t → (row a << 16) | i,
  // row a = index of j in i's list (N and the row below 2^16, checked at launch)
  uint32_t *own = nullptr;
  if (A.use_own) {
    own = S.take<uint32_t>(npair + ntri);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const int p0 = pfirst[i], n = pfirst[i + 1] - p0;
      for (int q = 0; q < n; ++q) own[p0 + q] = static_cast<uint32_t>(i);
      uint32_t *ot = own + npair + tfirst[i];
      for (int a = 0; a + 1 < n; ++a)
        for (int b = a + 1; b < n; ++b) *ot++ = (static_cast<uint32_t>(a) << 16) | static_cast<uint32_t>(i);
    }
    __syncthreads();
  }
  double e_acc = 0.0, sg[6] = {0, 0, 0, 0, 0, 0};
  const int rowE = 3 * N; // local rows of the block: 3N force, E, 6 stress
  // ---- 2-body: one thread per directed pair (½ v₂ each, force on i).  A
  // thread takes kSwChunk consecutive pairs, which mostly share atom i.
  {
    RowAcc<T, JAC ? 6 : 1> ra;
    AtomAcc<T, JAC ? 6 : 1, JAC> ia;
    for (int w0 = threadIdx.x * kSwChunk; w0 < npair; w0 += blockDim.x * kSwChunk) {
    const int w1 = min(w0 + kSwChunk, npair);
    for (int w = w0; w < w1; ++w) {
      const int i = own ? static_cast<int>(own[w]) : owner_of(pfirst, N, w);
      int j;
      T d[3];
      pair_vec(wpos, shift, i, nbp[w], j, d[0], d[1], d[2]);
      const T r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r < T(1e-14)) continue;
      const int sl = pair_ord(typ[i], typ[j], nt);
      const T *P = par + 8 * sl;
      T v2v, s;
      Dual<T, 6> v2, dv2;
      if constexpr (JAC) {
        v2_dual(r, P, v2, dv2);
        v2v = v2.v;
        s = dv2.v / r;
      } else {
        T dv2p;
        v2_plain(r, P, v2v, dv2p);
        s = dv2p / r;
      }
      const T f[3] = {s * d[0], s * d[1], s * d[2]};
      if constexpr (!JAC) {
        const int nocol[1] = {-1};
        ia.use(i, nocol, Fs, Jb, D);
#pragma unroll
        for (int a = 0; a < 3; ++a) ia.f[a] += f[a];
      }
      e_acc += 0.5 * static_cast<double>(v2v);
      const T hx = T(0.5) * d[0], hy = T(0.5) * d[1], hz = T(0.5) * d[2];
      sg[0] -= hx * f[0];
      sg[1] -= hy * f[1];
      sg[2] -= hz * f[2];
      sg[3] -= hx * f[1];
      sg[4] -= hx * f[2];
      sg[5] -= hy * f[2];
      if constexpr (JAC) {
        int cols[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) cols[k] = pcol[8 * sl + k];
        ra.use(cols, Jb, D, rowE);
        ia.use(i, cols, Fs, Jb, D);
#pragma unroll
        for (int a = 0; a < 3; ++a) ia.f[a] += f[a];
        const T we = static_cast<T>(0.5 * A.w_e), ir = rcp_t(r);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          const T ds = dv2.d[k] * ir;
          const T df[3] = {ds * d[0], ds * d[1], ds * d[2]};
#pragma unroll
          for (int a = 0; a < 3; ++a) ia.g[k][a] += df[a];
          ra.a[k][0] += we * v2.d[k];
          ra.a[k][1] -= hx * df[0];
          ra.a[k][2] -= hy * df[1];
          ra.a[k][3] -= hz * df[2];
          ra.a[k][4] -= hx * df[1];
          ra.a[k][5] -= hx * df[2];
          ra.a[k][6] -= hy * df[2];
        }
      }
    }
    ia.flush(Fs, Jb, D);
    }
    if constexpr (JAC) ra.flush(Jb, D, rowE);
  }
  // ---- 3-body: one thread per neighbour pair (j < k) of a central atom i.
  // A thread takes kSwChunk consecutive items, which mostly share their
  // central atom i (its force and Jacobian rows go through AtomAcc).
  {
    RowAcc<T, JAC ? 5 : 1> rb;
    AtomAcc<T, JAC ? 5 : 1, JAC> ia;
    for (int w0 = threadIdx.x * kSwChunk; w0 < ntri; w0 += blockDim.x * kSwChunk) {
    const int w1 = min(w0 + kSwChunk, ntri);
    for (int w = w0; w < w1; ++w) {
      int i, a0, u;
      if (own) {
        const uint32_t v = own[npair + w];
        i = static_cast<int>(v & 0xFFFFu);
        a0 = static_cast<int>(v >> 16);
        const int n = pfirst[i + 1] - pfirst[i];
        u = w - tfirst[i] - a0 * (2 * n - a0 - 1) / 2; // row a0 starts after Σ_{a<a0} (n − 1 − a)
      } else {
        i = owner_of(tfirst, N, w);
        const int n = pfirst[i + 1] - pfirst[i];
        u = w - tfirst[i];
        pair_row(n, u, a0);
      }
      const int pj = pfirst[i] + a0, pk = pj + 1 + u;
      const int ti = typ[i];
      int j;
      T d1[3];
      pair_vec(wpos, shift, i, nbp[pj], j, d1[0], d1[1], d1[2]);
      const T r1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
      if (r1 < T(1e-14)) continue;
      const int tj = typ[j];
      const int s1 = pair_ord(ti, tj, nt);
      Dual<T, 5> h1, dh1;
      h_dual<T, 5>(r1, par[8 * s1 + 6], par[8 * s1 + 7], 0, 1, h1, dh1);
      if (h1.v == T(0) && dh1.v == T(0)) continue; // make_jbond (stiweb_force.cpp:107-121)
      int k;
      T d2[3];
      pair_vec(wpos, shift, i, nbp[pk], k, d2[0], d2[1], d2[2]);
      const T r2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
      if (r2 < T(1e-14)) continue;
      const int tk = typ[k];
      const int s2 = pair_ord(ti, tk, nt);
      Dual<T, 5> h2, dh2;
      h_dual<T, 5>(r2, par[8 * s2 + 6], par[8 * s2 + 7], 2, 3, h2, dh2);
      if (h2.v == T(0) && dh2.v == T(0)) continue;
      const T ir1 = rcp_t(r1), ir2 = rcp_t(r2);
      const int lt = ti * np + pair_ord(tj, tk, nt);
      const Dual<T, 5> L = Dual<T, 5>::var(lam[lt], 4);
      const T cth = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) * ir1 * ir2;
      const T cp = cth + T(1) / T(3);
      const Dual<T, 5> wg = (cp * cp) * L, dw = (T(2) * cp) * L;
      // three_body_forces (kernels.hpp:44-58)
      const T irr = ir1 * ir2;
      Dual<T, 5> c1 = (ir1 * dh1) * h2 * wg; // df1·inv_r1·f2·g
      Dual<T, 5> c2 = h1 * (ir2 * dh2) * wg; // f1·df2·inv_r2·g
      Dual<T, 5> c3 = h1 * h2 * dw;          // f1·f2·dg
      Dual<T, 5> e3 = h1 * h2 * wg;
      T Fi[3], Fj[3], Fk[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        Fj[a] = -(c1.v * d1[a]) - c3.v * (irr * d2[a] - cth * ir1 * ir1 * d1[a]);
        Fk[a] = -(c2.v * d2[a]) - c3.v * (irr * d1[a] - cth * ir2 * ir2 * d2[a]);
        Fi[a] = -(Fj[a] + Fk[a]); // the three forces sum to zero
        atomicAdd(&Fs[3 * j + a], Fj[a]);
        atomicAdd(&Fs[3 * k + a], Fk[a]);
      }
      if constexpr (!JAC) {
        const int nocol[1] = {-1};
        ia.use(i, nocol, Fs, Jb, D);
#pragma unroll
        for (int a = 0; a < 3; ++a) ia.f[a] += Fi[a];
      }
      e_acc += static_cast<double>(e3.v);
      sg[0] += d1[0] * Fj[0] + d2[0] * Fk[0];
      sg[1] += d1[1] * Fj[1] + d2[1] * Fk[1];
      sg[2] += d1[2] * Fj[2] + d2[2] * Fk[2];
      sg[3] += d1[0] * Fj[1] + d2[0] * Fk[1];
      sg[4] += d1[0] * Fj[2] + d2[0] * Fk[2];
      sg[5] += d1[1] * Fj[2] + d2[1] * Fk[2];
      if constexpr (JAC) {
        int cols[5] = {pcol[8 * s1 + 6], pcol[8 * s1 + 7], pcol[8 * s2 + 6], pcol[8 * s2 + 7], lcol[lt]};
        // both ends in the same pair slot: one column each for γ and a2
#pragma unroll
        for (int q = 2; q < 4; ++q)
          if (cols[q] == cols[q - 2]) {
            c1.d[q - 2] += c1.d[q];
            c2.d[q - 2] += c2.d[q];
            c3.d[q - 2] += c3.d[q];
            e3.d[q - 2] += e3.d[q];
            cols[q] = -1;
          }
        rb.use(cols, Jb, D, rowE);
        ia.use(i, cols, Fs, Jb, D);
#pragma unroll
        for (int a = 0; a < 3; ++a) ia.f[a] += Fi[a];
        const T we = static_cast<T>(A.w_e);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          T gj[3], gk[3];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            gj[a] = -(c1.d[q] * d1[a]) - c3.d[q] * (irr * d2[a] - cth * ir1 * ir1 * d1[a]);
            gk[a] = -(c2.d[q] * d2[a]) - c3.d[q] * (irr * d1[a] - cth * ir2 * ir2 * d2[a]);
            ia.g[q][a] -= gj[a] + gk[a];
            add_row(Jb, D, 3 * j + a, cols[q], gj[a]);
            add_row(Jb, D, 3 * k + a, cols[q], gk[a]);
          }
          rb.a[q][0] += we * e3.d[q];
          rb.a[q][1] += d1[0] * gj[0] + d2[0] * gk[0];
          rb.a[q][2] += d1[1] * gj[1] + d2[1] * gk[1];
          rb.a[q][3] += d1[2] * gj[2] + d2[2] * gk[2];
          rb.a[q][4] += d1[0] * gj[1] + d2[0] * gk[1];
          rb.a[q][5] += d1[0] * gj[2] + d2[0] * gk[2];
          rb.a[q][6] += d1[1] * gj[2] + d2[1] * gk[2];
        }
      }
    }
    ia.flush(Fs, Jb, D);
    }
    if constexpr (JAC) rb.flush(Jb, D, rowE);
  }
  __syncthreads();
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  double objp = 0.0;
  for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) {
    const int64_t ga = static_cast<int64_t>(cd.atom0) * 3 + k;
    const double f = static_cast<double>(Fs[k]);
    const double res = f - A.c.ref_force[ga];
    A.F[row0 + k] = res;
    if (A.forces) A.forces[ga] = f;
    objp += res * res;
  }
  double sums[8] = {e_acc, sg[0], sg[1], sg[2], sg[3], sg[4], sg[5], objp};
  block_sum_k(sums, red);
  if (threadIdx.x == 0) {
    const double E = sums[0];
    double st[6];
    const double iv = 1.0 / cd.volume;
    for (int a = 0; a < 6; ++a) st[a] = sums[1 + a] * iv;
    int64_t row = row0 + 3 * N;
    double o = sums[7];
    const double re = A.w_e * (E - cd.ref_energy);
    A.F[row++] = re;
    o += re * re;
    static constexpr int vi[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    if (A.w_s > 0.0)
      for (int v = 0; v < 6; ++v) {
        const double rs = A.w_s * (st[v] - cd.ref_stress[3 * vi[v][0] + vi[v][1]]);
        A.F[row++] = rs;
        o += rs * rs;
      }
    A.F[row++] = 0.0; // no embedding: limit row is zero
    A.obj_part[c] = o;
    if (A.energy) A.energy[c] = E;
    if (A.limit) A.limit[c] = 0.0;
    if (A.stress9) {
      double *s9 = A.stress9 + 9 * static_cast<int64_t>(c);
      s9[0] = st[0];
      s9[4] = st[1];
      s9[8] = st[2];
      s9[1] = s9[3] = st[3];
      s9[2] = s9[6] = st[4];
      s9[5] = s9[7] = st[5];
    }
  }
  if constexpr (JAC) {
    __syncthreads();
    const double sc = A.w_s / cd.volume;
    const int nrow = 3 * N + 2 + (A.w_s > 0.0 ? 6 : 0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int col = 0; col < D; ++col) {
      double jr = 0.0;
      for (int r = threadIdx.x; r < nrow; r += blockDim.x) {
        double v;
        if (r < 3 * N)
          v = static_cast<double>(Jb[static_cast<int64_t>(r) * D + col]);
        else if (r == 3 * N)
          v = static_cast<double>(Jb[static_cast<int64_t>(rowE) * D + col]);
        else if (A.w_s > 0.0 && r < 3 * N + 7)
          v = sc * static_cast<double>(Jb[static_cast<int64_t>(rowE + (r - 3 * N)) * D + col]);
        else
          v = 0.0; // limit row
        A.J[static_cast<int64_t>(col) * A.ld + row0 + r] = static_cast<T>(v);
        jr += v * A.F[row0 + r];
      }
      for (int o = 16; o > 0; o >>= 1) jr += __shfl_xor_sync(0xffffffffu, jr, o);
      if (lane == 0) jpart[col * nw + w] = jr;
    }
    __syncthreads();
    for (int col = threadIdx.x; col < D; col += blockDim.x) {
      double jr = 0.0;
      for (int k = 0; k < nw; ++k) jr += jpart[col * nw + k];
      A.jtr_part[static_cast<int64_t>(c) * D + col] = jr;
    }
  }
}

template <class T> size_t sw_smem(fs_gpu *h, int max_img, bool jac) {
  const int nt = h->ntypes, np = npair_of(nt), N = h->max_natoms;
  size_t b = align16(3 * N * sizeof(double)) + align16(3 * max_img * sizeof(double)) + align16(N) +
             align16(3 * N * sizeof(T)) + align16(8 * np * sizeof(T)) + align16(nt * np * sizeof(T)) +
             align16(8 * np * sizeof(int)) + align16(nt * np * sizeof(int)) + align16(8 * 32 * sizeof(double)) +
             2 * align16((N + 1) * sizeof(int)) + align16(32 * sizeof(int));
  if (jac)
    b += align16(static_cast<size_t>(3 * N + 7) * h->D * sizeof(T)) +
         align16(static_cast<size_t>(h->D) * (kSwThreads / 32) * sizeof(double));
  return b + 128;
}

int max_images_of(const fs_gpu *h) {
  int m = 1;
  for (const CfgDev &cd : h->cfg_host) m = std::max(m, (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1));
  return m;
}

__global__ void sum_parts(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *out = s;
}

__global__ void sw_jtr_reduce(const double *__restrict__ part, int n_cfg, int D, double *__restrict__ Jtr) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= D) return;
  double s = 0.0;
  for (int c = 0; c < n_cfg; ++c) s += part[static_cast<int64_t>(c) * D + col];
  Jtr[col] = s;
}

template <class T> int launch_sw(fs_gpu *h, double w_e, double w_s, bool jac) {
  SwArgs<T> a;
  a.c.cfg = h->d_cfg;
  a.c.wpos = h->d_wpos;
  a.c.type = h->d_type;
  a.c.ref_force = h->d_ref_force;
  a.c.nb_start = h->d_nb_start;
  a.c.nb_pack = h->d_nb_pack;
  a.c.desc = h->d_desc;
  a.c.cmap = h->d_cmap;
  a.c.n_tables = static_cast<int>(h->desc.size());
  a.c.n_segs = h->n_segs;
  a.c.n_cmap = h->n_cmap;
  a.c.ntypes = h->ntypes;
  a.c.family = h->family;
  a.vals = h->d_vals;
  a.w_e = w_e;
  a.w_s = w_s;
  a.F = h->d_F;
  a.forces = h->d_forces;
  a.energy = h->d_energy;
  a.stress9 = h->d_stress9;
  a.limit = h->d_limit;
  a.obj_part = h->d_obj_part;
  a.J = nullptr;
  a.ld = 0;
  a.D = h->D;
  a.jtr_part = nullptr;
  if (jac) {
    const int64_t M = rows_of(h, w_s);
    const int64_t ldj = (M + 31) / 32 * 32;
    const size_t jn = static_cast<size_t>(ldj) * h->D;
    if (static_cast<size_t>(h->jac_alloc) != jn || h->ldj != ldj || !h->d_J || h->j_rowmajor) {
      if (h->d_J) cudaFree(h->d_J);
      h->d_J = nullptr;
      FS_CUDA(cudaMalloc(&h->d_J, std::max<size_t>(jn, 1) * sizeof(T)));
      FS_CUDA(cudaMemsetAsync(h->d_J, 0, std::max<size_t>(jn, 1) * sizeof(T), h->stream));
      h->jac_alloc = static_cast<int64_t>(jn);
      h->ldj = ldj;
      h->j_rowmajor = false;
    }
    if (!h->d_JtJ) {
      FS_CUDA(cudaMalloc(&h->d_JtJ, std::max(h->D * h->D, 1) * sizeof(double)));
      FS_CUDA(cudaMalloc(&h->d_Jtr, std::max(h->D, 1) * sizeof(double)));
    }
    const size_t need = static_cast<size_t>(h->n_cfg) * h->D;
    if (h->jtr_part_alloc < need || !h->d_jtr_part) {
      if (h->d_jtr_part) cudaFree(h->d_jtr_part);
      h->d_jtr_part = nullptr;
      FS_CUDA(cudaMalloc(&h->d_jtr_part, std::max<size_t>(need, 1) * sizeof(double)));
      h->jtr_part_alloc = need;
    }
    a.J = static_cast<T *>(h->d_J);
    a.ld = ldj;
    a.jtr_part = h->d_jtr_part;
  }
  size_t sm = sw_smem<T>(h, max_images_of(h), jac);
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "SW: configuration too large for shared memory");
  // the owner table when it fits (else each work item finds its atom by binary search)
  const size_t own_bytes = align16(static_cast<size_t>(h->max_cfg_work) * sizeof(uint32_t));
  a.use_own = (sm + own_bytes <= 227 * 1024 && h->max_natoms < 65536) ? 1 : 0;
  if (a.use_own) sm += own_bytes;
  a.order = h->d_cfg_by_work;
  auto k = jac ? sw_kernel<T, true> : sw_kernel<T, false>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, kSwThreads, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  sum_parts<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  if (jac) {
    sw_jtr_reduce<<<(h->D + 127) / 128, 128, 0, h->stream>>>(h->d_jtr_part, h->n_cfg, h->D, h->d_Jtr);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  return FS_OK;
}

} // namespace

int eval_residual_adp(fs_gpu *h, double w_e, double w_s);
int eval_residual_tersoff(fs_gpu *h, double w_e, double w_s);
int eval_residual_angular(fs_gpu *h, double w_e, double w_s);
int eval_residual_acsf(fs_gpu *h, double w_e, double w_s);
int eval_jacobian_acsf(fs_gpu *h, double w_e, double w_s);
int eval_residual_lmbtr(fs_gpu *h, double w_e, double w_s);
int eval_jacobian_lmbtr(fs_gpu *h, double w_e, double w_s);
int eval_jacobian_fd(fs_gpu *h, double w_e, double w_s);

int eval_residual_other(fs_gpu *h, double w_e, double w_s) {
  if (h->family == FS_FAMILY_SW)
    return h->precision == FS_PREC_FP64 ? launch_sw<double>(h, w_e, w_s, false) : launch_sw<float>(h, w_e, w_s, false);
  if (h->family == FS_FAMILY_ADP) return eval_residual_adp(h, w_e, w_s);
  if (h->family == FS_FAMILY_TERSOFF) return eval_residual_tersoff(h, w_e, w_s);
  if (h->family == FS_FAMILY_ANGULAR) return eval_residual_angular(h, w_e, w_s);
  if (h->family == FS_FAMILY_ACSF) return eval_residual_acsf(h, w_e, w_s);
  if (h->family == FS_FAMILY_LMBTR) return eval_residual_lmbtr(h, w_e, w_s);
  return set_error(h, FS_ERR_UNSUPPORTED, "residual: family not handled by this build");
}

int eval_jacobian_other(fs_gpu *h, double w_e, double w_s) {
  if (h->family == FS_FAMILY_SW) {
    mark(h, 2);
    const int rc = h->precision == FS_PREC_FP64 ? launch_sw<double>(h, w_e, w_s, true)
                                                : launch_sw<float>(h, w_e, w_s, true);
    mark(h, 3);
    return rc;
  }
  // ACSF with linear heads: exact (the model is linear in its coefficients)
  if (h->family == FS_FAMILY_ACSF) return eval_jacobian_acsf(h, w_e, w_s);
  // LMBTR with linear heads: exact, like ACSF
  if (h->family == FS_FAMILY_LMBTR) return eval_jacobian_lmbtr(h, w_e, w_s);
  // ADP: exact, forward mode (adp.cu)
  if (h->family == FS_FAMILY_ADP) {
    extern int eval_jacobian_adp(fs_gpu * h, double w_e, double w_s);
    return eval_jacobian_adp(h, w_e, w_s);
  }
  // Tersoff, Angular: the reference's own central differences (FP64 contexts)
  if (h->family == FS_FAMILY_TERSOFF || h->family == FS_FAMILY_ANGULAR) return eval_jacobian_fd(h, w_e, w_s);
  return set_error(h, FS_ERR_UNSUPPORTED, "Jacobian: family not handled by this build");
}

} // namespace fsg
