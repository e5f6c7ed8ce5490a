// Angular-dependent potential (ADP) on the device: the residual of
// ADPForceCalculator::eval_forces (src/force/adp_force.cpp:73-135) and its
// exact parameter Jacobian.
//   pass 1: ρ_i = Σ ρ_{tj}(r), μ_i = Σ u_{ij}(r) d, λ_i = Σ w_{ij}(r) d dᵀ
//   pass 2: clamp, E_i = F(ρ̄_i) + ½|μ_i|² + ½(‖λ_i‖²_F − tr²λ_i/3), F'(ρ̄_i)
//   pass 3: f = (φ' + F'_i ρ'_{tj} + F'_j ρ'_{ti})/r d
//             + (u'/r (μ_i − μ_j)·d) d + u (μ_i − μ_j)
//             + (w'/r ν) d + 2 w ξ,  ν = Σ_{i,j} d·λd − |d|² trλ/3,
//             ξ = Σ_{i,j} λd − (trλ/3) d   (quad_nu / quad_xi, adp_force.hpp:63-69)
// Tables: pair[np], density[nt], embedding[nt], dipole[np], quadrupole[np],
// makima splines or analytic forms, with the closed range gate.
//
// The Jacobian runs the same passes in forward mode: every quantity carries
// its tangent along one parameter direction (one column of J per CTA row of
// the grid), so each column is the exact derivative of the residual above,
// in FP32 or FP64.  The tangent of a table's value enters only through the
// table that owns the column: for a spline, the segment's knot-derivative
// block ∂a/∂y; for an analytic form, its hyper-dual parameter partial.  The
// reference computes this Jacobian analytically for all-analytic tables
// (ADPForceCalculator::write_param_jacobian, adp_force.cpp:141-386) and by
// central differences otherwise; both are this derivative.
#include "jtr.cuh"
#include "kern_common.cuh"

#include <algorithm>
#include <type_traits>
#include <vector>

namespace fsg {
namespace {

// A value and its tangent along one parameter direction.
template <class T> struct Dl {
  T v, t;
  __device__ __forceinline__ Dl() {}
  __device__ __forceinline__ Dl(T x) : v(x), t(T(0)) {}
  __device__ __forceinline__ Dl(T x, T y) : v(x), t(y) {}
};
template <class T> __device__ __forceinline__ Dl<T> operator+(Dl<T> a, Dl<T> b) { return {a.v + b.v, a.t + b.t}; }
template <class T> __device__ __forceinline__ Dl<T> operator-(Dl<T> a, Dl<T> b) { return {a.v - b.v, a.t - b.t}; }
template <class T> __device__ __forceinline__ Dl<T> operator-(Dl<T> a) { return {-a.v, -a.t}; }
template <class T> __device__ __forceinline__ Dl<T> operator*(Dl<T> a, Dl<T> b) {
  return {a.v * b.v, a.v * b.t + a.t * b.v};
}
template <class T> __device__ __forceinline__ Dl<T> operator/(Dl<T> a, Dl<T> b) {
  const T q = a.v / b.v;
  return {q, (a.t - q * b.t) / b.v};
}
template <class T> __device__ __forceinline__ Dl<T> &operator+=(Dl<T> &a, Dl<T> b) { return a = a + b; }
template <class T> __device__ __forceinline__ Dl<T> &operator-=(Dl<T> &a, Dl<T> b) { return a = a - b; }

// Working scalar S (T, or Dl<T> in tangent mode) and its FP64 accumulator.
template <class S> struct Sc;
template <> struct Sc<float> {
  using Acc = double;
  __device__ static float val(float x) { return x; }
  __device__ static double acc(float x) { return static_cast<double>(x); }
};
template <> struct Sc<double> {
  using Acc = double;
  __device__ static double val(double x) { return x; }
  __device__ static double acc(double x) { return x; }
};
template <class T> struct Sc<Dl<T>> {
  using Acc = Dl<double>;
  __device__ static T val(Dl<T> x) { return x.v; }
  __device__ static Dl<double> acc(Dl<T> x) { return Dl<double>(static_cast<double>(x.v), static_cast<double>(x.t)); }
};
template <class A> __device__ __forceinline__ double acc_val(A a) {
  if constexpr (std::is_same_v<A, double>) return a;
  else return a.v;
}

template <class T> struct AdpArgs {
  Common c;
  const typename Vec4T<T>::type *seg_a;
  const T *seg_g;        // [segment][4][kWin] knot-derivative blocks (tangent mode)
  const int32_t *seg_ws; // window start of each segment
  const int2 *col_of;    // tangent mode: per column {table, value index}
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
  T *J;                  // tangent mode: column-major J
  int64_t ld;
};

template <class T> struct TabCtx {
  const STab<T> *tabs;
  const typename Vec4T<T>::type *seg;
  const T *segg;
  const int32_t *segws;
  const double *vals;
  int col_tab, col_k; // the column's table and value index (−1: none)
};

// Value and d/dr of table `tid` at the pair distance r (0 outside its gate),
// with their tangents along the column when S is a dual.
template <class S, class T, class R64>
__device__ __forceinline__ void tab_eval(const TabCtx<T> &C, int tid, T r, R64 &&r64, S &v, S &d) {
  const STab<T> &tb = C.tabs[tid];
  T t;
  const int e = gate_seg(tb, r, t, r64);
  if (e < 0) {
    v = d = S(T(0));
    return;
  }
  T vv, dd;
  if (tb.kind == FS_TABLE_ANALYTIC) {
    const VD<T> q = form_vd<T>(tb.form, C.vals + tb.pv0, tb.n, r, tb.xmax);
    vv = q.v;
    dd = q.d;
  } else {
    vv = seg_val<T>(C.seg[e], t);
    dd = seg_der<T>(C.seg[e], t, tb.inv_h);
  }
  v = S(vv);
  d = S(dd);
  if constexpr (!std::is_same_v<S, T>) {
    if (tid != C.col_tab) return;
    if (tb.kind == FS_TABLE_ANALYTIC) {
      const double *pp = C.vals + tb.pv0;
      if (form_outside<T>(tb.form, pp, r)) return;
      const Hd<T> q = form_seeded<T>(tb.form, pp, tb.n, r, tb.xmax, T(0), C.col_k);
      v.t = q.c;
      d.t = q.d;
    } else {
      const int q = C.col_k - C.segws[e];
      if (q < 0 || q >= kWin) return;
      const T *G = C.segg + e * 4 * kWin;
      v.t = G[q] + t * (G[kWin + q] + t * (G[2 * kWin + q] + t * G[3 * kWin + q]));
      d.t = (G[kWin + q] + t * (T(2) * G[2 * kWin + q] + T(3) * t * G[3 * kWin + q])) * tb.inv_h;
    }
  }
}

// The embedding F of table `tid` at ρ̄ (clamped ρ), value and F', with the
// tangents of ρ (when not clamped) and of the table's own parameters.
template <class S, class T>
__device__ __forceinline__ void emb_eval(const TabCtx<T> &C, int tid, T rb, S rho, bool clamped, S &Fv, S &Fd) {
  const STab<T> &te = C.tabs[tid];
  T v, d, d2 = T(0);
  if (te.kind == FS_TABLE_ANALYTIC) {
    const Hd<T> q = form_seeded<T>(te.form, C.vals + te.pv0, te.n, rb, te.xmax, T(1), -1);
    v = q.a;
    d = q.b;
    d2 = q.d;
  } else {
    T t;
    const int e = seg_of(te, rb, t);
    v = seg_val<T>(C.seg[e], t);
    d = seg_der<T>(C.seg[e], t, te.inv_h);
    if constexpr (!std::is_same_v<S, T>) d2 = seg_der2<T>(C.seg[e], t, te.inv_h);
  }
  Fv = S(v);
  Fd = S(d);
  if constexpr (!std::is_same_v<S, T>) {
    if (!clamped) {
      Fv.t = d * rho.t;
      Fd.t = d2 * rho.t;
    }
    if (tid != C.col_tab) return;
    if (te.kind == FS_TABLE_ANALYTIC) {
      const Hd<T> q = form_seeded<T>(te.form, C.vals + te.pv0, te.n, rb, te.xmax, T(0), C.col_k);
      Fv.t += q.c;
      Fd.t += q.d;
    } else {
      T t;
      const int e = seg_of(te, rb, t);
      const int q = C.col_k - C.segws[e];
      if (q < 0 || q >= kWin) return;
      const T *G = C.segg + e * 4 * kWin;
      Fv.t += G[q] + t * (G[kWin + q] + t * (G[2 * kWin + q] + t * G[3 * kWin + q]));
      Fd.t += (G[kWin + q] + t * (T(2) * G[2 * kWin + q] + T(3) * t * G[3 * kWin + q])) * te.inv_h;
    }
  }
}

template <class A> __device__ __forceinline__ A block_sum_a(A v, double *red) {
  if constexpr (std::is_same_v<A, double>) {
    return block_sum(v, red);
  } else {
    const double a = block_sum(v.v, red);
    const double b = block_sum(v.t, red);
    return A(a, b);
  }
}

// One CTA per configuration (per configuration and column in tangent mode:
// blockIdx.y is the column).  Residual mode writes F and the calculator
// outputs; tangent mode writes the column of J.
template <class T, bool TAN>
__global__ void __launch_bounds__(256) adp_kernel(AdpArgs<T> A) {
  using T4 = typename Vec4T<T>::type;
  using S = std::conditional_t<TAN, Dl<T>, T>;
  using Acc = typename Sc<S>::Acc;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  Smem Sm(smem_raw);
  STab<T> *tabs = Sm.take<STab<T>>(A.c.n_tables);
  T4 *seg = Sm.take<T4>(A.c.n_segs);
  double *wpos = Sm.take<double>(3 * N);
  double *shift = Sm.take<double>(3 * nimg);
  uint8_t *typ = Sm.take<uint8_t>(N);
  S *gF = Sm.take<S>(N);
  S *mu = Sm.take<S>(3 * N);
  S *lam = Sm.take<S>(9 * N);
  double *red = Sm.take<double>(64);
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  for (int k = threadIdx.x; k < A.c.n_segs; k += blockDim.x) seg[k] = A.seg_a[k];
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();
  TabCtx<T> C{tabs, seg, A.seg_g, A.seg_ws, A.c.vals, -1, -1};
  const int col = TAN ? static_cast<int>(blockIdx.y) : -1;
  if constexpr (TAN) {
    C.col_tab = A.col_of[col].x;
    C.col_k = A.col_of[col].y;
  }
  const int32_t *start = A.c.nb_start + cd.atom0;
  Acc e_acc = Acc(0.0), lim = Acc(0.0);
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int ti = typ[i];
    S rho = S(T(0)), m[3] = {S(T(0)), S(T(0)), S(T(0))}, L[9];
    for (int k = 0; k < 9; ++k) L[k] = S(T(0));
    for (int p = start[i]; p < start[i + 1]; ++p) {
      int j;
      T d[3];
      const uint32_t pk = A.c.nb_pack[p];
      pair_vec(wpos, shift, i, pk, j, d[0], d[1], d[2]);
      const T r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r < T(1e-14)) continue;
      const auto r64 = [=] { return pair_len64(wpos, shift, i, pk); };
      const int tj = typ[j], pt = pair_ord(ti, tj, nt);
      S v, dv;
      tab_eval<S>(C, np + tj, r, r64, v, dv);
      rho += v;
      tab_eval<S>(C, 2 * nt + np + pt, r, r64, v, dv); // dipole u_{ij}
      for (int a = 0; a < 3; ++a) m[a] += v * S(d[a]);
      tab_eval<S>(C, 2 * nt + 2 * np + pt, r, r64, v, dv); // quadrupole w_{ij}
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) L[3 * a + b] += v * S(d[a] * d[b]);
    }
    for (int a = 0; a < 3; ++a) mu[3 * i + a] = m[a];
    for (int k = 0; k < 9; ++k) lam[9 * i + k] = L[k];
    const STab<T> &te = tabs[np + nt + ti];
    T rb = Sc<S>::val(rho);
    bool clamped = false;
    if (rb > te.xmax) {
      const Acc dd = Sc<S>::acc(rho) - Acc(static_cast<double>(te.xmax));
      lim += Acc(1000.0) * dd * dd;
      rb = te.xmax;
      clamped = true;
    } else if (rb < te.x0) {
      const Acc dd = Acc(static_cast<double>(te.x0)) - Sc<S>::acc(rho);
      lim += Acc(1000.0) * dd * dd;
      rb = te.x0;
      clamped = true;
    }
    S Fv, Fd;
    emb_eval<S>(C, np + nt + ti, rb, rho, clamped, Fv, Fd);
    gF[i] = Fd;
    Acc ei = Sc<S>::acc(Fv);
    ei += Acc(0.5) * Sc<S>::acc(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const Acc tr = Sc<S>::acc(L[0] + L[4] + L[8]);
    Acc sq = Acc(0.0);
    for (int k = 0; k < 9; ++k) sq += Sc<S>::acc(L[k]) * Sc<S>::acc(L[k]);
    ei += Acc(0.5) * (sq - tr * tr / Acc(3.0));
    e_acc += ei;
  }
  __syncthreads();
  Acc sg[6] = {Acc(0.0), Acc(0.0), Acc(0.0), Acc(0.0), Acc(0.0), Acc(0.0)};
  double objp = 0.0;
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int ti = typ[i];
    S f[3] = {S(T(0)), S(T(0)), S(T(0))};
    Acc ep = Acc(0.0);
    const S *Li = lam + 9 * i;
    const S trLi = (Li[0] + Li[4] + Li[8]) / S(T(3));
    for (int p = start[i]; p < start[i + 1]; ++p) {
      int j;
      T dr[3];
      const uint32_t pk = A.c.nb_pack[p];
      pair_vec(wpos, shift, i, pk, j, dr[0], dr[1], dr[2]);
      const T r = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
      if (r < T(1e-14)) continue;
      const auto r64 = [=] { return pair_len64(wpos, shift, i, pk); };
      const S ir = S(T(1) / r);
      const S d[3] = {S(dr[0]), S(dr[1]), S(dr[2])};
      const int tj = typ[j], pt = pair_ord(ti, tj, nt);
      S phi, dphi, rj, drj, ri, dri, u, du, w, dw;
      tab_eval<S>(C, pt, r, r64, phi, dphi);
      tab_eval<S>(C, np + tj, r, r64, rj, drj);
      tab_eval<S>(C, np + ti, r, r64, ri, dri);
      tab_eval<S>(C, 2 * nt + np + pt, r, r64, u, du);
      tab_eval<S>(C, 2 * nt + 2 * np + pt, r, r64, w, dw);
      S g[3];
      const S es = (dphi + gF[i] * drj + gF[j] * dri) * ir;
      const S *mi = mu + 3 * i, *mj = mu + 3 * j;
      const S dot = (mi[0] * d[0] + mi[1] * d[1] + mi[2] * d[2]) - (mj[0] * d[0] + mj[1] * d[1] + mj[2] * d[2]);
      const S *Lj = lam + 9 * j;
      const S trLj = (Lj[0] + Lj[4] + Lj[8]) / S(T(3));
      const S dd2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      S Ld_i[3], Ld_j[3];
      for (int a = 0; a < 3; ++a) {
        Ld_i[a] = Li[3 * a] * d[0] + Li[3 * a + 1] * d[1] + Li[3 * a + 2] * d[2];
        Ld_j[a] = Lj[3 * a] * d[0] + Lj[3 * a + 1] * d[1] + Lj[3 * a + 2] * d[2];
      }
      const S nu = (d[0] * Ld_i[0] + d[1] * Ld_i[1] + d[2] * Ld_i[2] - dd2 * trLi) +
                   (d[0] * Ld_j[0] + d[1] * Ld_j[1] + d[2] * Ld_j[2] - dd2 * trLj);
      for (int a = 0; a < 3; ++a) {
        const S xi = (Ld_i[a] - trLi * d[a]) + (Ld_j[a] - trLj * d[a]);
        g[a] = es * d[a] + (du * ir * dot) * d[a] + u * (mi[a] - mj[a]) + (dw * ir * nu) * d[a] + S(T(2)) * w * xi;
        f[a] += g[a];
      }
      ep += Sc<S>::acc(phi);
      const Acc h0 = Acc(0.5 * static_cast<double>(dr[0])), h1 = Acc(0.5 * static_cast<double>(dr[1])),
                h2 = Acc(0.5 * static_cast<double>(dr[2]));
      sg[0] -= h0 * Sc<S>::acc(g[0]);
      sg[1] -= h1 * Sc<S>::acc(g[1]);
      sg[2] -= h2 * Sc<S>::acc(g[2]);
      sg[3] -= h0 * Sc<S>::acc(g[1]);
      sg[4] -= h0 * Sc<S>::acc(g[2]);
      sg[5] -= h1 * Sc<S>::acc(g[2]);
    }
    const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
    if constexpr (TAN) {
      T *Jc = A.J + static_cast<int64_t>(col) * A.ld + row0 + 3 * i;
      for (int a = 0; a < 3; ++a) Jc[a] = f[a].t;
    } else {
      for (int a = 0; a < 3; ++a) {
        const double fa = static_cast<double>(f[a]);
        const double res = fa - A.c.ref_force[3 * ga + a];
        A.F[row0 + 3 * i + a] = res;
        if (A.forces) A.forces[3 * ga + a] = fa;
        objp += res * res;
      }
    }
    e_acc += Acc(0.5) * ep;
  }
  const Acc E = block_sum_a(e_acc, red);
  const Acc Lm = block_sum_a(lim, red);
  Acc st[6];
  for (int a = 0; a < 6; ++a) st[a] = block_sum_a(sg[a], red);
  const double op = block_sum(objp, red);
  if (threadIdx.x != 0) return;
  const double iv = 1.0 / cd.volume;
  for (int a = 0; a < 6; ++a) st[a] = st[a] * Acc(iv);
  int64_t row = row0 + 3 * N;
  static constexpr int vi[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
  if constexpr (TAN) {
    T *Jc = A.J + static_cast<int64_t>(col) * A.ld;
    Jc[row++] = static_cast<T>(A.w_e * E.t);
    if (A.w_s > 0.0)
      for (int v = 0; v < 6; ++v) Jc[row++] = static_cast<T>(A.w_s * st[v].t);
    Jc[row] = static_cast<T>(Lm.t);
  } else {
    double o = op;
    const double re = A.w_e * (E - cd.ref_energy);
    A.F[row++] = re;
    o += re * re;
    if (A.w_s > 0.0)
      for (int v = 0; v < 6; ++v) {
        const double rs = A.w_s * (st[v] - cd.ref_stress[3 * vi[v][0] + vi[v][1]]);
        A.F[row++] = rs;
        o += rs * rs;
      }
    A.F[row++] = Lm;
    o += Lm * Lm;
    A.obj_part[c] = o;
    if (A.energy) A.energy[c] = E;
    if (A.limit) A.limit[c] = Lm;
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
}

__global__ void adp_sum(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *out = s;
}

// Residual (jac = false) or Jacobian (jac = true: one CTA per configuration
// and column, then Jᵀr) of an ADP model.
template <class T> int launch_adp(fs_gpu *h, double w_e, double w_s, bool jac) {
  using T4 = typename Vec4T<T>::type;
  AdpArgs<T> a;
  a.c = make_common<T>(h);
  a.seg_a = static_cast<const T4 *>(h->d_seg_a);
  a.seg_g = static_cast<const T *>(h->d_seg_g);
  a.seg_ws = h->d_seg_ws;
  a.col_of = nullptr;
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
  const int N = h->max_natoms, max_img = max_images(h);
  const size_t s = jac ? sizeof(Dl<T>) : sizeof(T);
  const size_t sm = align16(a.c.n_tables * sizeof(STab<T>)) + align16(h->n_segs * 4 * sizeof(T)) +
                    align16(3 * N * sizeof(double)) + align16(3 * max_img * sizeof(double)) + align16(N) +
                    align16(N * s) + align16(3 * N * s) + align16(9 * N * s) + align16(64 * sizeof(double)) + 128;
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "ADP: configuration too large for shared memory");
  if (!jac) {
    FS_CUDA(cudaFuncSetAttribute(adp_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sm)));
    adp_kernel<T, false><<<h->n_cfg, 256, sm, h->stream>>>(a);
    FS_CUDA(cudaGetLastError());
    adp_sum<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
    FS_CUDA(cudaGetLastError());
    h->launches += 2;
    return FS_OK;
  }
  const int D = h->D;
  if (D > 65535) return set_error(h, FS_ERR_UNSUPPORTED, "ADP Jacobian: more than 65535 columns");
  const int64_t M = rows_of(h, w_s);
  const int64_t ldj = (M + 31) / 32 * 32;
  const size_t jn = static_cast<size_t>(ldj) * D;
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
    FS_CUDA(cudaMalloc(&h->d_JtJ, std::max(D * D, 1) * sizeof(double)));
    FS_CUDA(cudaMalloc(&h->d_Jtr, std::max(D, 1) * sizeof(double)));
  }
  // each column's table and value index, kept with the context
  std::vector<int2> cols(std::max(D, 1), make_int2(-1, -1));
  for (int t = 0; t < static_cast<int>(h->tables.size()); ++t)
    for (int k = 0; k < h->tables[t].n; ++k)
      if (h->tables[t].cols[k] >= 0) cols[h->tables[t].cols[k]] = make_int2(t, k);
  const size_t need = sizeof(int2) * cols.size();
  if (h->an_alloc < need || !h->d_an) {
    if (h->d_an) cudaFree(h->d_an);
    h->d_an = nullptr;
    h->an_alloc = 0;
    FS_CUDA(cudaMalloc(&h->d_an, need));
    h->an_alloc = need;
  }
  FS_CUDA(cudaMemcpyAsync(h->d_an, cols.data(), need, cudaMemcpyHostToDevice, h->stream));
  a.col_of = static_cast<const int2 *>(h->d_an);
  a.J = static_cast<T *>(h->d_J);
  a.ld = ldj;
  mark(h, 2);
  if (D > 0) {
    FS_CUDA(cudaFuncSetAttribute(adp_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sm)));
    adp_kernel<T, true><<<dim3(h->n_cfg, D), 256, sm, h->stream>>>(a);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  mark(h, 3);
  return launch_jtr<T>(h, static_cast<const T *>(h->d_J), ldj, M, D, h->d_F, h->d_Jtr);
}

} // namespace

int eval_residual_adp(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_adp<double>(h, w_e, w_s, false) : launch_adp<float>(h, w_e, w_s, false);
}

// The exact ADP Jacobian (forward mode), spline or analytic tables, FP32 or FP64.
int eval_jacobian_adp(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_adp<double>(h, w_e, w_s, true) : launch_adp<float>(h, w_e, w_s, true);
}

} // namespace fsg
