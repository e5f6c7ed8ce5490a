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
// One CTA per configuration, one thread per central atom.  Forces on the end
// atoms j, k of a triplet and the Jacobian block of the configuration
// ((3N + rows) × D, D = the few free SW parameters) accumulate in shared
// memory with atomics, then stream out.
#include "kern_common.cuh"

#include <algorithm>

namespace fsg {
namespace {

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
  const T ib = T(1) / b.v;
  Dual<T, N> r(a.v * ib);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
template <class T, int N> __device__ Dual<T, N> dexp(const Dual<T, N> &a) {
  Dual<T, N> r(exp(a.v));
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
  const T lr = log(r);
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
};

template <class T>
__device__ __forceinline__ void add_row(T *Jb, int D, int row, int col, T v) {
  if (col >= 0 && v != T(0)) atomicAdd(&Jb[static_cast<int64_t>(row) * D + col], v);
}

template <class T, bool JAC>
__global__ void __launch_bounds__(256) sw_kernel(SwArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
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
  double *red = S.take<double>(64);
  T *Jb = JAC ? S.take<T>(static_cast<size_t>(3 * N + 7) * D) : nullptr; // force rows, E, 6 stress
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
  __syncthreads();
  const int32_t *start = A.c.nb_start + cd.atom0;
  double e_acc = 0.0, sg[6] = {0, 0, 0, 0, 0, 0};
  const int rowE = 3 * N; // local rows of the block: 3N force, E, 6 stress
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int ti = typ[i];
    T fi[3] = {0, 0, 0};
    // ---- 2-body (½ v₂ per directed pair, force on i)
    for (int p = start[i]; p < start[i + 1]; ++p) {
      int j;
      T d[3];
      pair_vec(wpos, shift, i, A.c.nb_pack[p], j, d[0], d[1], d[2]);
      const T r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r < T(1e-14)) continue;
      const int sl = pair_ord(ti, typ[j], nt);
      const T *P = par + 8 * sl;
      if constexpr (JAC) {
        Dual<T, 6> v2, dv2;
        v2_dual(r, P, v2, dv2);
        const T s = dv2.v / r;
        for (int a = 0; a < 3; ++a) fi[a] += s * d[a];
        e_acc += 0.5 * static_cast<double>(v2.v);
        const T f[3] = {s * d[0], s * d[1], s * d[2]};
        sg[0] -= 0.5 * d[0] * f[0];
        sg[1] -= 0.5 * d[1] * f[1];
        sg[2] -= 0.5 * d[2] * f[2];
        sg[3] -= 0.5 * d[0] * f[1];
        sg[4] -= 0.5 * d[0] * f[2];
        sg[5] -= 0.5 * d[1] * f[2];
        for (int k = 0; k < 6; ++k) {
          const int col = pcol[8 * sl + k];
          if (col < 0) continue;
          const T ds = dv2.d[k] / r;
          for (int a = 0; a < 3; ++a) add_row(Jb, D, 3 * i + a, col, ds * d[a]);
          add_row(Jb, D, rowE, col, static_cast<T>(0.5 * A.w_e) * v2.d[k]);
          const T df[3] = {ds * d[0], ds * d[1], ds * d[2]};
          add_row(Jb, D, rowE + 1, col, T(-0.5) * d[0] * df[0]);
          add_row(Jb, D, rowE + 2, col, T(-0.5) * d[1] * df[1]);
          add_row(Jb, D, rowE + 3, col, T(-0.5) * d[2] * df[2]);
          add_row(Jb, D, rowE + 4, col, T(-0.5) * d[0] * df[1]);
          add_row(Jb, D, rowE + 5, col, T(-0.5) * d[0] * df[2]);
          add_row(Jb, D, rowE + 6, col, T(-0.5) * d[1] * df[2]);
        }
      } else {
        T v2, dv2;
        v2_plain(r, P, v2, dv2);
        const T s = dv2 / r;
        const T f[3] = {s * d[0], s * d[1], s * d[2]};
        for (int a = 0; a < 3; ++a) fi[a] += f[a];
        e_acc += 0.5 * static_cast<double>(v2);
        const T hx = T(0.5) * d[0], hy = T(0.5) * d[1], hz = T(0.5) * d[2];
        sg[0] -= hx * f[0];
        sg[1] -= hy * f[1];
        sg[2] -= hz * f[2];
        sg[3] -= hx * f[1];
        sg[4] -= hx * f[2];
        sg[5] -= hy * f[2];
      }
    }
    // ---- 3-body, neighbour pairs jj < kk of central atom i
    for (int pj = start[i]; pj < start[i + 1]; ++pj) {
      int j;
      T d1[3];
      pair_vec(wpos, shift, i, A.c.nb_pack[pj], j, d1[0], d1[1], d1[2]);
      const T r1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
      if (r1 < T(1e-14)) continue;
      const int tj = typ[j];
      const int s1 = pair_ord(ti, tj, nt);
      Dual<T, 5> h1, dh1;
      h_dual<T, 5>(r1, par[8 * s1 + 6], par[8 * s1 + 7], 0, 1, h1, dh1);
      if (h1.v == T(0) && dh1.v == T(0)) continue; // make_jbond (stiweb_force.cpp:107-121)
      const T ir1 = T(1) / r1;
      for (int pk = pj + 1; pk < start[i + 1]; ++pk) {
        int k;
        T d2[3];
        pair_vec(wpos, shift, i, A.c.nb_pack[pk], k, d2[0], d2[1], d2[2]);
        const T r2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
        if (r2 < T(1e-14)) continue;
        const int tk = typ[k];
        const int s2 = pair_ord(ti, tk, nt);
        Dual<T, 5> h2, dh2;
        h_dual<T, 5>(r2, par[8 * s2 + 6], par[8 * s2 + 7], 2, 3, h2, dh2);
        if (h2.v == T(0) && dh2.v == T(0)) continue;
        const T ir2 = T(1) / r2;
        const int lt = ti * np + pair_ord(tj, tk, nt);
        const Dual<T, 5> L = Dual<T, 5>::var(lam[lt], 4);
        const T cth = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) * ir1 * ir2;
        const T cp = cth + T(1) / T(3);
        const Dual<T, 5> w = (cp * cp) * L, dw = (T(2) * cp) * L;
        // three_body_forces (kernels.hpp:44-58)
        const T irr = ir1 * ir2;
        const T Aa = cth * ir1 * ir1 - irr, Bb = cth * ir2 * ir2 - irr;
        const Dual<T, 5> c1 = (ir1 * dh1) * h2 * w;   // df1·inv_r1·f2·g
        const Dual<T, 5> c2 = h1 * (ir2 * dh2) * w;   // f1·df2·inv_r2·g
        const Dual<T, 5> c3 = h1 * h2 * dw;           // f1·f2·dg
        const Dual<T, 5> e3 = h1 * h2 * w;
        T Fi[3], Fj[3], Fk[3];
        for (int a = 0; a < 3; ++a) {
          Fi[a] = c1.v * d1[a] + c2.v * d2[a] - c3.v * (Aa * d1[a] + Bb * d2[a]);
          Fj[a] = -(c1.v * d1[a]) - c3.v * (irr * d2[a] - cth * ir1 * ir1 * d1[a]);
          Fk[a] = -(c2.v * d2[a]) - c3.v * (irr * d1[a] - cth * ir2 * ir2 * d2[a]);
          fi[a] += Fi[a];
        }
        atomicAdd(&Fs[3 * j], Fj[0]);
        atomicAdd(&Fs[3 * j + 1], Fj[1]);
        atomicAdd(&Fs[3 * j + 2], Fj[2]);
        atomicAdd(&Fs[3 * k], Fk[0]);
        atomicAdd(&Fs[3 * k + 1], Fk[1]);
        atomicAdd(&Fs[3 * k + 2], Fk[2]);
        e_acc += static_cast<double>(e3.v);
        sg[0] += d1[0] * Fj[0] + d2[0] * Fk[0];
        sg[1] += d1[1] * Fj[1] + d2[1] * Fk[1];
        sg[2] += d1[2] * Fj[2] + d2[2] * Fk[2];
        sg[3] += d1[0] * Fj[1] + d2[0] * Fk[1];
        sg[4] += d1[0] * Fj[2] + d2[0] * Fk[2];
        sg[5] += d1[1] * Fj[2] + d2[1] * Fk[2];
        if constexpr (JAC) {
          const int cols[5] = {pcol[8 * s1 + 6], pcol[8 * s1 + 7], pcol[8 * s2 + 6], pcol[8 * s2 + 7], lcol[lt]};
          for (int q = 0; q < 5; ++q) {
            const int col = cols[q];
            if (col < 0) continue;
            T gi[3], gj[3], gk[3];
            for (int a = 0; a < 3; ++a) {
              gi[a] = c1.d[q] * d1[a] + c2.d[q] * d2[a] - c3.d[q] * (Aa * d1[a] + Bb * d2[a]);
              gj[a] = -(c1.d[q] * d1[a]) - c3.d[q] * (irr * d2[a] - cth * ir1 * ir1 * d1[a]);
              gk[a] = -(c2.d[q] * d2[a]) - c3.d[q] * (irr * d1[a] - cth * ir2 * ir2 * d2[a]);
              add_row(Jb, D, 3 * i + a, col, gi[a]);
              add_row(Jb, D, 3 * j + a, col, gj[a]);
              add_row(Jb, D, 3 * k + a, col, gk[a]);
            }
            add_row(Jb, D, rowE, col, static_cast<T>(A.w_e) * e3.d[q]);
            add_row(Jb, D, rowE + 1, col, d1[0] * gj[0] + d2[0] * gk[0]);
            add_row(Jb, D, rowE + 2, col, d1[1] * gj[1] + d2[1] * gk[1]);
            add_row(Jb, D, rowE + 3, col, d1[2] * gj[2] + d2[2] * gk[2]);
            add_row(Jb, D, rowE + 4, col, d1[0] * gj[1] + d2[0] * gk[1]);
            add_row(Jb, D, rowE + 5, col, d1[0] * gj[2] + d2[0] * gk[2]);
            add_row(Jb, D, rowE + 6, col, d1[1] * gj[2] + d2[1] * gk[2]);
          }
        }
      }
    }
    atomicAdd(&Fs[3 * i], fi[0]);
    atomicAdd(&Fs[3 * i + 1], fi[1]);
    atomicAdd(&Fs[3 * i + 2], fi[2]);
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
  const double E = block_sum(e_acc, red);
  double st[6];
  for (int a = 0; a < 6; ++a) st[a] = block_sum(sg[a], red);
  const double op = block_sum(objp, red);
  __shared__ double s_rows[8];
  if (threadIdx.x == 0) {
    const double iv = 1.0 / cd.volume;
    for (int a = 0; a < 6; ++a) st[a] *= iv;
    int64_t row = row0 + 3 * N;
    double o = op;
    const double re = A.w_e * (E - cd.ref_energy);
    A.F[row++] = re;
    s_rows[0] = re;
    o += re * re;
    static constexpr int vi[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    if (A.w_s > 0.0)
      for (int v = 0; v < 6; ++v) {
        const double rs = A.w_s * (st[v] - cd.ref_stress[3 * vi[v][0] + vi[v][1]]);
        A.F[row++] = rs;
        s_rows[1 + v] = rs;
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
      jr = block_sum(jr, red);
      if (threadIdx.x == 0) A.jtr_part[static_cast<int64_t>(c) * D + col] = jr;
    }
  }
}

template <class T> size_t sw_smem(fs_gpu *h, int max_img, bool jac) {
  const int nt = h->ntypes, np = npair_of(nt), N = h->max_natoms;
  size_t b = align16(3 * N * sizeof(double)) + align16(3 * max_img * sizeof(double)) + align16(N) +
             align16(3 * N * sizeof(T)) + align16(8 * np * sizeof(T)) + align16(nt * np * sizeof(T)) +
             align16(8 * np * sizeof(int)) + align16(nt * np * sizeof(int)) + align16(64 * sizeof(double));
  if (jac) b += align16(static_cast<size_t>(3 * N + 7) * h->D * sizeof(T));
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
    if (static_cast<size_t>(h->jac_alloc) != jn || h->ldj != ldj || !h->d_J) {
      if (h->d_J) cudaFree(h->d_J);
      h->d_J = nullptr;
      FS_CUDA(cudaMalloc(&h->d_J, std::max<size_t>(jn, 1) * sizeof(T)));
      FS_CUDA(cudaMemsetAsync(h->d_J, 0, std::max<size_t>(jn, 1) * sizeof(T), h->stream));
      h->jac_alloc = static_cast<int64_t>(jn);
      h->ldj = ldj;
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
  const size_t sm = sw_smem<T>(h, max_images_of(h), jac);
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "SW: configuration too large for shared memory");
  auto k = jac ? sw_kernel<T, true> : sw_kernel<T, false>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, 256, sm, h->stream>>>(a);
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
int eval_jacobian_fd(fs_gpu *h, double w_e, double w_s);

int eval_residual_other(fs_gpu *h, double w_e, double w_s) {
  if (h->family == FS_FAMILY_SW)
    return h->precision == FS_PREC_FP64 ? launch_sw<double>(h, w_e, w_s, false) : launch_sw<float>(h, w_e, w_s, false);
  if (h->family == FS_FAMILY_ADP) return eval_residual_adp(h, w_e, w_s);
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
  if (h->family == FS_FAMILY_ADP) return eval_jacobian_fd(h, w_e, w_s);
  return set_error(h, FS_ERR_UNSUPPORTED, "Jacobian: family not handled by this build");
}

} // namespace fsg
