// ACSF descriptors with a linear energy head per species, on the device.
//
//   ACSF::get_descriptor (src/force/acsf.cpp:84-196): per central atom i and
//   neighbour j with 1e-14 ≤ r < rcut, f_c = ½(1 + cos(πr/rcut)):
//     G1 = f_c, G2 = e^{−η(r − rs)²} f_c, G3 = cos(κr) f_c   (per species of j),
//   per neighbour pair j < k (per species pair):
//     G4/G5 = 2^{1−ζ}(1 + λ cos θ)^ζ e^{−η(r_ij² + r_ik² [+ r_jk²])}
//             f_c(r_ij) f_c(r_ik) [f_c(r_jk)],   skipped when 1 + λ cos θ ≤ 1e-12,
//   laid out as AcsfLayout (acsf.hpp:23-46).
//   LinearHead (src/force/ml_force.cpp:11-47): E_i = w_{t_i}·D_i + b_{t_i}.
//   MLBase::eval_forces (include/forcesmith/force/ml_force.hpp): F −= (∂D/∂r)ᵀ w
//   on i and its neighbours, σ += d_ij ⊗ (force on j).
//   The Jacobian with respect to the head coefficients is exact and does not
//   depend on them: ∂F/∂w = −∂D/∂r, ∂E/∂w = Σ_i D_i, ∂E/∂b = atom count
//   (eval_cached_jacobian, ml_force.hpp).
//
// One CTA per configuration; each warp takes 32 consecutive work items from a
// block scan: directed pairs (G1–G3), then neighbour pairs (j < k) of a
// central atom (G4, G5).  Items are ordered by central atom, so runs of lanes
// share atom i (and, for neighbour pairs, atom j): their force updates are
// summed over each run with shuffles and added once.  Residual: forces in
// shared memory; energy and stress as per-thread FP64 sums.  Jacobian: force
// rows into the configuration's force-row block in shared memory, written out
// once (or, when the block does not fit, straight into J, zeroed first); the
// energy and stress rows, which every term hits, summed over the warp and
// then in FP64 shared memory, written to J once;
// a two-pass column reduction forms Jᵀr.
#include "jtr.cuh"
#include "kern_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fsg {
namespace {

constexpr int kAcThreads = 256;

// exp, x^y, 1/x and the cutoff's sine and cosine (argument in [0, π]): the
// hardware approximations in FP32 (a few ulp, or 2^-21 absolute for the
// sine and cosine, inside the FP32 path's stated tolerances), IEEE in FP64
__device__ __forceinline__ float ac_exp(float x) { return __expf(x); }
__device__ __forceinline__ double ac_exp(double x) { return exp(x); }
__device__ __forceinline__ float ac_pow(float a, float z) { return __expf(z * __logf(a)); }
__device__ __forceinline__ double ac_pow(double a, double z) { return pow(a, z); }
__device__ __forceinline__ float ac_rcp(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double ac_rcp(double x) { return 1.0 / x; }
__device__ __forceinline__ void ac_sincos(float x, float &s, float &c) { __sincosf(x, &s, &c); }
__device__ __forceinline__ void ac_sincos(double x, double &s, double &c) { sincos(x, &s, &c); }
// sine and cosine of any argument (G3's κr): the full-range library functions
__device__ __forceinline__ void ac_sincos_full(float x, float &s, float &c) { sincosf(x, &s, &c); }
__device__ __forceinline__ void ac_sincos_full(double x, double &s, double &c) { sincos(x, &s, &c); }

// f_c(r) = ½(1 + cos(πr/rc)) and its derivative; prc = π/rc
template <class T> __device__ __forceinline__ void ac_fc(T r, T rc, T prc, T &fc, T &fcp) {
  if (r >= rc) {
    fc = fcp = T(0);
    return;
  }
  T sn, cs;
  ac_sincos(prc * r, sn, cs);
  fc = T(0.5) * (T(1) + cs);
  fcp = T(-0.5) * prc * sn;
}

// The descriptor hyperparameters and layout (acsf.hpp:23-46), from the ACSF
// table's values {rcut, nG1..nG5, parameters}.
struct AcLayout {
  int g1, n2, n3, n4, n5, nt, S;
  int base[5];
  __device__ __host__ void init(const double *v, int ntypes) {
    g1 = static_cast<int>(v[1]);
    n2 = static_cast<int>(v[2]);
    n3 = static_cast<int>(v[3]);
    n4 = static_cast<int>(v[4]);
    n5 = static_cast<int>(v[5]);
    nt = ntypes;
    const int P = nt * (nt + 1) / 2;
    base[0] = 0;
    base[1] = base[0] + g1 * nt;
    base[2] = base[1] + n2 * nt;
    base[3] = base[2] + n3 * nt;
    base[4] = base[3] + n4 * P;
    S = base[4] + n5 * P;
  }
};

template <class T> struct AcArgs {
  Common c;
  const double *vals; // all model values (FP64)
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
  const int32_t *order;
  // Jacobian
  T *J;
  int64_t ld;
  int D;   // columns (free head values)
  int smj; // 1: the configuration's J block is summed in shared memory first
  int std_on;   // 1: standardization tables follow the heads ({mean[S], inv_std[S]} per species)
  double *desc; // MODE 2: per-atom descriptors [atom][S] (zeroed before)
};

// One CTA per configuration.  MODE 0: residual; 1: J rows; 2: each atom's
// descriptors (for the standardization statistics).
//
// Standardized heads (the head sees (D − mean) ⊙ inv_std) act as heads of
// raw descriptors with w' = w ⊙ inv_std and b' = b − Σ w·inv_std·mean; in the
// Jacobian, w_k's column is inv_std_k times the raw one, and its energy row
// also gets −w_e·inv_std_k·mean_k per atom of the species.
template <class T, int MODE> __global__ void __launch_bounds__(kAcThreads) acsf_kernel(AcArgs<T> A) {
  constexpr bool JAC = MODE == 1, DESC = MODE == 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = A.order ? A.order[blockIdx.x] : blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nt = A.c.ntypes;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  const double *spec = A.vals + A.c.desc[0].pv0;
  AcLayout L;
  L.init(spec, nt);
  const int nspec = A.c.desc[0].n;
  Smem S(smem_raw);
  T *par = S.take<T>(nspec);           // rcut, counts, function parameters
  T *W = S.take<T>(nt * (L.S + 1));    // heads: w[S], b per species
  int *col = S.take<int>(nt * (L.S + 1)); // head value → J column (−1 fixed)
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  T *Fs = S.take<T>(3 * N);
  double *red = S.take<double>(8 * 32);
  int *pfirst = S.take<int>(N + 1);
  int *tfirst = S.take<int>(N + 1);
  int *wsum = S.take<int>(32);
  T *cz = S.take<T>(L.n4 + L.n5); // 2^{1−ζ} of each G4, G5 function
  // JAC with standardization: inv_std per (species, descriptor) and atoms per species
  T *ivs = (JAC && A.std_on) ? S.take<T>(nt * L.S) : nullptr;
  int *ntyp = (JAC && A.std_on) ? S.take<int>(nt) : nullptr;
  // JAC with smj: the 3N force rows (local) × D columns
  T *Jb = (JAC && A.smj) ? S.take<T>(static_cast<size_t>(3 * N) * A.D) : nullptr;
  // JAC: the configuration's energy and 6 stress rows, summed in FP64 (every
  // term of the configuration adds to them, and a standardized column then
  // cancels most of its energy row against the mean shift)
  double *E64 = JAC ? S.take<double>(static_cast<size_t>(7) * A.D) : nullptr;
  if (E64)
    for (int k = threadIdx.x; k < 7 * A.D; k += blockDim.x) E64[k] = 0.0;
  if (Jb)
    for (int k = threadIdx.x; k < 3 * N * A.D; k += blockDim.x) Jb[k] = T(0);
  for (int k = threadIdx.x; k < nspec; k += blockDim.x) par[k] = static_cast<T>(spec[k]);
  for (int k = threadIdx.x; k < L.n4 + L.n5; k += blockDim.x) {
    const double zeta = k < L.n4 ? spec[6 + 2 * L.n2 + L.n3 + 3 * k + 1] : spec[6 + 2 * L.n2 + L.n3 + 3 * L.n4 + 3 * (k - L.n4) + 1];
    cz[k] = static_cast<T>(pow(2.0, 1.0 - zeta));
  }
  for (int k = threadIdx.x; k < nt * (L.S + 1); k += blockDim.x) {
    const int t = k / (L.S + 1), q = k % (L.S + 1);
    const TableDesc &td = A.c.desc[1 + t];
    const double *w = A.vals + td.pv0;
    double v = w[q];
    if (A.std_on) { // w ⊙ inv_std; b − Σ w·inv_std·mean
      const double *st = A.vals + A.c.desc[1 + nt + t].pv0; // mean[S], inv_std[S]
      if (q < L.S) {
        v = w[q] * st[L.S + q];
      } else {
        for (int u = 0; u < L.S; ++u) v -= w[u] * st[L.S + u] * st[u];
      }
    }
    W[k] = static_cast<T>(v);
    col[k] = A.c.cmap[td.cmap0 + q];
  }
  if (ivs) {
    for (int k = threadIdx.x; k < nt * L.S; k += blockDim.x)
      ivs[k] = static_cast<T>(A.vals[A.c.desc[1 + nt + k / L.S].pv0 + L.S + k % L.S]);
    for (int k = threadIdx.x; k < nt; k += blockDim.x) ntyp[k] = 0;
  }
  for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) Fs[k] = T(0);
  stage_geometry(cd, A.c, wpos, shift, typ);
  const int32_t *start = A.c.nb_start + cd.atom0;
  stage_work(start, N, pfirst, tfirst, wsum);
  __syncthreads();
  const T rc = par[0];
  const T prc = static_cast<T>(3.14159265358979323846 / spec[0]);
  const T *p2 = par + 6, *p3 = p2 + 2 * L.n2, *p4 = p3 + L.n3, *p5 = p4 + 3 * L.n4;
  const T *c4 = cz, *c5 = cz + L.n4;
  const uint32_t *nbp = A.c.nb_pack + start[0];
  const int npair = pfirst[N], ntri = tfirst[N];
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  const int64_t rowE = row0 + 3 * N;
  const T sw = static_cast<T>(A.w_s / cd.volume), we = static_cast<T>(A.w_e);
  double e_acc = 0.0, sg[6] = {0, 0, 0, 0, 0, 0}; // xx, yy, zz, xy, xz, yz
  // J entry (local row r of this configuration: 3N force rows, then E, 6
  // stress) in column cl: force rows to the shared block when there is one,
  // else to J
  auto jadd = [&](int cl, int r, T v) {
    if (Jb && r < 3 * N) atomicAdd(&Jb[r * A.D + cl], v);
    else atomicAdd(&A.J[static_cast<int64_t>(cl) * A.ld + row0 + r], v);
  };
  const int rE = 3 * N;
  const int lane = threadIdx.x & 31;
  const int nrow = A.w_s > 0.0 ? 7 : 1;
  // The energy and stress rows of one term in column c0, which every term of
  // the configuration hits: summed over the warp and added once per row.
  // Lanes without a term pass zeros; all 32 lanes call this together.
  auto erows_warp = [&](int c0, T e, const T (&st)[6]) {
    const T v[8] = {we * e, st[0], st[1], st[2], st[3], st[4], st[5], T(0)};
    const T t = warp_sum_tr<8>(v, lane); // lanes 4m hold row m
    const int m = lane >> 2;
    if ((lane & 3) == 0 && m < nrow) atomicAdd(&E64[m * A.D + c0], static_cast<double>(t));
  };
  // the same rows from one lane
  auto erows_lane = [&](int cl, T e, const T (&st)[6]) {
    atomicAdd(&E64[cl], static_cast<double>(we * e));
    for (int m = 1; m < nrow; ++m) atomicAdd(&E64[m * A.D + cl], static_cast<double>(st[m - 1]));
  };
  // ---- G1–G3: one thread per directed pair; each warp takes 32 consecutive
  // items (the Jacobian's warp sums need every lane; spare lanes repeat the
  // last item with ok false)
  for (int w0 = threadIdx.x - lane; w0 < npair; w0 += blockDim.x) {
    const int w = min(w0 + lane, npair - 1);
    const int i = owner_of(pfirst, N, w);
    int j;
    T d[3];
    pair_vec(wpos, shift, i, nbp[w], j, d[0], d[1], d[2]);
    const T r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const bool ok = w0 + lane < npair && r >= T(1e-14) && r < rc;
    if (!__any_sync(0xffffffffu, ok)) continue;
    const T ir = ok ? ac_rcp(r) : T(0);
    const T rh[3] = {d[0] * ir, d[1] * ir, d[2] * ir};
    T fc, fcp;
    ac_fc(r, rc, prc, fc, fcp);
    const int s = typ[j], ti = typ[i];
    const T *w_ = W + ti * (L.S + 1);
    const int *cl = col + ti * (L.S + 1);
    T cw = T(0), ew = T(0);
    bool hi = false;
    const unsigned xi = run_links(i, lane, hi);
    auto term = [&](int idx, T g, T dg) {
      if constexpr (DESC) {
        if (ok) atomicAdd(&A.desc[(static_cast<int64_t>(cd.atom0) + i) * L.S + idx], static_cast<double>(g));
      } else if constexpr (JAC) {
        if (ivs) { // standardized: the column of w_idx scales by inv_std_idx
          const T sv = ivs[ti * L.S + idx];
          g *= sv;
          dg *= sv;
        }
        // force rows: +g on i, −g on j; stress −sw d ⊗ g
        T gv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) gv[a] = ok ? dg * rh[a] : T(0);
        const T st[6] = {-sw * d[0] * gv[0], -sw * d[1] * gv[1], -sw * d[2] * gv[2],
                         -sw * d[0] * gv[1], -sw * d[0] * gv[2], -sw * d[1] * gv[2]};
        const int cc = cl[idx];
        const int c0 = __shfl_sync(0xffffffffu, cc, 0);
        if (__all_sync(0xffffffffu, cc == c0)) {
          // one column for the warp (always, with one species): atom i's rows
          // summed over its run of lanes, energy and stress over the warp
          if (c0 < 0) return;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const T t = run_sum(gv[a], xi);
            if (hi) jadd(c0, 3 * i + a, t);
            if (ok) jadd(c0, 3 * j + a, -gv[a]);
          }
          erows_warp(c0, ok ? g : T(0), st);
        } else if (ok && cc >= 0) {
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            jadd(cc, 3 * i + a, gv[a]);
            jadd(cc, 3 * j + a, -gv[a]);
          }
          erows_lane(cc, g, st);
        }
      } else {
        cw += w_[idx] * dg;
        ew += w_[idx] * g;
      }
    };
    for (int t = 0; t < L.g1; ++t) term(L.base[0] + s * L.g1 + t, fc, fcp);
    for (int t = 0; t < L.n2; ++t) {
      const T eta = p2[2 * t], dr = r - p2[2 * t + 1];
      const T gs = ac_exp(-eta * dr * dr);
      term(L.base[1] + s * L.n2 + t, gs * fc, gs * (T(-2) * eta * dr * fc + fcp));
    }
    for (int t = 0; t < L.n3; ++t) {
      const T k = p3[t];
      T ss, cc;
      ac_sincos_full(k * r, ss, cc);
      term(L.base[2] + s * L.n3 + t, cc * fc, -k * ss * fc + cc * fcp);
    }
    if constexpr (MODE == 0) {
      // atom i's force summed over its run of lanes (rh is zero without a term)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const T f = cw * rh[a];
        const T t = run_sum(f, xi);
        if (hi) atomicAdd(&Fs[3 * i + a], t);
        if (ok) atomicAdd(&Fs[3 * j + a], -f);
      }
      if (ok) e_acc += static_cast<double>(ew);
      sg[0] -= static_cast<double>(cw * d[0] * rh[0]);
      sg[1] -= static_cast<double>(cw * d[1] * rh[1]);
      sg[2] -= static_cast<double>(cw * d[2] * rh[2]);
      sg[3] -= static_cast<double>(cw * d[0] * rh[1]);
      sg[4] -= static_cast<double>(cw * d[0] * rh[2]);
      sg[5] -= static_cast<double>(cw * d[1] * rh[2]);
    }
  }
  // ---- G4, G5: one thread per neighbour pair (j < k) of a central atom i,
  // in warp-sized runs as above
  if (L.n4 + L.n5 > 0)
    for (int w0 = threadIdx.x - lane; w0 < ntri; w0 += blockDim.x) {
      const int w = min(w0 + lane, ntri - 1);
      const int i = owner_of(tfirst, N, w);
      const int n = pfirst[i + 1] - pfirst[i];
      int u = w - tfirst[i], a0 = 0;
      pair_row(n, u, a0);
      const int pj = pfirst[i] + a0, pk = pj + 1 + u;
      int j, k;
      T d1[3], d2[3];
      pair_vec(wpos, shift, i, nbp[pj], j, d1[0], d1[1], d1[2]);
      const T r1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
      bool ok = w0 + lane < ntri && r1 >= T(1e-14) && r1 < rc;
      pair_vec(wpos, shift, i, nbp[pk], k, d2[0], d2[1], d2[2]);
      const T r2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
      ok = ok && r2 >= T(1e-14) && r2 < rc;
      if (!__any_sync(0xffffffffu, ok)) continue;
      const int ti = typ[i];
      const T *w_ = W + ti * (L.S + 1);
      const int *cl = col + ti * (L.S + 1);
      const T ir1 = ok ? ac_rcp(r1) : T(0), ir2 = ok ? ac_rcp(r2) : T(0);
      const T h1[3] = {d1[0] * ir1, d1[1] * ir1, d1[2] * ir1}, h2[3] = {d2[0] * ir2, d2[1] * ir2, d2[2] * ir2};
      T costh = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) * (ir1 * ir2);
      costh = min(max(costh, T(-1)), T(1));
      const T djk[3] = {d2[0] - d1[0], d2[1] - d1[1], d2[2] - d1[2]};
      const T rjk = sqrt(djk[0] * djk[0] + djk[1] * djk[1] + djk[2] * djk[2]);
      T hjk[3] = {T(0), T(0), T(0)};
      if (rjk > T(1e-14)) {
        const T irjk = ac_rcp(rjk);
        for (int a = 0; a < 3; ++a) hjk[a] = djk[a] * irjk;
      }
      T f1, fp1, f2, fp2, fjk, fpjk;
      ac_fc(r1, rc, prc, f1, fp1);
      ac_fc(r2, rc, prc, f2, fp2);
      ac_fc(rjk, rc, prc, fjk, fpjk);
      T dcj[3], dck[3];
      for (int a = 0; a < 3; ++a) {
        dcj[a] = (h2[a] - costh * h1[a]) * ir1;
        dck[a] = (h1[a] - costh * h2[a]) * ir2;
      }
      const int po = pair_ord(typ[j], typ[k], nt);
      bool hi = false, hj = false;
      const unsigned xi = run_links(i, lane, hi);
      const unsigned xj = run_links(pj, lane, hj); // atom j: runs of the same neighbour slot
      const bool iw = __all_sync(0xffffffffu, i == __shfl_sync(0xffffffffu, i, 0)); // one atom i for the warp
      T GJ[3] = {0, 0, 0}, GK[3] = {0, 0, 0}, ew = T(0);
      auto term = [&](int idx, T eta, T zeta, T lambda, T Cz, bool with_jk) {
        const T Aa = T(1) + lambda * costh;
        const bool on = ok && Aa > T(1e-12);
        // 2^{1−ζ} per function (precomputed); ζ λ A^{ζ−1} = ζ λ A^ζ / A (A > 1e-12)
        const T Ab = on ? Aa : T(1);
        const T C = Cz, ang = ac_pow(Ab, zeta), dang = zeta * lambda * ang * ac_rcp(Ab);
        const T rsum = r1 * r1 + r2 * r2 + (with_jk ? rjk * rjk : T(0));
        const T rad = ac_exp(-eta * rsum);
        const T fj = with_jk ? fjk : T(1);
        const T fcs = f1 * f2 * fj;
        const T g = C * ang * rad * fcs;
        const T cij = C * ang * (rad * (T(-2) * eta * r1) * fcs + rad * fp1 * f2 * fj);
        const T cik = C * ang * (rad * (T(-2) * eta * r2) * fcs + rad * f1 * fp2 * fj);
        const T cjk = with_jk ? C * ang * (rad * (T(-2) * eta * rjk) * fcs + rad * f1 * f2 * fpjk) : T(0);
        const T ccos = C * rad * fcs * dang;
        T gj[3], gk[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          gj[a] = cij * h1[a] - cjk * hjk[a] + ccos * dcj[a];
          gk[a] = cik * h2[a] + cjk * hjk[a] + ccos * dck[a];
        }
        if constexpr (DESC) {
          if (on) atomicAdd(&A.desc[(static_cast<int64_t>(cd.atom0) + i) * L.S + idx], static_cast<double>(g));
        } else if constexpr (JAC) {
          // rows: j gets −gj, k gets −gk, i gets gj + gk; stress d1 ⊗ −gj + d2 ⊗ −gk
          // (standardized: the column of w_idx scales by inv_std_idx)
          const T sv = ivs ? ivs[ti * L.S + idx] : T(1);
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            gj[a] = on ? gj[a] * sv : T(0);
            gk[a] = on ? gk[a] * sv : T(0);
          }
          const T st[6] = {-sw * (d1[0] * gj[0] + d2[0] * gk[0]), -sw * (d1[1] * gj[1] + d2[1] * gk[1]),
                           -sw * (d1[2] * gj[2] + d2[2] * gk[2]), -sw * (d1[0] * gj[1] + d2[0] * gk[1]),
                           -sw * (d1[0] * gj[2] + d2[0] * gk[2]), -sw * (d1[1] * gj[2] + d2[1] * gk[2])};
          const int cc = cl[idx];
          const int c0 = __shfl_sync(0xffffffffu, cc, 0);
          if (__all_sync(0xffffffffu, cc == c0)) {
            if (c0 < 0) return;
            if (iw) { // atom i's three rows by halving exchanges (lanes 8a hold row a)
              const T v[4] = {gj[0] + gk[0], gj[1] + gk[1], gj[2] + gk[2], T(0)};
              const T t = warp_sum_tr<4>(v, lane);
              if ((lane & 7) == 0 && lane < 24) jadd(c0, 3 * i + (lane >> 3), t);
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              if (!iw) {
                const T ti_ = run_sum(gj[a] + gk[a], xi);
                if (hi) jadd(c0, 3 * i + a, ti_);
              }
              const T tj = run_sum(gj[a], xj);
              if (hj) jadd(c0, 3 * j + a, -tj);
              if (on) jadd(c0, 3 * k + a, -gk[a]);
            }
            erows_warp(c0, on ? g * sv : T(0), st);
          } else if (on && cc >= 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              jadd(cc, 3 * i + a, gj[a] + gk[a]);
              jadd(cc, 3 * j + a, -gj[a]);
              jadd(cc, 3 * k + a, -gk[a]);
            }
            erows_lane(cc, g * sv, st);
          }
        } else if (on) {
          ew += w_[idx] * g;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            GJ[a] += w_[idx] * gj[a];
            GK[a] += w_[idx] * gk[a];
          }
        }
      };
      for (int t = 0; t < L.n4; ++t)
        term(L.base[3] + po * L.n4 + t, p4[3 * t], p4[3 * t + 1], p4[3 * t + 2], c4[t], true);
      for (int t = 0; t < L.n5; ++t)
        term(L.base[4] + po * L.n5 + t, p5[3 * t], p5[3 * t + 1], p5[3 * t + 2], c5[t], false);
      if constexpr (MODE == 0) {
        // atoms i and j summed over their runs of lanes (zeros without a term)
        if (iw) { // one atom i for the warp: halving exchanges (lanes 8a hold component a)
          const T v[4] = {GJ[0] + GK[0], GJ[1] + GK[1], GJ[2] + GK[2], T(0)};
          const T t = warp_sum_tr<4>(v, lane);
          if ((lane & 7) == 0 && lane < 24) atomicAdd(&Fs[3 * i + (lane >> 3)], t);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          if (!iw) {
            const T ti_ = run_sum(GJ[a] + GK[a], xi);
            if (hi) atomicAdd(&Fs[3 * i + a], ti_);
          }
          const T tj = run_sum(GJ[a], xj);
          if (hj) atomicAdd(&Fs[3 * j + a], -tj);
          if (ok) atomicAdd(&Fs[3 * k + a], -GK[a]);
        }
        e_acc += static_cast<double>(ew);
        sg[0] -= static_cast<double>(d1[0] * GJ[0] + d2[0] * GK[0]);
        sg[1] -= static_cast<double>(d1[1] * GJ[1] + d2[1] * GK[1]);
        sg[2] -= static_cast<double>(d1[2] * GJ[2] + d2[2] * GK[2]);
        sg[3] -= static_cast<double>(d1[0] * GJ[1] + d2[0] * GK[1]);
        sg[4] -= static_cast<double>(d1[0] * GJ[2] + d2[0] * GK[2]);
        sg[5] -= static_cast<double>(d1[1] * GJ[2] + d2[1] * GK[2]);
      }
    }
  if constexpr (DESC) return;
  // biases: one per atom
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int ti = typ[i];
    if constexpr (JAC) {
      const int cb = col[ti * (L.S + 1) + L.S];
      if (cb >= 0) atomicAdd(&E64[cb], A.w_e);
      if (ntyp) atomicAdd(&ntyp[ti], 1);
    } else {
      e_acc += static_cast<double>(W[ti * (L.S + 1) + L.S]);
    }
  }
  if constexpr (JAC) {
    __syncthreads();
    if (ivs) // standardized: ∂E/∂w_k also holds −inv_std_k·mean_k per atom of the species
      for (int q = threadIdx.x; q < nt * L.S; q += blockDim.x) {
        const int t = q / L.S, kk = q % L.S;
        const int ck = col[t * (L.S + 1) + kk];
        if (ck < 0 || ntyp[t] == 0) continue;
        const double mu = A.vals[A.c.desc[1 + nt + t].pv0 + kk];
        atomicAdd(&E64[ck], -A.w_e * static_cast<double>(ivs[q]) * mu * ntyp[t]);
      }
    __syncthreads();
    // the energy and stress rows to J (J is zeroed; this CTA owns them)
    for (int q = threadIdx.x; q < nrow * A.D; q += blockDim.x) {
      const int m = q / A.D, cl = q % A.D;
      A.J[static_cast<int64_t>(cl) * A.ld + row0 + rE + m] = static_cast<T>(E64[q]);
    }
    if (!Jb) return;
    __syncthreads();
    // the force rows to J (the limit row stays zero)
    for (int k = threadIdx.x; k < 3 * N * A.D; k += blockDim.x) {
      const int cl = k / (3 * N), r = k % (3 * N);
      A.J[static_cast<int64_t>(cl) * A.ld + row0 + r] = Jb[r * A.D + cl];
    }
    return;
  }
  __syncthreads();
  // residual rows of the configuration (residual_layout.hpp:37-54)
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
    const double E = sums[0], iv = 1.0 / cd.volume;
    double st[6];
    for (int a = 0; a < 6; ++a) st[a] = sums[1 + a] * iv;
    int64_t row = rowE;
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
    A.F[row++] = 0.0; // ML models have no embedding range penalty
    A.obj_part[c] = o;
    if (A.energy) A.energy[c] = E;
    if (A.limit) A.limit[c] = 0.0;
    if (A.stress9) { // the configuration's virial is symmetric: upper triangle mirrored
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

__global__ void ac_sum_parts(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double r[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, r);
  if (threadIdx.x == 0) *out = s;
}

template <class T> size_t ac_smem(const fs_gpu *h, int mi) {
  AcLayout L;
  L.init(h->tables[0].v.data(), h->ntypes);
  const int N = h->max_natoms, nt = h->ntypes, nspec = h->tables[0].n;
  return align16(nspec * sizeof(T)) + align16(nt * (L.S + 1) * sizeof(T)) + align16(nt * (L.S + 1) * sizeof(int)) +
         align16((L.n4 + L.n5) * sizeof(T)) +
         align16(3 * N * sizeof(double)) + align16(3 * mi * sizeof(double)) + align16(N) + align16(3 * N * sizeof(T)) +
         align16(8 * 32 * sizeof(double)) + 2 * align16((N + 1) * sizeof(int)) + align16(32 * sizeof(int)) +
         align16(nt * L.S * sizeof(T)) + align16(nt * sizeof(int)) + 192;
}

// Σ D, Σ D² and the atom count of species q / S for descriptor q % S
// (CTA q), in FP64 and a fixed order; out = [Σ D | Σ D² | count] × (nt·S)
__global__ void ac_desc_stats(const double *__restrict__ Dsc, const int32_t *__restrict__ type, int64_t n_atoms,
                              int S, double *__restrict__ out) {
  __shared__ double r[32];
  const int q = blockIdx.x, t = q / S, k = q % S;
  double s1 = 0.0, s2 = 0.0, n = 0.0;
  for (int64_t i = threadIdx.x; i < n_atoms; i += blockDim.x)
    if (type[i] == t) {
      const double v = Dsc[i * S + k];
      s1 += v;
      s2 += v * v;
      n += 1.0;
    }
  s1 = block_sum(s1, r);
  s2 = block_sum(s2, r);
  n = block_sum(n, r);
  if (threadIdx.x == 0) {
    out[q] = s1;
    out[gridDim.x + q] = s2;
    out[2 * gridDim.x + q] = n;
  }
}

// mode 0: residual; 1: Jacobian rows (+ Jᵀr); 2: descriptors into desc
template <class T> int launch_acsf(fs_gpu *h, double w_e, double w_s, int mode, double *desc = nullptr) {
  const bool jac = mode == 1;
  AcArgs<T> a;
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
  a.order = h->d_cfg_by_work;
  a.J = nullptr;
  a.ld = 0;
  a.D = h->D;
  a.smj = 0;
  a.std_on = static_cast<int>(h->tables.size()) == 1 + 2 * h->ntypes ? 1 : 0;
  a.desc = desc;
  int mi = 1;
  for (const CfgDev &cd : h->cfg_host) mi = std::max(mi, (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1));
  size_t sm = ac_smem<T>(h, mi);
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "ACSF: configuration too large for shared memory");
  const int64_t M = rows_of(h, w_s);
  const int D = h->D;
  if (jac) {
    // the Jacobian mode adds the FP64 energy and stress rows (7 × D doubles)
    const size_t e64 = align16(static_cast<size_t>(7) * D * sizeof(double));
    if (sm + e64 > 227 * 1024)
      return set_error(h, FS_ERR_UNSUPPORTED,
                       "ACSF Jacobian: " + std::to_string(sm + e64) + " bytes of shared memory for D = " +
                           std::to_string(D) + " and " + std::to_string(h->max_natoms) +
                           " atoms in the largest configuration (the limit is 232448)");
    const int64_t ldj = (M + 31) / 32 * 32;
    const size_t jn = static_cast<size_t>(ldj) * D;
    if (static_cast<size_t>(h->jac_alloc) != jn || h->ldj != ldj || !h->d_J || h->j_rowmajor) {
      if (h->d_J) cudaFree(h->d_J);
      h->d_J = nullptr;
      FS_CUDA(cudaMalloc(&h->d_J, std::max<size_t>(jn, 1) * sizeof(T)));
      h->jac_alloc = static_cast<int64_t>(jn);
      h->ldj = ldj;
      h->j_rowmajor = false;
    }
    if (!h->d_JtJ) {
      FS_CUDA(cudaMalloc(&h->d_JtJ, std::max(D * D, 1) * sizeof(double)));
      FS_CUDA(cudaMalloc(&h->d_Jtr, std::max(D, 1) * sizeof(double)));
    }
    FS_CUDA(cudaMemsetAsync(h->d_J, 0, std::max<size_t>(jn, 1) * sizeof(T), h->stream));
    a.J = static_cast<T *>(h->d_J);
    a.ld = ldj;
    sm += e64;
    // the configuration's J block in shared memory when it fits
    const size_t jb = align16(static_cast<size_t>(3 * h->max_natoms) * D * sizeof(T));
    if (D > 0 && sm + jb <= 200 * 1024) {
      a.smj = 1;
      sm += jb;
    }
  }
  auto k = mode == 1 ? acsf_kernel<T, 1> : mode == 2 ? acsf_kernel<T, 2> : acsf_kernel<T, 0>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, kAcThreads, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  if (mode == 2) return FS_OK;
  if (jac) {
    if (D > 0) {
      FS_TRY(launch_jtr<T>(h, static_cast<const T *>(h->d_J), h->ldj, M, D, h->d_F, h->d_Jtr));
    }
  } else {
    ac_sum_parts<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  return FS_OK;
}

} // namespace

int eval_residual_acsf(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_acsf<double>(h, w_e, w_s, 0) : launch_acsf<float>(h, w_e, w_s, 0);
}
int eval_jacobian_acsf(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_acsf<double>(h, w_e, w_s, 1) : launch_acsf<float>(h, w_e, w_s, 1);
}

// Per-species descriptor statistics (MLBase::compute_standardization,
// ml_force.hpp:644-688): the descriptors of every atom (formed in the context
// precision, summed in FP64), then Σ D and Σ D² per (species, descriptor).
int lmbtr_descriptors(fs_gpu *h, double *desc);

int acsf_standardization(fs_gpu *h, double *mean, double *inv_std, int64_t *count) {
  const bool lm = h->family == FS_FAMILY_LMBTR;
  AcLayout L;
  L.init(h->tables[0].v.data(), h->ntypes);
  const double *lv = h->tables[0].v.data();
  const int nt = h->ntypes;
  const int S = lm ? nt * static_cast<int>(lv[3]) + nt * (nt + 1) / 2 * static_cast<int>(lv[7]) : L.S;
  const int64_t na = h->n_atoms;
  double *d_desc = nullptr, *d_out = nullptr;
  FS_CUDA(cudaMalloc(&d_desc, std::max<int64_t>(na * S, 1) * sizeof(double)));
  if (cudaMalloc(&d_out, std::max(3 * nt * S, 1) * sizeof(double)) != cudaSuccess) {
    cudaFree(d_desc);
    return set_error(h, FS_ERR_NOMEM, "cudaMalloc (ACSF statistics)");
  }
  int rc = FS_OK;
  std::vector<double> out(static_cast<size_t>(3) * nt * S);
  do {
    if (cudaMemsetAsync(d_desc, 0, std::max<int64_t>(na * S, 1) * sizeof(double), h->stream) != cudaSuccess) {
      rc = set_error(h, FS_ERR_CUDA, "cudaMemsetAsync");
      break;
    }
    rc = lm                             ? lmbtr_descriptors(h, d_desc)
         : h->precision == FS_PREC_FP64 ? launch_acsf<double>(h, 1.0, 0.0, 2, d_desc)
                                        : launch_acsf<float>(h, 1.0, 0.0, 2, d_desc);
    if (rc != FS_OK) break;
    if (nt * S > 0) {
      ac_desc_stats<<<nt * S, 256, 0, h->stream>>>(d_desc, h->d_type, na, S, d_out);
      ++h->launches;
      if (cudaGetLastError() != cudaSuccess ||
          cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream) !=
              cudaSuccess ||
          cudaStreamSynchronize(h->stream) != cudaSuccess) {
        rc = set_error(h, FS_ERR_CUDA, "ACSF statistics");
        break;
      }
    }
  } while (false);
  cudaFree(d_desc);
  cudaFree(d_out);
  if (rc != FS_OK) return rc;
  // mean = Σ D / n, σ² = Σ D² / n − mean², inv_std = σ² > 1e-12 ? 1/σ : 0; no atoms: identity
  for (int t = 0; t < nt; ++t) {
    const double n = nt * S > 0 ? out[2 * nt * S + t * S] : 0.0;
    count[t] = static_cast<int64_t>(n);
    for (int k = 0; k < S; ++k) {
      const size_t q = static_cast<size_t>(t) * S + k;
      if (n == 0.0) {
        mean[q] = 0.0;
        inv_std[q] = 1.0;
        continue;
      }
      const double mu = out[q] / n, var = out[nt * S + q] / n - mu * mu;
      mean[q] = mu;
      inv_std[q] = var > 1e-12 ? 1.0 / std::sqrt(var) : 0.0;
    }
  }
  return FS_OK;
}

} // namespace fsg
