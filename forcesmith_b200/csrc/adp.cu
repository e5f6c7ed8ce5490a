// Angular-dependent potential (ADP) residual on the device:
// ADPForceCalculator::eval_forces (src/force/adp_force.cpp:73-135).
//   pass 1: ρ_i = Σ ρ_{tj}(r), μ_i = Σ u_{ij}(r) d, λ_i = Σ w_{ij}(r) d dᵀ
//   pass 2: clamp, E_i = F(ρ̄_i) + ½|μ_i|² + ½(‖λ_i‖²_F − tr²λ_i/3), F'(ρ̄_i)
//   pass 3: f = (φ' + F'_i ρ'_{tj} + F'_j ρ'_{ti})/r d
//             + (u'/r (μ_i − μ_j)·d) d + u (μ_i − μ_j)
//             + (w'/r ν) d + 2 w ξ,  ν = Σ_{i,j} d·λd − |d|² trλ/3,
//             ξ = Σ_{i,j} λd − (trλ/3) d   (quad_nu / quad_xi, adp_force.hpp:63-69)
// Tables: pair[np], density[nt], embedding[nt], dipole[np], quadrupole[np],
// all makima splines with the closed range gate.
#include "kern_common.cuh"

#include <algorithm>

namespace fsg {
namespace {

template <class T> struct AdpArgs {
  Common c;
  const typename Vec4T<T>::type *seg_a;
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
};

template <class T, class R64>
__device__ __forceinline__ void gated(const STab<T> &tb, const typename Vec4T<T>::type *seg, T r, R64 &&r64, T &v,
                                      T &d) {
  v = d = T(0);
  T t;
  const int e = gate_seg(tb, r, t, r64);
  if (e < 0) return;
  v = seg_val<T>(seg[e], t);
  d = seg_der<T>(seg[e], t, tb.inv_h);
}

template <class T>
__global__ void __launch_bounds__(256) adp_residual_kernel(AdpArgs<T> A) {
  using T4 = typename Vec4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  Smem S(smem_raw);
  STab<T> *tabs = S.take<STab<T>>(A.c.n_tables);
  T4 *seg = S.take<T4>(A.c.n_segs);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  T *gF = S.take<T>(N);
  T *mu = S.take<T>(3 * N);
  T *lam = S.take<T>(9 * N);
  double *red = S.take<double>(64);
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  for (int k = threadIdx.x; k < A.c.n_segs; k += blockDim.x) seg[k] = A.seg_a[k];
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();
  const int32_t *start = A.c.nb_start + cd.atom0;
  double e_acc = 0.0, lim = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int ti = typ[i];
    T rho = T(0), m[3] = {0, 0, 0}, L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int p = start[i]; p < start[i + 1]; ++p) {
      int j;
      T d[3];
      const uint32_t pk = A.c.nb_pack[p];
      pair_vec(wpos, shift, i, pk, j, d[0], d[1], d[2]);
      const T r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r < T(1e-14)) continue;
      const auto r64 = [=] { return pair_len64(wpos, shift, i, pk); };
      const int tj = typ[j], pt = pair_ord(ti, tj, nt);
      T v, dv;
      gated(tabs[np + tj], seg, r, r64, v, dv);
      rho += v;
      gated(tabs[2 * nt + np + pt], seg, r, r64, v, dv); // dipole u_{ij}
      for (int a = 0; a < 3; ++a) m[a] += v * d[a];
      gated(tabs[2 * nt + 2 * np + pt], seg, r, r64, v, dv); // quadrupole w_{ij}
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) L[3 * a + b] += v * (d[a] * d[b]);
    }
    for (int a = 0; a < 3; ++a) mu[3 * i + a] = m[a];
    for (int k = 0; k < 9; ++k) lam[9 * i + k] = L[k];
    const STab<T> &te = tabs[np + nt + ti];
    T rb = rho;
    if (rb > te.xmax) {
      const double dd = static_cast<double>(rb) - static_cast<double>(te.xmax);
      lim += 1000.0 * dd * dd;
      rb = te.xmax;
    } else if (rb < te.x0) {
      const double dd = static_cast<double>(te.x0) - static_cast<double>(rb);
      lim += 1000.0 * dd * dd;
      rb = te.x0;
    }
    T t;
    const int e = seg_of(te, rb, t);
    gF[i] = seg_der<T>(seg[e], t, te.inv_h);
    double ei = static_cast<double>(seg_val<T>(seg[e], t));
    ei += 0.5 * static_cast<double>(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const double tr = static_cast<double>(L[0] + L[4] + L[8]);
    double sq = 0.0;
    for (int k = 0; k < 9; ++k) sq += static_cast<double>(L[k]) * static_cast<double>(L[k]);
    ei += 0.5 * (sq - tr * tr / 3.0);
    e_acc += ei;
  }
  __syncthreads();
  double objp = 0.0, sg[6] = {0, 0, 0, 0, 0, 0};
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int ti = typ[i];
    T f[3] = {0, 0, 0};
    double ep = 0.0;
    const T *Li = lam + 9 * i;
    const T trLi = (Li[0] + Li[4] + Li[8]) / T(3);
    for (int p = start[i]; p < start[i + 1]; ++p) {
      int j;
      T d[3];
      const uint32_t pk = A.c.nb_pack[p];
      pair_vec(wpos, shift, i, pk, j, d[0], d[1], d[2]);
      const T r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r < T(1e-14)) continue;
      const auto r64 = [=] { return pair_len64(wpos, shift, i, pk); };
      const T ir = T(1) / r;
      const int tj = typ[j], pt = pair_ord(ti, tj, nt);
      T phi, dphi, rj, drj, ri, dri, u, du, w, dw;
      gated(tabs[pt], seg, r, r64, phi, dphi);
      gated(tabs[np + tj], seg, r, r64, rj, drj);
      gated(tabs[np + ti], seg, r, r64, ri, dri);
      gated(tabs[2 * nt + np + pt], seg, r, r64, u, du);
      gated(tabs[2 * nt + 2 * np + pt], seg, r, r64, w, dw);
      T g[3];
      const T es = (dphi + gF[i] * drj + gF[j] * dri) * ir;
      const T *mi = mu + 3 * i, *mj = mu + 3 * j;
      const T dot = (mi[0] * d[0] + mi[1] * d[1] + mi[2] * d[2]) - (mj[0] * d[0] + mj[1] * d[1] + mj[2] * d[2]);
      const T *Lj = lam + 9 * j;
      const T trLj = (Lj[0] + Lj[4] + Lj[8]) / T(3);
      const T dd2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      T Ld_i[3], Ld_j[3];
      for (int a = 0; a < 3; ++a) {
        Ld_i[a] = Li[3 * a] * d[0] + Li[3 * a + 1] * d[1] + Li[3 * a + 2] * d[2];
        Ld_j[a] = Lj[3 * a] * d[0] + Lj[3 * a + 1] * d[1] + Lj[3 * a + 2] * d[2];
      }
      const T nu = (d[0] * Ld_i[0] + d[1] * Ld_i[1] + d[2] * Ld_i[2] - dd2 * trLi) +
                   (d[0] * Ld_j[0] + d[1] * Ld_j[1] + d[2] * Ld_j[2] - dd2 * trLj);
      for (int a = 0; a < 3; ++a) {
        const T xi = (Ld_i[a] - trLi * d[a]) + (Ld_j[a] - trLj * d[a]);
        g[a] = es * d[a] + (du * ir * dot) * d[a] + u * (mi[a] - mj[a]) + (dw * ir * nu) * d[a] + T(2) * w * xi;
        f[a] += g[a];
      }
      ep += static_cast<double>(phi);
      sg[0] -= 0.5 * d[0] * g[0];
      sg[1] -= 0.5 * d[1] * g[1];
      sg[2] -= 0.5 * d[2] * g[2];
      sg[3] -= 0.5 * d[0] * g[1];
      sg[4] -= 0.5 * d[0] * g[2];
      sg[5] -= 0.5 * d[1] * g[2];
    }
    const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
    for (int a = 0; a < 3; ++a) {
      const double fa = static_cast<double>(f[a]);
      const double res = fa - A.c.ref_force[3 * ga + a];
      A.F[row0 + 3 * i + a] = res;
      if (A.forces) A.forces[3 * ga + a] = fa;
      objp += res * res;
    }
    e_acc += 0.5 * ep;
  }
  const double E = block_sum(e_acc, red);
  const double Lm = block_sum(lim, red);
  double st[6];
  for (int a = 0; a < 6; ++a) st[a] = block_sum(sg[a], red);
  const double op = block_sum(objp, red);
  if (threadIdx.x == 0) {
    const double iv = 1.0 / cd.volume;
    for (int a = 0; a < 6; ++a) st[a] *= iv;
    int64_t row = row0 + 3 * N;
    double o = op;
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

template <class T> int launch_adp(fs_gpu *h, double w_e, double w_s) {
  using T4 = typename Vec4T<T>::type;
  for (const HostTable &t : h->tables)
    if (t.kind != FS_TABLE_SPLINE) return set_error(h, FS_ERR_UNSUPPORTED, "ADP: spline tables only in this build");
  AdpArgs<T> a;
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
  a.seg_a = static_cast<const T4 *>(h->d_seg_a);
  a.w_e = w_e;
  a.w_s = w_s;
  a.F = h->d_F;
  a.forces = h->d_forces;
  a.energy = h->d_energy;
  a.stress9 = h->d_stress9;
  a.limit = h->d_limit;
  a.obj_part = h->d_obj_part;
  int max_img = 1;
  for (const CfgDev &cd : h->cfg_host) max_img = std::max(max_img, (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1));
  const int N = h->max_natoms;
  const size_t sm = align16(a.c.n_tables * sizeof(STab<T>)) + align16(h->n_segs * 4 * sizeof(T)) +
                    align16(3 * N * sizeof(double)) + align16(3 * max_img * sizeof(double)) + align16(N) +
                    align16(N * sizeof(T)) + align16(3 * N * sizeof(T)) + align16(9 * N * sizeof(T)) +
                    align16(64 * sizeof(double)) + 128;
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "ADP: configuration too large for shared memory");
  FS_CUDA(cudaFuncSetAttribute(adp_residual_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(sm)));
  adp_residual_kernel<T><<<h->n_cfg, 256, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  adp_sum<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

} // namespace

int eval_residual_adp(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_adp<double>(h, w_e, w_s) : launch_adp<float>(h, w_e, w_s);
}

} // namespace fsg
