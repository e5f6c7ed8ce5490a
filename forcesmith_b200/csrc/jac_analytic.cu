// Exact parameter Jacobian of EAM and pair models whose tables are all
// analytic forms: the chain rule of EAMForceCalculator::write_param_jacobian
// (src/force/eam_force.cpp:108-279) and PairForceCalculator::
// write_param_jacobian (src/force/pair_force.cpp:80-111), with the per-form
// partials param_grad / dderiv_dparam / deriv2 (analytic_potential.hpp:
// 238-250) taken from the hyper-dual forms of forms_dev.cuh.  The reference
// uses this path exactly when every table is analytic (ForcesmithFunctor::df,
// src/optimization/forcesmith_functor.cpp:265-277); mixed models keep central
// differences.
//
// Two kernels per evaluation, one CTA per configuration:
//   an_atoms_kernel (EAM)  thread per atom: ρ_i, the embedding clamp, F'(ρ̄),
//                          F''(ρ̄), ∂ρ_i/∂θ over the density columns, and
//                          ∂F(ρ̄)/∂θ, ∂F'(ρ̄)/∂θ over the atom's embedding
//                          columns
//   an_rows_kernel         warp per atom, lane per column: the atom's three
//                          force rows, and per-column sums of the energy,
//                          stress and limit rows, added over warps in a fixed
//                          order at the end
// J is column-major (leading dimension the row count rounded up to 32); the
// columns are few (a handful of parameters per table), so a lane per column
// with the form's partial for its own parameter is the natural mapping.
#include "jtr.cuh"
#include "kern_common.cuh"

#include <algorithm>
#include <vector>

namespace fsg {
namespace {

// What a column is: the table and parameter it differentiates, its role and
// the role's species slot (pair ordinal for pair tables).
enum { kRolePair = 0, kRoleDens = 1, kRoleEmb = 2 };

template <class T> struct AnArgs {
  Common c;
  const int4 *cols; // per column: {table, parameter, role, slot}
  int D, dens0, ndens, emb0, nemb;
  double w_e, w_s;
  int max_img;
  // per-atom data (EAM): F'(ρ̄), F''(ρ̄) (0 when clamped), clamp penalty slope
  T *gF, *cF;
  double *over;
  T *drho;  // [atom][ndens]   ∂ρ_i/∂θ
  T *demb;  // [atom][nemb]    ∂F(ρ̄_i)/∂θ  (the atom's own embedding table)
  T *dgrad; // [atom][nemb]    ∂F'(ρ̄_i)/∂θ
  T *J;
  int64_t ld;
};

// Partials of a table's form at r with respect to its parameter k:
// (∂v/∂θ_k, ∂²v/∂r∂θ_k); zero where the form is identically zero.
template <class T>
__device__ __forceinline__ Hd<T> form_partial(const STab<T> &tb, const double *vals, T r, int k) {
  const double *pp = vals + tb.pv0;
  if (form_outside<T>(tb.form, pp, r)) return hd_c(T(0));
  return form_seeded<T>(tb.form, pp, tb.n, r, tb.xmax, T(0), k);
}

template <class T>
__device__ __forceinline__ T form_deriv(const STab<T> &tb, const double *vals, T r) {
  return form_vd<T>(tb.form, vals + tb.pv0, tb.n, r, tb.xmax).d;
}

template <class T> __global__ void __launch_bounds__(256) an_atoms_kernel(AnArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  Smem S(smem_raw);
  STab<T> *tabs = S.take<STab<T>>(A.c.n_tables);
  int32_t *cmap = S.take<int32_t>(A.c.n_cmap);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * A.max_img);
  uint8_t *typ = S.take<uint8_t>(N);
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  for (int k = threadIdx.x; k < A.c.n_cmap; k += blockDim.x) cmap[k] = A.c.cmap[k];
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();
  const int32_t *start = A.c.nb_start + cd.atom0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
    T *dr = A.drho + ga * A.ndens;
    for (int m = 0; m < A.ndens; ++m) dr[m] = T(0);
    // ρ_i and ∂ρ_i/∂θ (closed gate, eam_force.cpp:59-66)
    T rho = T(0);
    for (int p = start[i]; p < start[i + 1]; ++p) {
      int j;
      T dx, dy, dz;
      const double r64 = pair_vec_len(wpos, shift, i, A.c.nb_pack[p], j, dx, dy, dz);
      const STab<T> &g = tabs[np + typ[j]];
      if (!gate64(g, r64)) continue;
      const T r = static_cast<T>(r64);
      rho += form_vd<T>(g.form, A.c.vals + g.pv0, g.n, r, g.xmax).v;
      for (int k = 0; k < g.n; ++k) {
        const int col = cmap[g.cmap0 + k];
        if (col >= 0) dr[col - A.dens0] += form_partial(g, A.c.vals, r, k).c;
      }
    }
    // clamp_embedding (kernels.hpp:19-31): a ρ outside the embedding span is
    // clamped, and its ρ-derivatives go to the limit row (eam_force.cpp:151-190)
    const int ti = typ[i];
    const STab<T> &te = tabs[np + nt + ti];
    T rb = rho;
    double over = 0.0;
    if (rb > te.xmax) {
      over = 2.0 * 100.0 * 10.0 * (static_cast<double>(rb) - static_cast<double>(te.xmax));
      rb = te.xmax;
    } else if (rb < te.x0) {
      over = -2.0 * 100.0 * 10.0 * (static_cast<double>(te.x0) - static_cast<double>(rb));
      rb = te.x0;
    }
    const double *pe = A.c.vals + te.pv0;
    const Hd<T> f = form_seeded<T>(te.form, pe, te.n, rb, te.xmax, T(1), -1); // F, F', F''
    A.gF[ga] = f.b;
    A.cF[ga] = over != 0.0 ? T(0) : f.d;
    A.over[ga] = over;
    T *de = A.demb + ga * A.nemb, *dg = A.dgrad + ga * A.nemb;
    for (int m = 0; m < A.nemb; ++m) de[m] = dg[m] = T(0);
    for (int k = 0; k < te.n; ++k) {
      const int col = cmap[te.cmap0 + k];
      if (col < 0) continue;
      const Hd<T> q = form_seeded<T>(te.form, pe, te.n, rb, te.xmax, T(0), k);
      de[col - A.emb0] = q.c;
      dg[col - A.emb0] = q.d;
    }
  }
}

constexpr int kAnWarps = 8;

// Force rows of each atom and the configuration's energy / stress / limit
// rows.  Per pair (i, j, d = x_j + s − x_i) the force scalar is
//   φ'_{ti tj}(r) + F'_i ρ'_{tj}(r) + F'_j ρ'_{ti}(r)
// and the lane for column θ adds its partial (param_jacobian.hpp:91-122):
//   pair table φ_{ti tj}:  ∂φ'/∂θ                 (energy: ½ ∂φ/∂θ)
//   density ρ_{tj} / ρ_{ti}: F'_i ∂ρ'_{tj}/∂θ, F'_j ∂ρ'_{ti}/∂θ
//   every density column:  F''_i ∂ρ_i/∂θ ρ'_{tj} + F''_j ∂ρ_j/∂θ ρ'_{ti}
//   embedding columns:     ∂F'_i/∂θ ρ'_{tj} + ∂F'_j/∂θ ρ'_{ti}
// times d/r; stress adds −w_s ½ d ⊗ ∂f / V.  Per atom the energy row gains
// ∂F_i/∂θ and F'_i ∂ρ_i/∂θ (or, for a clamped atom, the limit row its
// penalty slope times ∂ρ_i/∂θ).
template <class T, bool EAM> __global__ void __launch_bounds__(kAnWarps * 32) an_rows_kernel(AnArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms, D = A.D;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  Smem S(smem_raw);
  STab<T> *tabs = S.take<STab<T>>(A.c.n_tables);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * A.max_img);
  uint8_t *typ = S.take<uint8_t>(N);
  // per warp and column: energy, 6 stress, limit (FP64)
  double *acc = S.take<double>(static_cast<size_t>(kAnWarps) * 8 * D);
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  for (int k = threadIdx.x; k < kAnWarps * 8 * D; k += blockDim.x) acc[k] = 0.0;
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int32_t *start = A.c.nb_start + cd.atom0;
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  double *my = acc + static_cast<size_t>(w) * 8 * D;
  for (int i = w; i < N; i += kAnWarps) {
    const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
    const int ti = typ[i];
    T gFi = T(0), cFi = T(0);
    double overi = 0.0;
    if constexpr (EAM) {
      gFi = A.gF[ga];
      cFi = A.cF[ga];
      overi = A.over[ga];
    }
    for (int c0 = 0; c0 < D; c0 += 32) {
      const int col = c0 + lane;
      const bool live = col < D;
      const int4 ci = live ? A.cols[col] : make_int4(0, 0, -1, 0);
      const STab<T> &tc = tabs[ci.x];
      const int dm = ci.z == kRoleDens ? col - A.dens0 : 0;
      const int em = ci.z == kRoleEmb ? col - A.emb0 : 0;
      T f[3] = {T(0), T(0), T(0)};
      double e = 0.0, s[6] = {0, 0, 0, 0, 0, 0};
      for (int p = start[i]; p < start[i + 1]; ++p) {
        int j;
        T d[3];
        const double r64 = pair_vec_len(wpos, shift, i, A.c.nb_pack[p], j, d[0], d[1], d[2]);
        if (r64 < 1e-14) continue;
        const T r = static_cast<T>(r64), ir = T(1) / r;
        const int tj = typ[j];
        const int64_t gj = static_cast<int64_t>(cd.atom0) + j;
        T cf = T(0);
        if (ci.z == kRolePair && ci.w == pair_ord(ti, tj, nt) && (EAM ? gate64(tc, r64) : gate64<false>(tc, r64))) {
          const Hd<T> q = form_partial(tc, A.c.vals, r, ci.y);
          cf += q.d;
          e += 0.5 * static_cast<double>(q.c);
        }
        if constexpr (EAM) {
          const STab<T> &g_j = tabs[np + tj], &g_i = tabs[np + ti];
          const bool in_j = gate64(g_j, r64), in_i = gate64(g_i, r64);
          const T rp_j = in_j ? form_deriv(g_j, A.c.vals, r) : T(0); // ρ'_{tj}(r)
          const T rp_i = in_i ? form_deriv(g_i, A.c.vals, r) : T(0); // ρ'_{ti}(r)
          if (ci.z == kRoleDens) {
            const T w_dir = (ci.w == tj && in_j ? gFi : T(0)) + (ci.w == ti && in_i ? A.gF[gj] : T(0));
            if (w_dir != T(0)) cf += w_dir * form_partial(tc, A.c.vals, r, ci.y).d;
            cf += cFi * A.drho[ga * A.ndens + dm] * rp_j + A.cF[gj] * A.drho[gj * A.ndens + dm] * rp_i;
          } else if (ci.z == kRoleEmb) {
            cf += A.dgrad[ga * A.nemb + em] * rp_j + A.dgrad[gj * A.nemb + em] * rp_i;
          }
        }
        if (cf != T(0)) {
          const T sc = cf * ir;
          const T df[3] = {sc * d[0], sc * d[1], sc * d[2]};
          for (int a = 0; a < 3; ++a) f[a] += df[a];
          s[0] += static_cast<double>(d[0] * df[0]);
          s[1] += static_cast<double>(d[1] * df[1]);
          s[2] += static_cast<double>(d[2] * df[2]);
          s[3] += static_cast<double>(d[0] * df[1]);
          s[4] += static_cast<double>(d[0] * df[2]);
          s[5] += static_cast<double>(d[1] * df[2]);
        }
      }
      if (!live) continue;
      double lim = 0.0;
      if constexpr (EAM) {
        if (ci.z == kRoleEmb && ci.w == ti) e += static_cast<double>(A.demb[ga * A.nemb + em]);
        if (ci.z == kRoleDens) {
          const double dd = static_cast<double>(A.drho[ga * A.ndens + dm]);
          if (overi != 0.0) lim += overi * dd;
          else e += static_cast<double>(gFi) * dd;
        }
      }
      T *Jc = A.J + static_cast<int64_t>(col) * A.ld + row0 + 3 * i;
      Jc[0] = f[0];
      Jc[1] = f[1];
      Jc[2] = f[2];
      double *mc = my + 8 * col;
      mc[0] += e;
      for (int v = 0; v < 6; ++v) mc[1 + v] += s[v];
      mc[7] += lim;
    }
  }
  __syncthreads();
  // the configuration's energy, stress and limit rows: warps added in order
  const int64_t rE = row0 + 3 * N, rL = rE + 1 + (A.w_s > 0.0 ? 6 : 0);
  const double sc = -A.w_s * 0.5 / cd.volume;
  for (int col = threadIdx.x; col < D; col += blockDim.x) {
    double v8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int ww = 0; ww < kAnWarps; ++ww)
      for (int k = 0; k < 8; ++k) v8[k] += acc[static_cast<size_t>(ww) * 8 * D + 8 * col + k];
    T *Jc = A.J + static_cast<int64_t>(col) * A.ld;
    Jc[rE] = static_cast<T>(A.w_e * v8[0]);
    if (A.w_s > 0.0)
      for (int v = 0; v < 6; ++v) Jc[rE + 1 + v] = static_cast<T>(sc * v8[1 + v]);
    Jc[rL] = static_cast<T>(v8[7]);
  }
}

template <class T> int launch_analytic(fs_gpu *h, double w_e, double w_s) {
  const bool eam = h->family == FS_FAMILY_EAM;
  const int D = h->D, nt = h->ntypes, np = npair_of(nt);
  const int64_t M = rows_of(h, w_s);
  // columns: table, parameter, role, slot (pair ordinal or species)
  std::vector<int4> cols(std::max(D, 1));
  int dens0 = D, dens1 = 0, emb0 = D, emb1 = 0;
  for (int t = 0; t < static_cast<int>(h->tables.size()); ++t) {
    const HostTable &ht = h->tables[t];
    const int role = t < np ? kRolePair : (t < np + nt ? kRoleDens : kRoleEmb);
    const int slot = t < np ? t : (t < np + nt ? t - np : t - np - nt);
    for (int k = 0; k < ht.n; ++k) {
      const int col = ht.cols[k];
      if (col < 0) continue;
      cols[col] = make_int4(t, k, role, slot);
      if (role == kRoleDens) dens0 = std::min(dens0, col), dens1 = std::max(dens1, col + 1);
      if (role == kRoleEmb) emb0 = std::min(emb0, col), emb1 = std::max(emb1, col + 1);
    }
  }
  const int ndens = std::max(0, dens1 - dens0), nemb = std::max(0, emb1 - emb0);
  if (dens0 == D) dens0 = 0;
  if (emb0 == D) emb0 = 0;
  // J (column-major, rows rounded up to 32; the padding rows stay zero)
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
  // column table and per-atom scratch, kept with the context; every block
  // is carved on a 256-byte boundary
  const size_t NA = static_cast<size_t>(std::max<int64_t>(h->n_atoms, 1));
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  size_t need = up(sizeof(int4) * cols.size());
  if (eam)
    need += up(NA * sizeof(double)) + 2 * up(NA * sizeof(T)) + up(NA * std::max(ndens, 1) * sizeof(T)) +
            2 * up(NA * std::max(nemb, 1) * sizeof(T));
  if (h->an_alloc < need || !h->d_an) {
    if (h->d_an) cudaFree(h->d_an);
    h->d_an = nullptr;
    h->an_alloc = 0;
    FS_CUDA(cudaMalloc(&h->d_an, need));
    h->an_alloc = need;
  }
  char *base = static_cast<char *>(h->d_an);
  auto carve = [&](size_t bytes) {
    char *p = base;
    base += up(bytes);
    return p;
  };
  AnArgs<T> a;
  a.c = make_common<T>(h);
  int4 *d_cols = reinterpret_cast<int4 *>(carve(sizeof(int4) * cols.size()));
  FS_CUDA(cudaMemcpyAsync(d_cols, cols.data(), sizeof(int4) * cols.size(), cudaMemcpyHostToDevice, h->stream));
  a.cols = d_cols;
  a.D = D;
  a.dens0 = dens0;
  a.ndens = ndens;
  a.emb0 = emb0;
  a.nemb = nemb;
  a.w_e = w_e;
  a.w_s = w_s;
  a.max_img = max_images(h);
  a.over = eam ? reinterpret_cast<double *>(carve(NA * sizeof(double))) : nullptr;
  a.gF = eam ? reinterpret_cast<T *>(carve(NA * sizeof(T))) : nullptr;
  a.cF = eam ? reinterpret_cast<T *>(carve(NA * sizeof(T))) : nullptr;
  a.drho = eam ? reinterpret_cast<T *>(carve(NA * std::max(ndens, 1) * sizeof(T))) : nullptr;
  a.demb = eam ? reinterpret_cast<T *>(carve(NA * std::max(nemb, 1) * sizeof(T))) : nullptr;
  a.dgrad = eam ? reinterpret_cast<T *>(carve(NA * std::max(nemb, 1) * sizeof(T))) : nullptr;
  a.J = static_cast<T *>(h->d_J);
  a.ld = ldj;
  const int N = h->max_natoms, mi = a.max_img, nT = a.c.n_tables;
  mark(h, 2);
  if (eam) {
    const size_t sm = align16(nT * sizeof(STab<T>)) + align16(h->n_cmap * sizeof(int32_t)) +
                      align16(3 * N * sizeof(double)) + align16(3 * mi * sizeof(double)) + align16(N) + 64;
    if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "analytic Jacobian: configuration too large");
    FS_CUDA(cudaFuncSetAttribute(an_atoms_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
    an_atoms_kernel<T><<<h->n_cfg, 256, sm, h->stream>>>(a);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  const size_t sm = align16(nT * sizeof(STab<T>)) + align16(3 * N * sizeof(double)) + align16(3 * mi * sizeof(double)) +
                    align16(N) + align16(static_cast<size_t>(kAnWarps) * 8 * D * sizeof(double)) + 64;
  if (sm > 227 * 1024)
    return set_error(h, FS_ERR_UNSUPPORTED, "analytic Jacobian: " + std::to_string(D) + " columns and " +
                                                std::to_string(N) + " atoms need " + std::to_string(sm) +
                                                " bytes of shared memory (the limit is 232448)");
  auto k = eam ? an_rows_kernel<T, true> : an_rows_kernel<T, false>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, kAnWarps * 32, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  mark(h, 3);
  return launch_jtr<T>(h, static_cast<const T *>(h->d_J), ldj, M, D, h->d_F, h->d_Jtr);
}

} // namespace

// The Jacobian of an EAM or pair model whose tables are all analytic, in the
// context's precision.
int eval_jacobian_analytic(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_analytic<double>(h, w_e, w_s) : launch_analytic<float>(h, w_e, w_s);
}

} // namespace fsg
