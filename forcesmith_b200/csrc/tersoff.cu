// Tersoff on the device: residual (forces, energy, stress, objective).
//
//   TersoffForceCalculator::eval_forces (src/force/tersoff_force.cpp:268-286),
//   per directed bond i→j with the (t_i, t_j) parameters p:
//     f_c(r) = 1 | ½ + ½ cos(π (r − R)/(S − R)) | 0 (fc_val / dfc_val :26-43),
//     V_R = A e^{−λr}, V_A = B e^{−μr} (make_bond :85-101),
//     ζ_ij = Σ_{k≠j} ω_ik f_c,ik(r_ik) g_ij(cos θ_ijk) with the (t_i, t_k)
//     cutoff and ω (add_zeta :103-128), g(c) = 1 + c²/d² − c²/(d² + (h − c)²)
//     (:45-61), b = (1 + (βζ)^n)^{−1/2n} (:63-83);
//     E += ½ f_c (V_R − b V_A), the radial pair force on i and its opposite on
//     j (accumulate_pair :135-151), then the ζ-gradient forces on i, j, k with
//     P = ½ f_c V_A ∂b/∂ζ (accumulate_three_body :153-206).
//   The reference's Jacobian for Tersoff is central differences; the device
//   keeps that method (fd.cu, FP64 contexts).
//
// One CTA per configuration; one thread per directed bond, taken flat from a
// block scan of the configuration's neighbour lists (so atoms with few or many
// neighbours cost the same lanes).  Each bond walks its central atom's other
// neighbours twice (ζ, then the three-body forces).  Forces accumulate in
// shared memory with atomics; energy and stress are per-thread FP64 sums.
#include "kern_common.cuh"

#include <algorithm>

namespace fsg {
namespace {

constexpr int kTsThreads = 256;
constexpr int kTsFields = 12; // A, B, λ, μ, β, n, c, d, h, R, S, ω

template <class T> __device__ __forceinline__ T cos_t(T x) { return cos(x); }
template <class T> __device__ __forceinline__ T sin_t(T x) { return sin(x); }
template <class T> __device__ __forceinline__ T pi_t() { return T(3.14159265358979323846); }

template <class T> __device__ __forceinline__ T ts_fc(T r, T R, T S) {
  if (r <= R) return T(1);
  if (r >= S) return T(0);
  return T(0.5) + T(0.5) * cos_t(pi_t<T>() * (r - R) / (S - R));
}
template <class T> __device__ __forceinline__ T ts_dfc(T r, T R, T S) {
  if (r <= R || r >= S) return T(0);
  return T(-0.5) * pi_t<T>() / (S - R) * sin_t(pi_t<T>() * (r - R) / (S - R));
}
// p: A, B, λ, μ, β, n, c, d, h, R, S, ω
template <class T> __device__ __forceinline__ T ts_g(T c, const T *p) {
  const T c2 = p[6] * p[6], d2 = p[7] * p[7], hc = p[8] - c;
  return T(1) + c2 / d2 - c2 / (d2 + hc * hc);
}
template <class T> __device__ __forceinline__ T ts_dg(T c, const T *p) {
  const T c2 = p[6] * p[6], d2 = p[7] * p[7], hc = p[8] - c;
  const T den = d2 + hc * hc;
  return T(-2) * c2 * hc / (den * den);
}
// b(ζ) and ∂b/∂ζ
template <class T> __device__ __forceinline__ void ts_b(T zeta, const T *p, T &b, T &db) {
  if (zeta == T(0)) {
    b = T(1);
    db = T(0);
    return;
  }
  const T bzn = pow(p[4] * zeta, p[5]);
  b = pow(T(1) + bzn, T(-0.5) / p[5]);
  db = T(-0.5) * b * bzn / (zeta * (T(1) + bzn));
}

template <class T> struct TsArgs {
  Common c;
  const double *vals; // all model values (FP64)
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
  const int32_t *order; // configurations by work, heaviest first
};

template <class T> __global__ void __launch_bounds__(kTsThreads) tersoff_kernel(TsArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = A.order ? A.order[blockIdx.x] : blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  Smem S(smem_raw);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  T *Fs = S.take<T>(3 * N);
  T *par = S.take<T>(kTsFields * np);
  double *red = S.take<double>(8 * 32);
  int *pfirst = S.take<int>(N + 1);
  int *tfirst = S.take<int>(N + 1);
  int *wsum = S.take<int>(32);
  for (int k = threadIdx.x; k < kTsFields * np; k += blockDim.x)
    par[k] = static_cast<T>(A.vals[A.c.desc[k / kTsFields].pv0 + k % kTsFields]);
  for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) Fs[k] = T(0);
  stage_geometry(cd, A.c, wpos, shift, typ);
  const int32_t *start = A.c.nb_start + cd.atom0;
  stage_work(start, N, pfirst, tfirst, wsum);
  __syncthreads();
  const uint32_t *nbp = A.c.nb_pack + start[0];
  const int nbond = pfirst[N];
  double e_acc = 0.0, sg[6] = {0, 0, 0, 0, 0, 0}; // xx, yy, zz, xy, xz, yz
  auto add_stress = [&](const T (&d)[3], const T (&f)[3], T s) {
    sg[0] += static_cast<double>(s * d[0] * f[0]);
    sg[1] += static_cast<double>(s * d[1] * f[1]);
    sg[2] += static_cast<double>(s * d[2] * f[2]);
    sg[3] += static_cast<double>(s * d[0] * f[1]);
    sg[4] += static_cast<double>(s * d[0] * f[2]);
    sg[5] += static_cast<double>(s * d[1] * f[2]);
  };
  for (int w = threadIdx.x; w < nbond; w += blockDim.x) {
    const int i = owner_of(pfirst, N, w);
    const int ti = typ[i];
    int j;
    T d1[3];
    pair_vec(wpos, shift, i, nbp[w], j, d1[0], d1[1], d1[2]);
    const T r1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
    if (r1 < T(1e-14)) continue;
    const T *p = par + kTsFields * pair_ord(ti, typ[j], nt);
    const T fc = ts_fc(r1, p[9], p[10]), dfc = ts_dfc(r1, p[9], p[10]);
    if (fc == T(0) && dfc == T(0)) continue; // make_bond
    const T VR = p[0] * exp(-p[2] * r1), VA = p[1] * exp(-p[3] * r1);
    const T VRp = -p[2] * VR, VAp = -p[3] * VA;
    const int k0 = pfirst[i], k1 = pfirst[i + 1];
    // ζ_ij (add_zeta)
    T zeta = T(0);
    for (int pk = k0; pk < k1; ++pk) {
      if (pk == w) continue;
      int k;
      T d2[3];
      pair_vec(wpos, shift, i, nbp[pk], k, d2[0], d2[1], d2[2]);
      const T r2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
      if (r2 < T(1e-14)) continue;
      const T *q = par + kTsFields * pair_ord(ti, typ[k], nt);
      const T fck = ts_fc(r2, q[9], q[10]);
      if (fck == T(0)) continue;
      const T cth = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) / (r1 * r2);
      zeta += q[11] * fck * ts_g(cth, p);
    }
    T b, db;
    ts_b(zeta, p, b, db);
    // accumulate_pair
    e_acc += 0.5 * static_cast<double>(fc * (VR - b * VA));
    const T pc = T(0.5) * (dfc * (VR - b * VA) + fc * (VRp - b * VAp)) / r1;
    const T Fp[3] = {pc * d1[0], pc * d1[1], pc * d1[2]};
    add_stress(d1, Fp, T(-0.5));
    // the forces on i and j of this bond and of its three-body terms, summed
    // here and added once (k's are added per neighbour)
    T fi[3] = {Fp[0], Fp[1], Fp[2]}, fj[3] = {-Fp[0], -Fp[1], -Fp[2]};
    if (zeta == T(0)) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        atomicAdd(&Fs[3 * i + a], fi[a]);
        atomicAdd(&Fs[3 * j + a], fj[a]);
      }
      continue;
    }
    // accumulate_three_body
    const T Pz = T(0.5) * fc * VA * db;
    const T ir1 = T(1) / r1;
    for (int pk = k0; pk < k1; ++pk) {
      if (pk == w) continue;
      int k;
      T d2[3];
      pair_vec(wpos, shift, i, nbp[pk], k, d2[0], d2[1], d2[2]);
      const T r2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
      if (r2 < T(1e-14)) continue;
      const T *q = par + kTsFields * pair_ord(ti, typ[k], nt);
      const T fck = ts_fc(r2, q[9], q[10]), dfck = ts_dfc(r2, q[9], q[10]);
      if (fck == T(0) && dfck == T(0)) continue;
      const T ir2 = T(1) / r2;
      const T cth = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) * ir1 * ir2;
      const T gv = ts_g(cth, p), dgv = ts_dg(cth, p);
      const T Ac = cth * ir1 * ir1 - ir1 * ir2, Bc = cth * ir2 * ir2 - ir1 * ir2;
      const T wk = q[11];
      T Fi[3], Fj[3], Fk[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        Fi[a] = Pz * (wk * (-dfck * ir2 * gv * d2[a] + fck * dgv * (Ac * d1[a] + Bc * d2[a])));
        Fj[a] = Pz * (wk * fck * dgv * (ir1 * ir2 * d2[a] - cth * ir1 * ir1 * d1[a]));
        Fk[a] = Pz * (wk * (dfck * ir2 * gv * d2[a] + fck * dgv * (ir1 * ir2 * d1[a] - cth * ir2 * ir2 * d2[a])));
        fi[a] += Fi[a];
        fj[a] += Fj[a];
        atomicAdd(&Fs[3 * k + a], Fk[a]);
      }
      add_stress(d1, Fj, T(1));
      add_stress(d2, Fk, T(1));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicAdd(&Fs[3 * i + a], fi[a]);
      atomicAdd(&Fs[3 * j + a], fj[a]);
    }
  }
  __syncthreads();
  // residual rows of the configuration (residual_layout.hpp:37-54)
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
    const double E = sums[0], iv = 1.0 / cd.volume;
    double st[6];
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
    A.F[row++] = 0.0; // no embedding: the limit row is zero
    A.obj_part[c] = o;
    if (A.energy) A.energy[c] = E;
    if (A.limit) A.limit[c] = 0.0;
    if (A.stress9) {
      // the configuration's virial is symmetric (rotation invariance): the
      // upper triangle is mirrored
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

__global__ void ts_sum_parts(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double r[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, r);
  if (threadIdx.x == 0) *out = s;
}

int ts_max_images(const fs_gpu *h) {
  int m = 1;
  for (const CfgDev &cd : h->cfg_host) m = std::max(m, (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1));
  return m;
}

template <class T> int launch_tersoff(fs_gpu *h, double w_e, double w_s) {
  TsArgs<T> a;
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
  const int np = npair_of(h->ntypes), N = h->max_natoms, mi = ts_max_images(h);
  const size_t sm = align16(3 * N * sizeof(double)) + align16(3 * mi * sizeof(double)) + align16(N) +
                    align16(3 * N * sizeof(T)) + align16(kTsFields * np * sizeof(T)) +
                    align16(8 * 32 * sizeof(double)) + 2 * align16((N + 1) * sizeof(int)) +
                    align16(32 * sizeof(int)) + 128;
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "Tersoff: configuration too large for shared memory");
  auto k = tersoff_kernel<T>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, kTsThreads, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  ts_sum_parts<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

} // namespace

int eval_residual_tersoff(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_tersoff<double>(h, w_e, w_s) : launch_tersoff<float>(h, w_e, w_s);
}

} // namespace fsg
