// Angular on the device: residual (forces, energy, stress, objective).
//
//   AngularForceCalculator::eval_forces (src/force/angular_force.cpp:13-88):
//   the pair term φ_{t_i t_j}(r), ½ per directed pair (accumulate_pair,
//   kernels.hpp:33-38), plus, per central atom i and neighbour pair j < k,
//   f_{t_i t_j}(r_ij) f_{t_i t_k}(r_ik) g_{t_i}(cos θ_jik) with the forces of
//   three_body_forces / accumulate_triplet (kernels.hpp:44-68).  φ and f are
//   gated to their closed spans (force_calculator_concept.hpp:94-98); g is
//   evaluated ungated (a spline extrapolates linearly).  Each table is a
//   makima spline or one of the analytic forms.
//   With spline tables the reference's Jacobian is central differences; the
//   device keeps that method (fd.cu, FP64 contexts).
//
// One CTA per configuration; each thread takes 4 consecutive work items from
// a block scan: directed pairs (2-body), then neighbour pairs (j < k) of a
// central atom (3-body).  Forces accumulate in shared memory, summed first in
// registers over a thread's items that share an atom; energy and stress are
// per-thread FP64 sums.
#include "kern_common.cuh"

#include <algorithm>

namespace fsg {
namespace {

constexpr int kAgThreads = 256;
constexpr int kAgChunk = 4; // consecutive work items per thread

template <class T> struct AgArgs {
  Common c;
  const typename Vec4T<T>::type *seg; // segment coefficients (working precision)
  const double *vals;                 // all model values (FP64; analytic parameters)
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
  const int32_t *order; // configurations by work, heaviest first
};

template <class T> __global__ void __launch_bounds__(kAgThreads, sizeof(T) == 4 ? 3 : 2) angular_kernel(AgArgs<T> A) {
  using T4 = typename Vec4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = A.order ? A.order[blockIdx.x] : blockIdx.x;
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
  T *Fs = S.take<T>(3 * N);
  double *red = S.take<double>(8 * 32);
  int *pfirst = S.take<int>(N + 1);
  int *tfirst = S.take<int>(N + 1);
  int *wsum = S.take<int>(32);
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  for (int k = threadIdx.x; k < A.c.n_segs; k += blockDim.x) seg[k] = A.seg[k];
  for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) Fs[k] = T(0);
  stage_geometry(cd, A.c, wpos, shift, typ);
  const int32_t *start = A.c.nb_start + cd.atom0;
  stage_work(start, N, pfirst, tfirst, wsum);
  __syncthreads();
  const uint32_t *nbp = A.c.nb_pack + start[0];
  const int npair = pfirst[N], ntri = tfirst[N];
  double e_acc = 0.0, sg[6] = {0, 0, 0, 0, 0, 0}; // xx, yy, zz, xy, xz, yz
  // Each thread takes kAgChunk consecutive work items.  Items are ordered by
  // central atom (then by neighbour), so consecutive items mostly share atom
  // i (and, for neighbour pairs, atom j): their forces on i and j are summed
  // in registers and added to shared memory when the atom changes.
  struct Acc {
    T f[3] = {T(0), T(0), T(0)};
    int at = -1;
    __device__ __forceinline__ void to(int a, T *Fs) {
      if (a == at) return;
      if (at >= 0)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          atomicAdd(&Fs[3 * at + q], f[q]);
          f[q] = T(0);
        }
      at = a;
    }
  };
  // ---- 2-body: one item per directed pair
  for (int w0 = threadIdx.x * kAgChunk; w0 < npair; w0 += blockDim.x * kAgChunk) {
    const int w1 = min(w0 + kAgChunk, npair);
    int i = owner_of(pfirst, N, w0);
    Acc ai;
    for (int w = w0; w < w1; ++w) {
      while (pfirst[i + 1] <= w) ++i;
      int j;
      T d[3];
      pair_vec(wpos, shift, i, nbp[w], j, d[0], d[1], d[2]);
      const T r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r < T(1e-14)) continue;
      const STab<T> &tb = tabs[pair_ord(typ[i], typ[j], nt)];
      const uint32_t pw = nbp[w];
      T tq;
      const int eq = gate_seg(tb, r, tq, [=] { return pair_len64(wpos, shift, i, pw); });
      if (eq < 0) continue;
      const VD<T> ph = tab_vd_at<T, true>(tb, seg, A.vals, r, eq, tq);
      const T s = ph.d / r;
      const T f[3] = {s * d[0], s * d[1], s * d[2]};
      ai.to(i, Fs);
#pragma unroll
      for (int a = 0; a < 3; ++a) ai.f[a] += f[a];
      e_acc += 0.5 * static_cast<double>(ph.v);
      sg[0] -= static_cast<double>(T(0.5) * d[0] * f[0]);
      sg[1] -= static_cast<double>(T(0.5) * d[1] * f[1]);
      sg[2] -= static_cast<double>(T(0.5) * d[2] * f[2]);
      sg[3] -= static_cast<double>(T(0.5) * d[0] * f[1]);
      sg[4] -= static_cast<double>(T(0.5) * d[0] * f[2]);
      sg[5] -= static_cast<double>(T(0.5) * d[1] * f[2]);
    }
    ai.to(-1, Fs);
  }
  // ---- 3-body: one item per neighbour pair (j < k) of a central atom i
  for (int w0 = threadIdx.x * kAgChunk; w0 < ntri; w0 += blockDim.x * kAgChunk) {
    const int w1 = min(w0 + kAgChunk, ntri);
    int i = owner_of(tfirst, N, w0);
    Acc ai, aj;
    for (int w = w0; w < w1; ++w) {
      while (tfirst[i + 1] <= w) ++i;
      const int n = pfirst[i + 1] - pfirst[i];
      int u = w - tfirst[i], a0 = 0;
      pair_row(n, u, a0);
      const int pj = pfirst[i] + a0, pk = pj + 1 + u;
      const int ti = typ[i];
      int j, k;
      T d1[3], d2[3];
      pair_vec(wpos, shift, i, nbp[pj], j, d1[0], d1[1], d1[2]);
      const T r1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
      if (r1 < T(1e-14)) continue;
      const STab<T> &rj = tabs[np + pair_ord(ti, typ[j], nt)];
      const uint32_t pwj = nbp[pj];
      T t1;
      const int e1 = gate_seg(rj, r1, t1, [=] { return pair_len64(wpos, shift, i, pwj); });
      if (e1 < 0) continue;
      pair_vec(wpos, shift, i, nbp[pk], k, d2[0], d2[1], d2[2]);
      const T r2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
      if (r2 < T(1e-14)) continue;
      const STab<T> &rk = tabs[np + pair_ord(ti, typ[k], nt)];
      const uint32_t pwk = nbp[pk];
      T t2;
      const int e2 = gate_seg(rk, r2, t2, [=] { return pair_len64(wpos, shift, i, pwk); });
      if (e2 < 0) continue;
      const VD<T> F1 = tab_vd_at<T, true>(rj, seg, A.vals, r1, e1, t1),
                  F2 = tab_vd_at<T, true>(rk, seg, A.vals, r2, e2, t2);
      const T ir1 = T(1) / r1, ir2 = T(1) / r2;
      const T cth = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) * ir1 * ir2;
      const VD<T> G = tab_vd<T, true>(tabs[2 * np + ti], seg, A.vals, cth);
      e_acc += static_cast<double>(F1.v * F2.v * G.v);
      // three_body_forces (kernels.hpp:44-58)
      const T irr = ir1 * ir2;
      const T Aa = cth * ir1 * ir1 - irr, Bb = cth * ir2 * ir2 - irr;
      const T c1 = F1.d * ir1 * F2.v * G.v, c2 = F1.v * F2.d * ir2 * G.v, c3 = F1.v * F2.v * G.d;
      T Fj[3], Fk[3];
      ai.to(i, Fs);
      aj.to(j, Fs);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const T Fi = c1 * d1[a] + c2 * d2[a] - c3 * (Aa * d1[a] + Bb * d2[a]);
        Fj[a] = -(c1 * d1[a]) - c3 * (irr * d2[a] - cth * ir1 * ir1 * d1[a]);
        Fk[a] = -(c2 * d2[a]) - c3 * (irr * d1[a] - cth * ir2 * ir2 * d2[a]);
        ai.f[a] += Fi;
        aj.f[a] += Fj[a];
        atomicAdd(&Fs[3 * k + a], Fk[a]);
      }
      sg[0] += static_cast<double>(d1[0] * Fj[0] + d2[0] * Fk[0]);
      sg[1] += static_cast<double>(d1[1] * Fj[1] + d2[1] * Fk[1]);
      sg[2] += static_cast<double>(d1[2] * Fj[2] + d2[2] * Fk[2]);
      sg[3] += static_cast<double>(d1[0] * Fj[1] + d2[0] * Fk[1]);
      sg[4] += static_cast<double>(d1[0] * Fj[2] + d2[0] * Fk[2]);
      sg[5] += static_cast<double>(d1[1] * Fj[2] + d2[1] * Fk[2]);
    }
    ai.to(-1, Fs);
    aj.to(-1, Fs);
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

__global__ void ag_sum_parts(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double r[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, r);
  if (threadIdx.x == 0) *out = s;
}

template <class T> int launch_angular(fs_gpu *h, double w_e, double w_s) {
  AgArgs<T> a;
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
  a.seg = static_cast<const typename Vec4T<T>::type *>(h->d_seg_a);
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
  int mi = 1;
  for (const CfgDev &cd : h->cfg_host) mi = std::max(mi, (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1));
  const int N = h->max_natoms;
  const size_t sm = align16(a.c.n_tables * sizeof(STab<T>)) +
                    align16(static_cast<size_t>(h->n_segs) * sizeof(typename Vec4T<T>::type)) +
                    align16(3 * N * sizeof(double)) + align16(3 * mi * sizeof(double)) + align16(N) +
                    align16(3 * N * sizeof(T)) + align16(8 * 32 * sizeof(double)) +
                    2 * align16((N + 1) * sizeof(int)) + align16(32 * sizeof(int)) + 160;
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "Angular: configuration too large for shared memory");
  auto k = angular_kernel<T>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, kAgThreads, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  ag_sum_parts<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

} // namespace

int eval_residual_angular(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_angular<double>(h, w_e, w_s) : launch_angular<float>(h, w_e, w_s);
}

} // namespace fsg
