// EAM and tabulated-pair calculators on the device: the residual vector and
// its analytic Jacobian with respect to the free spline knots.
//
//   residual   EAMForceCalculator::eval_forces (src/force/eam_force.cpp:45-102),
//              PairForceCalculator::eval_forces (src/force/pair_force.cpp:21-60),
//              with_eval_scope (include/forcesmith/force/eval_scope.hpp:13-31)
//              and write_config_residuals
//              (include/forcesmith/optimization/residual_layout.hpp:37-54).
//   Jacobian   the chain rule of EAMForceCalculator::write_param_jacobian
//              (src/force/eam_force.cpp:108-279) and
//              PairForceCalculator::write_param_jacobian (pair_force.cpp:80-111),
//              with ∂(spline)/∂(knots) taken through the makima slopes.  The
//              reference differentiates splines by central differences
//              (forcesmith_functor.cpp:279-286); this is the exact derivative
//              of the same function.
//
// One CTA per configuration.  The configuration's wrapped positions, its
// periodic image shifts and the spline segment tables sit in shared memory;
// the neighbour list is a 4-byte (j, image) word per directed pair, and each
// pair vector is rebuilt in FP64 then rounded to the working precision T.
#include "kern_common.cuh"

#include <algorithm>
#include <mutex>
#include <string>

namespace fsg {
namespace {

template <class T> struct ResArgs {
  Common c;
  const typename Vec4T<T>::type *seg_a;
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
};

template <class T> size_t residual_smem(int n_tables, int n_segs, int max_atoms, int max_img) {
  size_t b = 0;
  b += align16(n_tables * sizeof(STab<T>));
  b += align16(n_segs * 4 * sizeof(T));
  b += align16(3 * max_atoms * sizeof(double));
  b += align16(3 * max_img * sizeof(double));
  b += align16(max_atoms);
  b += align16(2 * max_atoms * sizeof(T));
  b += 64 * sizeof(double) + 64;
  return b + 64;
}

// ---------------------------------------------------------------------------
// Residual: ρ pass → embedding → force/energy/stress pass → residual rows.
// ---------------------------------------------------------------------------
// The residual of one configuration from staged tables and geometry: writes
// its rows when ROWS, and returns Σ rows² (valid on thread 0) — shared by the
// residual kernel and the population kernel.
template <class T, int LPA, bool EAM, bool ROWS, bool AN = false>
__device__ double config_pass(const ResArgs<T> &A, int c, const CfgDev &cd, const STab<T> *tabs,
                              const typename Vec4T<T>::type *seg, const double *wpos, const double *shift,
                              const uint8_t *typ, T *rho, T *gradF, double *red) {
  const int N = cd.natoms;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int ngroups = blockDim.x / LPA, g = threadIdx.x / LPA, l = threadIdx.x % LPA;
  const int32_t *start = A.c.nb_start + cd.atom0;
  double e_emb = 0.0, lim = 0.0;
  if constexpr (EAM) {
    // ρ_i = Σ_j ρ_{t(j)}(r_ij), closed gate (eam_force.cpp:59-66)
    for (int i0 = 0; i0 < N; i0 += ngroups) {
      const int i = i0 + g;
      T acc = T(0);
      if (i < N) {
        for (int p = start[i] + l; p < start[i + 1]; p += LPA) {
          int j;
          T dx, dy, dz;
          const double r64 = pair_vec_len(wpos, shift, i, A.c.nb_pack[p], j, dx, dy, dz);
          const T r = static_cast<T>(r64);
          const STab<T> &tb = tabs[np + typ[j]];
          if (gate64(tb, r64)) acc += tab_vd64<T, AN>(tb, seg, A.c.vals, r, r64).v;
        }
      }
      acc = warp_sum_group(acc, LPA);
      if (i < N && l == 0) rho[i] = acc;
    }
    __syncthreads();
    // clamp_embedding + F(ρ), F'(ρ) (kernels.hpp:19-31; eam_force.cpp:68-73)
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const STab<T> &tb = tabs[np + nt + typ[i]];
      T rr = rho[i];
      if (rr > tb.xmax) {
        const double d = static_cast<double>(rr) - static_cast<double>(tb.xmax);
        lim += 100.0 * 10.0 * d * d;
        rr = tb.xmax;
      } else if (rr < tb.x0) {
        const double d = static_cast<double>(tb.x0) - static_cast<double>(rr);
        lim += 100.0 * 10.0 * d * d;
        rr = tb.x0;
      }
      const VD<T> fv = tab_vd<T, AN>(tb, seg, A.c.vals, rr);
      e_emb += static_cast<double>(fv.v);
      gradF[i] = fv.d;
    }
    __syncthreads();
  }
  // forces, ½φ energy and −½ d fᵀ stress (eam_force.cpp:75-100; kernels.hpp:33-38)
  double e_pair = 0.0, objp = 0.0;
  double sg[6] = {0, 0, 0, 0, 0, 0};
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  for (int i0 = 0; i0 < N; i0 += ngroups) {
    const int i = i0 + g;
    T f[3] = {0, 0, 0}, ep = T(0), s[6] = {0, 0, 0, 0, 0, 0};
    if (i < N) {
      const int ti = typ[i];
      for (int p = start[i] + l; p < start[i + 1]; p += LPA) {
        int j;
        T d[3];
        const double r64 = pair_vec_len(wpos, shift, i, A.c.nb_pack[p], j, d[0], d[1], d[2]);
        const T r = static_cast<T>(r64);
        if (r64 < 1e-14) continue;
        const int tj = typ[j];
        const STab<T> &tp = tabs[pair_ord(ti, tj, nt)];
        T phi = T(0), dphi = T(0);
        if constexpr (EAM) {
          if (gate64(tp, r64)) {
            const VD<T> pv = tab_vd64<T, AN>(tp, seg, A.c.vals, r, r64);
            phi = pv.v;
            dphi = pv.d;
          }
        } else {
          // make_pair_bond's half-open gate [rmin, rmax) (pair_force.cpp:28)
          if (!gate64<false>(tp, r64)) continue;
          const VD<T> pv = tab_vd64<T, AN>(tp, seg, A.c.vals, r, r64);
          phi = pv.v;
          dphi = pv.d;
        }
        T fs = dphi;
        if constexpr (EAM) {
          const STab<T> &gj = tabs[np + tj], &gi = tabs[np + ti];
          T drho_j = T(0), drho_i = T(0);
          if (gate64(gj, r64)) drho_j = tab_vd64<T, AN>(gj, seg, A.c.vals, r, r64).d;
          if (gate64(gi, r64)) drho_i = tab_vd64<T, AN>(gi, seg, A.c.vals, r, r64).d;
          fs = dphi + gradF[i] * drho_j + gradF[j] * drho_i;
        }
        fs = fs * (T(1) / r);
        const T fx = fs * d[0], fy = fs * d[1], fz = fs * d[2];
        f[0] += fx;
        f[1] += fy;
        f[2] += fz;
        ep += phi;
        const T hx = T(0.5) * d[0], hy = T(0.5) * d[1], hz = T(0.5) * d[2];
        s[0] -= hx * fx;
        s[1] -= hy * fy;
        s[2] -= hz * fz;
        s[3] -= hx * fy;
        s[4] -= hx * fz;
        s[5] -= hy * fz;
      }
    }
    for (int a = 0; a < 3; ++a) f[a] = warp_sum_group(f[a], LPA);
    ep = warp_sum_group(ep, LPA);
    for (int a = 0; a < 6; ++a) s[a] = warp_sum_group(s[a], LPA);
    if (i < N && l == 0) {
      const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
      for (int a = 0; a < 3; ++a) {
        const double fa = static_cast<double>(f[a]);
        const double res = fa - A.c.ref_force[3 * ga + a];
        if constexpr (ROWS) {
          A.F[row0 + 3 * i + a] = res;
          if (A.forces) A.forces[3 * ga + a] = fa;
        }
        objp += res * res;
      }
      e_pair += 0.5 * static_cast<double>(ep);
      for (int a = 0; a < 6; ++a) sg[a] += static_cast<double>(s[a]);
    }
  }
  const double E = block_sum(e_emb + e_pair, red);
  const double L = block_sum(lim, red);
  double st[6];
  for (int a = 0; a < 6; ++a) st[a] = block_sum(sg[a], red);
  const double op = block_sum(objp, red);
  double out = 0.0;
  if (threadIdx.x == 0) {
    const double iv = 1.0 / cd.volume;
    for (int a = 0; a < 6; ++a) st[a] = st[a] * iv; // σ /= V (eval_scope.hpp:28)
    int64_t row = row0 + 3 * N;
    double o = op;
    const double re = A.w_e * (E - cd.ref_energy);
    if constexpr (ROWS) A.F[row] = re;
    ++row;
    o += re * re;
    static constexpr int vi[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    if (A.w_s > 0.0) {
      for (int v = 0; v < 6; ++v) {
        const double rs = A.w_s * (st[v] - cd.ref_stress[3 * vi[v][0] + vi[v][1]]);
        if constexpr (ROWS) A.F[row] = rs;
        ++row;
        o += rs * rs;
      }
    }
    if constexpr (ROWS) A.F[row] = L;
    o += L * L;
    out = o;
    if (ROWS && A.energy) A.energy[c] = E;
    if (ROWS && A.limit) A.limit[c] = L;
    if (ROWS && A.stress9) {
      double *s9 = A.stress9 + 9 * static_cast<int64_t>(c);
      s9[0] = st[0];
      s9[4] = st[1];
      s9[8] = st[2];
      s9[1] = s9[3] = st[3];
      s9[2] = s9[6] = st[4];
      s9[5] = s9[7] = st[5];
    }
  }
  return out;
}

template <class T, int LPA, bool EAM, bool AN>
__global__ void __launch_bounds__(256) residual_kernel(ResArgs<T> A) {
  using T4 = typename Vec4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  Smem S(smem_raw);
  STab<T> *tabs = S.take<STab<T>>(A.c.n_tables);
  T4 *seg = S.take<T4>(A.c.n_segs);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  T *rho = S.take<T>(N);
  T *gradF = S.take<T>(N);
  double *red = S.take<double>(64);
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  for (int k = threadIdx.x; k < A.c.n_segs; k += blockDim.x) seg[k] = A.seg_a[k];
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();
  const double o = config_pass<T, LPA, EAM, true, AN>(A, c, cd, tabs, seg, wpos, shift, typ, rho, gradF, red);
  if (threadIdx.x == 0) A.obj_part[c] = o;
}

// Population objective: one CTA per (configuration, tile of trial vectors).
// The configuration's geometry is staged once; each trial's spline segments
// (built by pop_setup_kernel) are swapped in and the configuration's Σ rows²
// is written to part[trial][config].
template <class T, int LPA, bool EAM>
__global__ void __launch_bounds__(256) pop_eval_kernel(ResArgs<T> A, const typename Vec4T<T>::type *pop_seg,
                                                       int NP, int tile, int n_tiles, const int32_t *order,
                                                       double *part) {
  using T4 = typename Vec4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = order[blockIdx.x / n_tiles];
  const int k0 = (blockIdx.x % n_tiles) * tile, k1 = min(NP, k0 + tile);
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  Smem S(smem_raw);
  STab<T> *tabs = S.take<STab<T>>(A.c.n_tables);
  T4 *seg = S.take<T4>(A.c.n_segs);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  T *rho = S.take<T>(N);
  T *gradF = S.take<T>(N);
  double *red = S.take<double>(64);
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  stage_geometry(cd, A.c, wpos, shift, typ);
  for (int k = k0; k < k1; ++k) {
    for (int q = threadIdx.x; q < A.c.n_segs; q += blockDim.x) seg[q] = pop_seg[static_cast<int64_t>(k) * A.c.n_segs + q];
    __syncthreads();
    const double o = config_pass<T, LPA, EAM, false>(A, c, cd, tabs, seg, wpos, shift, typ, rho, gradF, red);
    if (threadIdx.x == 0) part[static_cast<int64_t>(k) * A.c.cfg_count + c] = o;
    __syncthreads();
  }
}

// Population objective, FP32, lanes = trials.  A CTA holds the spline
// coefficients of 32 trial vectors in shared memory ([segment][trial], so a
// warp's coefficient load is conflict-free) and walks a size-balanced stride
// of the configurations, staging each one's geometry in turn.  A warp takes
// atoms in turn; for a batch of 32 of the atom's pairs its lanes compute the
// trial-independent geometry once (unit vector, ½dd/r, and per spline role
// the segment and local coordinate) into a shared record, then every lane
// walks the batch reading each record as a broadcast and applying its own
// trial's coefficients.  Per-trial forces, energy and stress accumulate in
// the lane; the configuration's Σ rows² per trial is summed over warps in a
// fixed order (deterministic).
constexpr int kPopLanes = 32;
constexpr int kPopWarps = 16;

struct PopRec { // 80 B; 16 warps × 32 records also hold the 16 × 32 × 10 FP64 partials
  float4 a;  // ux, uy, uz, t(φ)
  float4 b;  // ½·dx·dx/r, ½·dy·dy/r, ½·dz·dz/r, ½·dx·dy/r
  float4 c;  // ½·dx·dz/r, ½·dy·dz/r, t(ρ_j), t(ρ_i)
  float4 ih; // 1/h of the φ, ρ_j, ρ_i tables
  int4 d;    // j, segment of φ, ρ_j, ρ_i (−1: outside the table's gate)
};

struct PopArgs {
  Common c;
  const float4 *pop_seg;              // [trial][n_segs]
  int NP, n_tiles, n_chunks, nseg_pd; // nseg_pd: segments of the pair + density tables (staged)
  int max_atoms, max_img;
  const int32_t *order;               // configurations by decreasing size
  double *part;                       // [trial][config]
  double w_e, w_s;
  // RUNS: each atom's pairs sorted by (neighbour species, segment) on the
  // grid shared by the pair and density tables (pair_runs.cu)
  const float4 *run_a; // u, t
  const int2 *run_b;   // packed neighbour entry, key
  const float *run_r;  // length (−1: coincident atoms)
  const int32_t *run_cnt;
  int runs;            // 1: walk the pair runs
};

size_t pop_lanes_smem(int n_tables, int nseg_pd, int max_atoms, int max_img, bool eam) {
  size_t b = 0;
  b += align16(static_cast<size_t>(nseg_pd) * kPopLanes * sizeof(float4));
  b += align16(n_tables * sizeof(STab<float>));
  b += align16(3 * max_atoms * sizeof(double));
  b += align16(3 * max_img * sizeof(double));
  b += align16(max_atoms);
  if (eam) b += align16(static_cast<size_t>(max_atoms) * kPopLanes * sizeof(float));
  b += align16(kPopWarps * 32 * sizeof(PopRec));
  b += align16(kPopLanes * 10 * sizeof(double));
  b += align16((max_atoms + 1) * sizeof(int32_t));
  return b + 64;
}

__device__ __forceinline__ float poly_val(const float4 &a, float t) { return a.x + t * (a.y + t * (a.z + t * a.w)); }
__device__ __forceinline__ float poly_der(const float4 &a, float t) { return a.y + t * (2.f * a.z + 3.f * t * a.w); }

// RUNS (EAM, pair and density tables on one knot grid): the pairs come
// from the sorted pair runs instead of the neighbour list; a run of pairs
// with one (neighbour species, segment) key shares the φ_{t_i t_j}, ρ_{t_j}
// and ρ_{t_i} segments, so each lane loads its trial's coefficients once per
// run, and the pair geometry is read instead of rebuilt for every tile.
// STRESS (w_s > 0): the per-trial virial sums; the DE objective of a fit
// without stress rows skips them.
template <bool EAM, bool RUNS, bool STRESS>
__global__ void __launch_bounds__(kPopWarps * 32, 1) pop_lanes_kernel(PopArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tile = blockIdx.x % A.n_tiles, chunk = blockIdx.x / A.n_tiles;
  const int k0 = tile * kPopLanes;
  const int ntr = min(kPopLanes, A.NP - k0);
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  Smem S(smem_raw);
  float4 *coef = S.take<float4>(static_cast<size_t>(A.nseg_pd) * kPopLanes);
  STab<float> *tabs = S.take<STab<float>>(A.c.n_tables);
  double *wpos = S.take<double>(3 * A.max_atoms);
  double *shift = S.take<double>(3 * A.max_img);
  uint8_t *typ = S.take<uint8_t>(A.max_atoms);
  float *rf = EAM ? S.take<float>(static_cast<size_t>(A.max_atoms) * kPopLanes) : nullptr; // ρ, then F'(ρ)
  PopRec *stage = S.take<PopRec>(kPopWarps * 32);
  double *red = S.take<double>(kPopLanes * 10);
  int32_t *sstart = S.take<int32_t>(A.max_atoms + 1);
  for (int q = threadIdx.x; q < A.nseg_pd * kPopLanes; q += blockDim.x) {
    const int k = q / A.nseg_pd, e = q % A.nseg_pd;
    coef[e * kPopLanes + k] =
        k < ntr ? A.pop_seg[static_cast<int64_t>(k0 + k) * A.c.n_segs + e] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  const uint32_t *pack = A.c.nb_pack;
  PopRec *wst = stage + w * 32;
  // this CTA's configurations: every n_chunks-th of the size-sorted order
  for (int ci = chunk; ci < A.c.cfg_count; ci += A.n_chunks) {
    const int c = A.order[ci];
    const CfgDev &cd = A.c.cfg[c];
    const int N = cd.natoms;
    __syncthreads(); // the previous configuration is done with the staged data
    stage_geometry(cd, A.c, wpos, shift, typ);
    for (int k = threadIdx.x; k <= N; k += blockDim.x) sstart[k] = A.c.nb_start[cd.atom0 + k];
    __syncthreads();
    const int32_t *start = sstart;
    // the neighbour words of an atom's first batch of 32 pairs (0 past its end)
    auto first_batch = [&](int ii) -> uint32_t {
      return (ii < N && start[ii] + l < start[ii + 1]) ? pack[start[ii] + l] : 0u;
    };
    double e_emb = 0.0, lim = 0.0, e_pair = 0.0, objf = 0.0;
    double sg[6] = {0, 0, 0, 0, 0, 0};

    if constexpr (EAM) {
     if constexpr (RUNS) {
      // ρ_i per trial (closed gate, eam_force.cpp:59-66) over the atom's runs
      int2 *wst2 = reinterpret_cast<int2 *>(wst);
      for (int i = w; i < N; i += kPopWarps) {
        const int64_t gi = static_cast<int64_t>(cd.atom0) + i;
        const int p0 = start[i], cnt = A.run_cnt[gi];
        float acc = 0.f;
        int cur = -1;
        float4 cf = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int pb = 0; pb < cnt; pb += 32) {
          int2 rec = make_int2(-1, 0);
          if (pb + l < cnt) {
            const int key = A.run_b[p0 + pb + l].y;
            const int tj = key >> kRunKeyBits, e = key & ((1 << kRunKeyBits) - 1);
            rec = make_int2(tabs[np + tj].seg0 + e, __float_as_int(A.run_a[p0 + pb + l].w));
          }
          wst2[l] = rec;
          __syncwarp();
          const int c = min(32, cnt - pb);
          for (int q = 0; q < c; ++q) {
            const int2 rr = wst2[q];
            if (rr.x != cur) { // a new run (warp-uniform)
              cur = rr.x;
              cf = coef[cur * kPopLanes + l];
            }
            acc += poly_val(cf, __int_as_float(rr.y));
          }
          __syncwarp();
        }
        rf[i * kPopLanes + l] = acc;
      }
     } else {
      // ρ_i per trial (closed gate, eam_force.cpp:59-66)
      int2 *wst2 = reinterpret_cast<int2 *>(wst);
      uint32_t pk = first_batch(w);
      for (int i = w; i < N; i += kPopWarps) {
        const int p0 = start[i], p1 = start[i + 1];
        float acc = 0.f;
        if (p0 == p1) pk = first_batch(i + kPopWarps);
        for (int pb = p0; pb < p1; pb += 32) {
          const int p = pb + l;
          const uint32_t cur = pk;
          // prefetch the next batch: this atom's, else the warp's next atom's first
          pk = pb + 32 < p1 ? (pb + 32 + l < p1 ? pack[pb + 32 + l] : 0u) : first_batch(i + kPopWarps);
          int2 rec = make_int2(-1, 0);
          if (p < p1) {
            int j;
            float dx, dy, dz;
            const double r64 = pair_vec_len(wpos, shift, i, cur, j, dx, dy, dz);
            const STab<float> &tb = tabs[np + typ[j]];
            if (gate64(tb, r64)) {
              float t;
              rec.x = seg_of64(tb, static_cast<float>(r64), r64, t);
              rec.y = __float_as_int(t);
            }
          }
          wst2[l] = rec;
          __syncwarp();
          const int cnt = min(32, p1 - pb);
          for (int q = 0; q < cnt; ++q) {
            const int2 rr = wst2[q];
            if (rr.x >= 0) acc += poly_val(coef[rr.x * kPopLanes + l], __int_as_float(rr.y));
          }
          __syncwarp();
        }
        rf[i * kPopLanes + l] = acc;
      }
     }
      __syncthreads();
      // clamp + F(ρ), F'(ρ) per (atom, trial) (kernels.hpp:19-31; eam_force.cpp:68-73)
      for (int i = w; i < N; i += kPopWarps) {
        const STab<float> &tb = tabs[np + nt + typ[i]];
        float rr = rf[i * kPopLanes + l];
        if (rr > tb.xmax) {
          const double d = static_cast<double>(rr) - static_cast<double>(tb.xmax);
          lim += 100.0 * 10.0 * d * d;
          rr = tb.xmax;
        } else if (rr < tb.x0) {
          const double d = static_cast<double>(tb.x0) - static_cast<double>(rr);
          lim += 100.0 * 10.0 * d * d;
          rr = tb.x0;
        }
        float t;
        const int e = seg_of(tb, rr, t);
        const float4 a =
            l < ntr ? A.pop_seg[static_cast<int64_t>(k0 + l) * A.c.n_segs + e] : make_float4(0.f, 0.f, 0.f, 0.f);
        e_emb += static_cast<double>(poly_val(a, t));
        rf[i * kPopLanes + l] = poly_der(a, t) * tb.inv_h;
      }
      __syncthreads();
    }
    // forces, ½φ energy, −½ d fᵀ stress (eam_force.cpp:75-100; kernels.hpp:33-38)
    if constexpr (RUNS) {
      static_assert(EAM, "pair runs: EAM models");
      const float inv_h = tabs[0].inv_h; // the shared grid
      for (int i = w; i < N; i += kPopWarps) {
        const int ti = typ[i];
        const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
        const int p0 = start[i], cnt = A.run_cnt[ga];
        const float gFi = rf[i * kPopLanes + l];
        const double fr0 = A.c.ref_force[3 * ga], fr1 = A.c.ref_force[3 * ga + 1], fr2 = A.c.ref_force[3 * ga + 2];
        float f0 = 0.f, f1 = 0.f, f2 = 0.f, ep = 0.f, s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, s4 = 0.f, s5 = 0.f;
        int cur = -1;
        float4 aP = make_float4(0.f, 0.f, 0.f, 0.f), aJ = aP, aI = aP;
        for (int pb = 0; pb < cnt; pb += 32) {
          if (pb + l < cnt) {
            const int p = p0 + pb + l;
            const float4 ua = A.run_a[p];
            const int2 b = A.run_b[p];
            const float r = A.run_r[p];
            const int tj = b.y >> kRunKeyBits, e = b.y & ((1 << kRunKeyBits) - 1);
            const float hr = 0.5f * r;
            PopRec rec;
            rec.a = ua;
            rec.b = make_float4(hr * ua.x * ua.x, hr * ua.y * ua.y, hr * ua.z * ua.z, hr * ua.x * ua.y);
            rec.c = make_float4(hr * ua.x * ua.z, hr * ua.y * ua.z, 0.f, 0.f);
            rec.ih = make_float4(0.f, 0.f, 0.f, 0.f);
            rec.d = make_int4(b.x & 0xFFFFF, r >= 0.f ? tabs[pair_ord(ti, tj, nt)].seg0 + e : -1, tabs[np + tj].seg0 + e,
                              tabs[np + ti].seg0 + e);
            wst[l] = rec;
          }
          __syncwarp();
          const int c = min(32, cnt - pb);
          for (int q = 0; q < c; ++q) {
            const float4 ra = wst[q].a;
            const int4 rd = wst[q].d;
            if (rd.y < 0) continue; // coincident atoms: no pair term (warp-uniform)
            if (rd.y != cur) {      // a new run (warp-uniform): this trial's three segments
              cur = rd.y;
              aP = coef[rd.y * kPopLanes + l];
              aJ = coef[rd.z * kPopLanes + l];
              aI = coef[rd.w * kPopLanes + l];
            }
            ep += poly_val(aP, ra.w);
            const float g = (poly_der(aP, ra.w) + gFi * poly_der(aJ, ra.w) +
                             rf[rd.x * kPopLanes + l] * poly_der(aI, ra.w)) * inv_h;
            f0 += g * ra.x;
            f1 += g * ra.y;
            f2 += g * ra.z;
            if constexpr (STRESS) {
              const float4 rb = wst[q].b, rc = wst[q].c;
              s0 -= g * rb.x;
              s1 -= g * rb.y;
              s2 -= g * rb.z;
              s3 -= g * rb.w;
              s4 -= g * rc.x;
              s5 -= g * rc.y;
            }
          }
          __syncwarp();
        }
        const double r0 = static_cast<double>(f0) - fr0;
        const double r1 = static_cast<double>(f1) - fr1;
        const double r2 = static_cast<double>(f2) - fr2;
        objf += r0 * r0 + r1 * r1 + r2 * r2;
        e_pair += 0.5 * static_cast<double>(ep);
        sg[0] += s0;
        sg[1] += s1;
        sg[2] += s2;
        sg[3] += s3;
        sg[4] += s4;
        sg[5] += s5;
      }
    } else {
    uint32_t pk = first_batch(w);
    for (int i = w; i < N; i += kPopWarps) {
      const int ti = typ[i];
      const int p0 = start[i], p1 = start[i + 1];
      const float gFi = EAM ? rf[i * kPopLanes + l] : 0.f;
      const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
      const double fr0 = A.c.ref_force[3 * ga], fr1 = A.c.ref_force[3 * ga + 1], fr2 = A.c.ref_force[3 * ga + 2];
      float f0 = 0.f, f1 = 0.f, f2 = 0.f, ep = 0.f, s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, s4 = 0.f, s5 = 0.f;
      if (p0 == p1) pk = first_batch(i + kPopWarps);
      for (int pb = p0; pb < p1; pb += 32) {
        const int p = pb + l;
        const uint32_t cur = pk;
        pk = pb + 32 < p1 ? (pb + 32 + l < p1 ? pack[pb + 32 + l] : 0u) : first_batch(i + kPopWarps);
        if (p < p1) {
          PopRec rec;
          rec.d = make_int4(0, -1, -1, -1);
          rec.a = rec.b = rec.c = rec.ih = make_float4(0.f, 0.f, 0.f, 0.f);
          int j;
          float dx, dy, dz;
          const double r64 = pair_vec_len(wpos, shift, i, cur, j, dx, dy, dz);
          const float r = static_cast<float>(r64);
          if (r64 >= 1e-14) {
            const float inv = 1.f / r, hi = 0.5f * inv;
            rec.d.x = j;
            rec.a = make_float4(dx * inv, dy * inv, dz * inv, 0.f);
            rec.b = make_float4(hi * dx * dx, hi * dy * dy, hi * dz * dz, hi * dx * dy);
            rec.c = make_float4(hi * dx * dz, hi * dy * dz, 0.f, 0.f);
            const int tj = typ[j];
            const STab<float> &tp = tabs[pair_ord(ti, tj, nt)];
            // EAM: closed gate; pair: [rmin, rmax) (pair_force.cpp:28)
            const bool gate = EAM ? gate64(tp, r64) : gate64<false>(tp, r64);
            if (gate) {
              float t;
              rec.d.y = seg_of64(tp, r, r64, t);
              rec.a.w = t;
              rec.ih.x = tp.inv_h;
            }
            if constexpr (EAM) {
              const STab<float> &gj = tabs[np + tj], &gi = tabs[np + ti];
              if (gate64(gj, r64)) {
                float t;
                rec.d.z = seg_of64(gj, r, r64, t);
                rec.c.z = t;
                rec.ih.y = gj.inv_h;
              }
              if (gate64(gi, r64)) {
                float t;
                rec.d.w = seg_of64(gi, r, r64, t);
                rec.c.w = t;
                rec.ih.z = gi.inv_h;
              }
            }
          }
          wst[l] = rec;
        }
        __syncwarp();
        const int cnt = min(32, p1 - pb);
        for (int q = 0; q < cnt; ++q) {
          // the whole record as five 128-bit broadcast loads
          const float4 ra = wst[q].a, rc = wst[q].c, rh = wst[q].ih;
          const int4 rd = wst[q].d;
          float g = 0.f;
          if (rd.y >= 0) {
            const float4 a = coef[rd.y * kPopLanes + l];
            ep += poly_val(a, ra.w);
            g = poly_der(a, ra.w) * rh.x;
          }
          if constexpr (EAM) {
            if (rd.z >= 0) g += gFi * poly_der(coef[rd.z * kPopLanes + l], rc.z) * rh.y;
            if (rd.w >= 0) g += rf[rd.x * kPopLanes + l] * poly_der(coef[rd.w * kPopLanes + l], rc.w) * rh.z;
          }
          f0 += g * ra.x;
          f1 += g * ra.y;
          f2 += g * ra.z;
          if constexpr (STRESS) {
            const float4 rb = wst[q].b;
            s0 -= g * rb.x;
            s1 -= g * rb.y;
            s2 -= g * rb.z;
            s3 -= g * rb.w;
            s4 -= g * rc.x;
            s5 -= g * rc.y;
          }
        }
        __syncwarp();
      }
      const double r0 = static_cast<double>(f0) - fr0;
      const double r1 = static_cast<double>(f1) - fr1;
      const double r2 = static_cast<double>(f2) - fr2;
      objf += r0 * r0 + r1 * r1 + r2 * r2;
      e_pair += 0.5 * static_cast<double>(ep);
      sg[0] += s0;
      sg[1] += s1;
      sg[2] += s2;
      sg[3] += s3;
      sg[4] += s4;
      sg[5] += s5;
    }
    } // RUNS
    // per-(warp, trial) partials into the staging area (16 × 32 × 10 doubles),
    // then a fixed-order sum over warps
    __syncthreads();
    double *pw = reinterpret_cast<double *>(stage) + (w * kPopLanes + l) * 10;
    pw[0] = objf;
    pw[1] = e_emb + e_pair;
    pw[2] = lim;
    for (int a = 0; a < 6; ++a) pw[3 + a] = sg[a];
    __syncthreads();
    if (threadIdx.x < kPopLanes) {
      const double *base = reinterpret_cast<const double *>(stage) + threadIdx.x * 10;
      for (int q = 0; q < 9; ++q) {
        double acc = 0.0;
        for (int ww = 0; ww < kPopWarps; ++ww) acc += base[ww * kPopLanes * 10 + q];
        red[threadIdx.x * 10 + q] = acc;
      }
    }
    __syncthreads();
    if (threadIdx.x < ntr) {
      const double *R = red + threadIdx.x * 10;
      const double iv = 1.0 / cd.volume;
      const double re = A.w_e * (R[1] - cd.ref_energy);
      double o = R[0] + re * re;
      static constexpr int vi[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
      if (A.w_s > 0.0)
        for (int v = 0; v < 6; ++v) {
          const double rs = A.w_s * (R[3 + v] * iv - cd.ref_stress[3 * vi[v][0] + vi[v][1]]);
          o += rs * rs;
        }
      o += R[2] * R[2];
      A.part[static_cast<int64_t>(k0 + threadIdx.x) * A.c.cfg_count + c] = o;
    }
  } // configurations
}

// Σ over configurations in a fixed order (deterministic objective).
__global__ void sum_kernel(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// Jacobian, kernel 1 (EAM): per atom ρ̄, ∂ρ/∂y^ρ, the clamp, F'(ρ̄), F''(ρ̄),
// the embedding knot windows, and the energy / limit rows
// (eam_force.cpp:121-210).
// ---------------------------------------------------------------------------
template <class T> struct JacArgs {
  Common c;
  const typename Vec4T<T>::type *seg_a;
  const T *seg_g;       // [seg][4][kWin]
  const int32_t *seg_ws;
  double w_e, w_s;
  int64_t M;            // rows of J
  int64_t cs, rs;       // J element (row, col) at row·rs + col·cs: (1, ld) row-major, (ld, 1) column-major
  int halves;           // force-row pass: CTAs per configuration (1 or 2)
  double *half_part;    // halves = 2: per (configuration, half) sums [8][D]: energy, 6 stress, Jᵀr
  int D;
  const double *F;      // residual (for the fused Jᵀr)
  double *jtr_part;     // [config][D] Jᵀr partials (FP64)
  int dens_c0, ndens;   // contiguous density columns
  int stage;            // 1: the per-atom Jacobian data of a config fits in shared memory
  T *J;                 // M × D, row- or column-major (cs, rs)
  T *gF, *cF, *over;    // [atom]: F'(ρ̄), F''(ρ̄), clamp overshoot term (0 = unclamped)
  T *drho;              // [atom][ndens]
  T *dgd;               // [atom][kWin]: ∂F'(ρ̄)/∂y over the embedding window
  int32_t *wsF;         // [atom]: embedding window start (knot)
  // FP32 EAM on a knot grid shared by the pair and density tables: each
  // atom's pairs from the sorted pair runs (pair_runs.cu), with u, t and the
  // segment already found (runs = 1)
  const float4 *run_a;  // u, t
  const int2 *run_b;    // packed neighbour entry, run key
  const int32_t *run_cnt;
  int runs;
};

template <class T> size_t jac_common_smem(int n_tables, int n_segs, int n_cmap, int max_atoms, int max_img) {
  size_t b = 0;
  b += align16(n_tables * sizeof(STab<T>));
  b += align16(n_segs * 4 * sizeof(T));
  b += align16(n_segs * 4 * kWin * sizeof(T));
  b += align16(n_segs * sizeof(int32_t));
  b += align16(n_cmap * sizeof(int32_t));
  b += align16(3 * max_atoms * sizeof(double));
  b += align16(3 * max_img * sizeof(double));
  b += align16(max_atoms);
  return b + 128;
}

// Shared-memory copy of the per-atom Jacobian data of one configuration
// (row stride ndens + 1 keeps a warp's column reads on distinct banks).
// The per-atom scalars alone (F', F'', embedding window start, ∂F'/∂y window).
template <class T> size_t atom_scalar_stage_smem(int max_atoms) {
  return 3 * align16(max_atoms * sizeof(T)) + align16(max_atoms * sizeof(int32_t)) +
         align16(static_cast<size_t>(max_atoms) * kWin * sizeof(T)) + 80;
}

template <class T> size_t atom_stage_smem(int max_atoms, int ndens) {
  return align16(static_cast<size_t>(max_atoms) * (ndens + 1) * sizeof(T)) +
         3 * align16(max_atoms * sizeof(T)) + align16(max_atoms * sizeof(int32_t)) +
         align16(static_cast<size_t>(max_atoms) * kWin * sizeof(T)) + 96;
}


// Stage the tables, segment coefficients, window starts and column map, with
// the knot-derivative blocks as one 4-vector per (segment, window knot), so
// that a thread reads a knot's four coefficients in one load
template <class T>
__device__ void stage_tables_g4(const JacArgs<T> &A, STab<T> *tabs, typename Vec4T<T>::type *seg,
                                typename Vec4T<T>::type *G4, int32_t *segws, int32_t *cmap) {
  for (int t = threadIdx.x; t < A.c.n_tables; t += blockDim.x) load_stab(tabs[t], A.c.desc[t]);
  for (int k = threadIdx.x; k < A.c.n_segs; k += blockDim.x) {
    seg[k] = A.seg_a[k];
    segws[k] = A.seg_ws[k];
  }
  for (int k = threadIdx.x; k < A.c.n_segs * kWin; k += blockDim.x) {
    const int sg = k / kWin, q = k - sg * kWin;
    const T *g = A.seg_g + static_cast<size_t>(sg) * 4 * kWin + q;
    G4[k] = typename Vec4T<T>::type{g[0], g[kWin], g[2 * kWin], g[3 * kWin]};
  }
  for (int k = threadIdx.x; k < A.c.n_cmap; k += blockDim.x) cmap[k] = A.c.cmap[k];
}

template <class T>
__global__ void __launch_bounds__(256) jac_atoms_kernel(JacArgs<T> A) {
  using T4 = typename Vec4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  const int nd = A.ndens, ds = nd + 1;
  Smem S(smem_raw);
  STab<T> *tabs = S.take<STab<T>>(A.c.n_tables);
  T4 *seg = S.take<T4>(A.c.n_segs);
  T4 *G4 = S.take<T4>(static_cast<size_t>(A.c.n_segs) * kWin); // [seg][q]: ∂a_0..3/∂y_{ws+q}
  int32_t *segws = S.take<int32_t>(A.c.n_segs);
  int32_t *cmap = S.take<int32_t>(A.c.n_cmap);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  double *erow = S.take<double>(A.D);
  double *lrow = S.take<double>(A.D);
  T *drs = S.take<T>(static_cast<size_t>(N) * ds); // ∂ρ_i/∂y rows (staged)
  T *sgf = S.take<T>(N);
  T *sov = S.take<T>(N);
  stage_tables_g4(A, tabs, seg, G4, segws, cmap);
  for (int k = threadIdx.x; k < A.D; k += blockDim.x) erow[k] = lrow[k] = 0.0;
  for (int k = threadIdx.x; k < N * ds; k += blockDim.x) drs[k] = T(0);
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();
  const int32_t *start = A.c.nb_start + cd.atom0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int64_t ga = static_cast<int64_t>(cd.atom0) + i;
    T *dr = drs + i * ds;
    T rho = T(0);
    for (int p = start[i]; p < start[i + 1]; ++p) {
      int j;
      T dx, dy, dz;
      const uint32_t pk = A.c.nb_pack[p];
      pair_vec(wpos, shift, i, pk, j, dx, dy, dz);
      const T r = sqrt_t(dx * dx + dy * dy + dz * dz);
      const STab<T> &tb = tabs[np + typ[j]];
      T t;
      const int e = gate_seg(tb, r, t, [=] { return pair_len64(wpos, shift, i, pk); });
      if (e < 0) continue;
      rho += seg_val<T>(seg[e], t);
      const int ws = segws[e];
      const T4 *G = G4 + e * kWin;
      // the window's knots are distinct columns: load all, add, store all
      // (knots past the table's end and fixed knots add zero to the pad column nd)
      int m[kWin];
      T add[kWin], cur[kWin];
#pragma unroll
      for (int q = 0; q < kWin; ++q) {
        const int col = ws + q < tb.n ? cmap[tb.cmap0 + ws + q] : -1;
        m[q] = col >= 0 ? col - A.dens_c0 : nd;
        const T4 g = G[q];
        add[q] = col >= 0 ? g.x + t * (g.y + t * (g.z + t * g.w)) : T(0);
      }
#pragma unroll
      for (int q = 0; q < kWin; ++q) cur[q] = dr[m[q]];
#pragma unroll
      for (int q = 0; q < kWin; ++q) dr[m[q]] = cur[q] + add[q];
    }
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
    T t;
    const int e = seg_of(te, rb, t);
    const T gF = seg_der<T>(seg[e], t, te.inv_h);
    A.gF[ga] = gF;
    A.cF[ga] = seg_der2<T>(seg[e], t, te.inv_h);
    A.over[ga] = static_cast<T>(over);
    sgf[i] = gF;
    sov[i] = static_cast<T>(over);
    const int ws = segws[e];
    A.wsF[ga] = ws;
    const T4 *G = G4 + e * kWin;
    for (int q = 0; q < kWin; ++q) {
      const bool ok = ws + q < te.n;
      const T4 g = G[q];
      const T dv = g.x + t * (g.y + t * (g.z + t * g.w));
      const T dd = (g.y + t * (T(2) * g.z + T(3) * t * g.w)) * te.inv_h;
      A.dgd[ga * kWin + q] = ok ? dd : T(0);
      if (!ok) continue;
      const int col = cmap[te.cmap0 + ws + q];
      if (col >= 0) atomicAdd(&erow[col], A.w_e * static_cast<double>(dv));
    }
  }
  __syncthreads();
  // energy row: Σ_i w_e F'_i ∂ρ_i/∂y (unclamped atoms); limit row: Σ over_i ∂ρ_i/∂y
  for (int m = threadIdx.x; m < nd; m += blockDim.x) {
    double e = 0.0, l = 0.0;
    for (int i = 0; i < N; ++i) {
      const double v = static_cast<double>(drs[i * ds + m]);
      const double ov = static_cast<double>(sov[i]);
      if (ov != 0.0)
        l += ov * v;
      else
        e += static_cast<double>(sgf[i]) * v;
    }
    erow[A.dens_c0 + m] += A.w_e * e;
    lrow[A.dens_c0 + m] = l;
  }
  __syncthreads();
  // ∂ρ/∂y of clamped atoms is dropped from the force chain (eam_force.cpp:188-190)
  for (int k = threadIdx.x; k < N * nd; k += blockDim.x) {
    const int i = k / nd, m = k % nd;
    A.drho[(static_cast<int64_t>(cd.atom0) + i) * nd + m] = sov[i] != T(0) ? T(0) : drs[i * ds + m];
  }
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  const int64_t rE = row0 + 3 * N, rL = rE + 1 + (A.w_s > 0.0 ? 6 : 0);
  for (int col = threadIdx.x; col < A.D; col += blockDim.x) {
    A.J[col * A.cs + rE * A.rs] = static_cast<T>(erow[col]);
    A.J[col * A.cs + rL * A.rs] = static_cast<T>(lrow[col]);
  }
}

// ---------------------------------------------------------------------------
// Jacobian, kernel 2: force rows of every atom and the stress rows
// (eam_force.cpp:212-278 / pair_force.cpp:89-110, add_force_column and
// add_radial_bond of include/forcesmith/force/param_jacobian.hpp:91-122).
//
// A warp owns an atom i.  Per chunk of ≤ 32 neighbours the lanes build pair
// records; then, pair by pair, 24 lanes scatter the knot-window terms
//   φ'       (col window of φ_{t_i t_j})         weight 1
//   ρ'_{tj}  (window of ρ_{t_j})                 weight F'_i
//   ρ'_{ti}  (window of ρ_{t_i})                 weight F'_j
//   F'_j     (embedding window of j)             weight ρ'_{t_i}(r)
// into the warp's row buffer (distinct columns per pair, no atomics), and
// every lane adds the dense ρ-chain term Σ_j F''_j ρ'_{t_i}(r) u drho_j for
// the density columns it owns.
//
// Stress rows, W = Σ_pairs d ⊗ ∂f/∂y over the full list.  The pair force is
// antisymmetric under (i, j, s) → (j, i, −s) (its scalar is symmetric in i, j
// and u flips), and d = x_j + s − x_i, so
//   W = −2 Σ_i (x_i − c) ⊗ ∂F_i/∂y + Σ_{pairs with s ≠ 0} s ⊗ ∂f/∂y
// for any origin c (Σ_i ∂F_i/∂y = 0); c is the cell centre.  The first term is
// added when atom i's rows are written; only pairs that leave the cell (about
// a third here) scatter stress.  Their chain terms use the same symmetry:
// Σ (s ⊗ u)(F''_i drho_i ρ'_{tj} + F''_j drho_j ρ'_{ti}) = 2 Σ_i P_i F''_i drho_i
// with P_i = Σ_{j, s≠0} (s ⊗ u) ρ'_{tj}(r_ij).
// The configuration's per-atom data (∂ρ/∂y rows, F', F'', embedding windows)
// is staged in shared memory when it fits, so the inner loops never wait on
// global memory.
// ---------------------------------------------------------------------------
template <class T> struct V2T;
template <> struct V2T<float> { using type = float2; };
template <> struct V2T<double> { using type = double2; };

// One pair, laid out for vector loads: a scatter lane reads its slot with
// one 128-bit load (FP32), and the neighbour terms read (weight, j) at once.
// Per slot (0: φ, 1: ρ_{tj} direct, 2: ρ_{ti} direct, 3: F_j window): index of
// the segment's first knot-derivative 4-vector, column-map index of the
// window's first knot (0, the map's leading block of −1, when the slot adds
// nothing; knots past the table's end read the −1 padding after it), local
// coordinate t, weight × the table's 1/h (F window: ρ'_{ti}(r)).
template <class T> struct SlotRec;
template <> struct __align__(16) SlotRec<float> {
  int g, c;
  float t, w;
};
template <> struct __align__(16) SlotRec<double> {
  int g, c, pad0, pad1;
  double t, w;
};
// F''_j ρ'_{ti}(r) (the dense ρ-chain weight); j, with bit 31 set when the
// pair leaves the cell and stress is wanted
template <class T> struct JW;
template <> struct __align__(8) JW<float> {
  float w;
  int jc;
};
template <> struct __align__(16) JW<double> {
  double w;
  int jc, pad;
};
template <class T> struct PairRec {
  SlotRec<T> s[4];
  typename Vec4T<T>::type uv; // u_x, u_y, u_z, v_xx     (v = s ⊗ u for pairs that leave the
  typename Vec4T<T>::type vv; // v_yy, v_zz, v_xy, v_xz  cell, image shift s; zero otherwise)
  T vyz;                      // v_yz
  JW<T> jw;
};

constexpr int kPairStep = 4; // pairs whose scatter terms are formed together
// warps per CTA of the force-row kernel: at most 11 in FP32 (the per-warp row
// buffers of 11 warps fill the shared memory), 8 in FP64 (registers)
template <class T> constexpr int kMaxK2Warps = sizeof(T) == 4 ? 11 : 8;

// A configuration's column of the energy, stress and limit rows, from the
// force-row pass's sums over its atoms (φ energy e, stress s, Jᵀr over the
// force rows jr), and its Jᵀr over all its rows into jtr_part.
template <class T, bool EAM>
__device__ void finish_cfg_column(const JacArgs<T> &A, int c, int col, double e, const double (&s)[6], double jr) {
  const CfgDev &cd = A.c.cfg[c];
  const bool want_stress = A.w_s > 0.0;
  const int64_t rows_per_extra = 2 + (want_stress ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  const int64_t rE = row0 + 3 * cd.natoms;
  const int64_t rL = rE + 1 + (want_stress ? 6 : 0);
  const double sc = -A.w_s * 0.5 / cd.volume;
  T *Jc = A.J + static_cast<int64_t>(col) * A.cs; // row r of this column: Jc[r · rs]
  const int64_t rs = A.rs;
  if constexpr (EAM)
    Jc[rE * rs] = static_cast<T>(static_cast<double>(Jc[rE * rs]) + e);
  else
    Jc[rE * rs] = static_cast<T>(e);
  // Jᵀr over this configuration's rows: force rows (jr), energy, stress, limit
  jr += static_cast<double>(Jc[rE * rs]) * A.F[rE];
  if constexpr (EAM) jr += static_cast<double>(Jc[rL * rs]) * A.F[rL];
  if (want_stress)
    for (int v = 0; v < 6; ++v) {
      Jc[(rE + 1 + v) * rs] = static_cast<T>(sc * s[v]);
      jr += static_cast<double>(Jc[(rE + 1 + v) * rs]) * A.F[rE + 1 + v];
    }
  if constexpr (!EAM) Jc[rL * rs] = T(0); // limit row: no embedding
  A.jtr_part[static_cast<int64_t>(c) * A.D + col] = jr;
}

template <class T, bool EAM, int STAGE>
__global__ void __launch_bounds__(32 * kMaxK2Warps<T>, 1) jac_forces_kernel(JacArgs<T> A, int warps) {
  using T4 = typename Vec4T<T>::type;
  using T2 = typename V2T<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // halves = 2: two CTAs per configuration, taking alternate strides of its
  // atoms (shorter CTAs fill the last wave of SMs better)
  const int c = blockIdx.x / A.halves, half = blockIdx.x % A.halves;
  const int astep = warps * A.halves;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms;
  const int D = A.D;
  const int nt = A.c.ntypes, np = nt * (nt + 1) / 2;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  const int nd = A.ndens;
  Smem S(smem_raw);
  STab<T> *tabs = S.take<STab<T>>(A.c.n_tables);
  T4 *seg = S.take<T4>(A.c.n_segs);
  T4 *G4 = S.take<T4>(static_cast<size_t>(A.c.n_segs) * kWin); // [seg][q]: ∂a_0..3/∂y_{ws+q}
  int32_t *segws = S.take<int32_t>(A.c.n_segs);
  int32_t *cmap = S.take<int32_t>(A.c.n_cmap);
  double *wpos = S.take<double>(3 * N);
  double *shift = S.take<double>(3 * nimg);
  uint8_t *typ = S.take<uint8_t>(N);
  // per warp: force rows + φ energy as [col] × (x, y, z, e); stress as
  // [col] × 3 pairs (xx,yy)(zz,xy)(xz,yz); energy row; pair records
  T4 *frow_all = S.take<T4>(static_cast<size_t>(warps) * (D + 1)); // + a spare column
  T2 *srow_all = S.take<T2>(static_cast<size_t>(warps) * 3 * D);
  T *erow_all = S.take<T>(static_cast<size_t>(warps) * D);
  PairRec<T> *recs = S.take<PairRec<T>>(static_cast<size_t>(warps) * 32);
  double *jtr_all = S.take<double>(static_cast<size_t>(warps) * D);
  int32_t *s_start = S.take<int32_t>(N + 1); // the configuration's neighbour offsets
  for (int k = threadIdx.x; k <= N; k += blockDim.x) s_start[k] = A.c.nb_start[cd.atom0 + k];
  const T *drho = A.drho + static_cast<int64_t>(cd.atom0) * nd;
  int dstr = nd;
  const T *gFa = A.gF + cd.atom0, *cFa = A.cF + cd.atom0, *dgda = A.dgd + static_cast<int64_t>(cd.atom0) * kWin;
  const int32_t *wsFa = A.wsF + cd.atom0;
  // STAGE 1: the configuration's per-atom scalars and ∂F'/∂y windows come
  // from shared memory; STAGE 2: also the ∂ρ/∂y rows (the pointers below then
  // address the shared window only)
  if constexpr (EAM && STAGE == 2) {
    T *s_dr = S.take<T>(static_cast<size_t>(N) * (nd + 1));
    for (int k = threadIdx.x; k < N * nd; k += blockDim.x) s_dr[(k / nd) * (nd + 1) + k % nd] = drho[k];
    drho = s_dr;
    dstr = nd + 1;
  }
  if constexpr (EAM && STAGE >= 1) {
    T *s_gf = S.take<T>(N);
    T *s_cf = S.take<T>(N);
    T *s_pad = S.take<T>(N);
    int32_t *s_ws = S.take<int32_t>(N);
    T *s_dgd = S.take<T>(static_cast<size_t>(N) * kWin);
    (void)s_pad;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
      s_gf[k] = gFa[k];
      s_cf[k] = cFa[k];
      s_ws[k] = wsFa[k];
    }
    for (int k = threadIdx.x; k < N * kWin; k += blockDim.x) s_dgd[k] = dgda[k];
    gFa = s_gf;
    cFa = s_cf;
    wsFa = s_ws;
    dgda = s_dgd;
  }
  stage_tables_g4(A, tabs, seg, G4, segws, cmap);
  for (int k = threadIdx.x; k < warps * 3 * D; k += blockDim.x) srow_all[k] = T2{T(0), T(0)};
  for (int k = threadIdx.x; k < warps * D; k += blockDim.x) {
    erow_all[k] = T(0);
    jtr_all[k] = 0.0;
  }
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T4 *frow = frow_all + static_cast<size_t>(w) * (D + 1);
  T2 *srow = srow_all + static_cast<size_t>(w) * 3 * D;
  T *erow = erow_all + static_cast<size_t>(w) * D;
  double *jtr = jtr_all + static_cast<size_t>(w) * D;
  PairRec<T> *rec = recs + w * 32;
  const int32_t *start = s_start;
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  const T half_we = static_cast<T>(0.5 * A.w_e);
  const bool want_stress = A.w_s > 0.0;
  // scatter lanes: lane = slot × 8 + knot, knots 6, 7 idle, so each 8-lane
  // phase of a 128-bit row-buffer access covers one window's consecutive
  // columns (distinct banks); idle lanes address knot 0 and add nothing
  const int slot = lane >> 3, q = (lane & 7) < kWin ? (lane & 7) : 0;
  const int slot_c = slot;
  const bool lane_ok = (lane & 7) < kWin;
  const int home = (cd.sx * (2 * cd.sy + 1) + cd.sy) * (2 * cd.sz + 1) + cd.sz; // image (0, 0, 0)
  double ctr[3];                                                                   // cell centre
  for (int a = 0; a < 3; ++a) ctr[a] = 0.5 * (cd.box[3 * a] + cd.box[3 * a + 1] + cd.box[3 * a + 2]);

  // each chunk's packed neighbour entries are loaded one chunk ahead
  int pre_p0 = -1;
  uint32_t pk_next = 0;
  float4 ra_next = make_float4(0.f, 0.f, 0.f, 0.f);
  int2 rb_next = make_int2(0, 0);
  constexpr bool kRunsOK = EAM && std::is_same_v<T, float>;
  const bool runs = kRunsOK && A.runs;
  // end of atom ii's pairs: its in-gate pair runs, else its neighbour list
  auto end_of = [&](int ii) { return runs ? start[ii] + A.run_cnt[cd.atom0 + ii] : start[ii + 1]; };
  auto prefetch = [&](int p, int end) {
    pre_p0 = p;
    const bool in = lane < end - p;
    if (runs) {
      rb_next = in ? A.run_b[p + lane] : make_int2(0, 0);
      ra_next = in ? A.run_a[p + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      pk_next = in ? A.c.nb_pack[p + lane] : 0u;
    }
  };
  const int i_first = w + half * warps;
  if (i_first < N) prefetch(start[i_first], end_of(i_first));
  for (int i = i_first; i < N; i += astep) {
    for (int k = lane; k <= D; k += 32) frow[k] = T4{T(0), T(0), T(0), T(0)};
    const int ti = typ[i];
    T gFi = T(0), cFi = T(0);
    int wsFi = 0;
    if constexpr (EAM) {
      gFi = gFa[i];
      cFi = cFa[i];
      wsFi = wsFa[i];
    }
    T V[3] = {0, 0, 0}, P[6] = {0, 0, 0, 0, 0, 0};
    T dacc[2][3] = {{0, 0, 0}, {0, 0, 0}}; // dense ρ-chain, columns m = lane, lane + 32
    __syncwarp();
    const int iend = end_of(i);
    for (int p0 = start[i]; p0 < iend; p0 += 32) {
      const int cnt = min(32, iend - p0);
      uint32_t pk_cur = pk_next;
      float4 ra_cur = ra_next;
      int2 rb_cur = rb_next;
      if (pre_p0 != p0) { // (after an atom without pairs)
        if (runs) {
          rb_cur = lane < cnt ? A.run_b[p0 + lane] : make_int2(0, 0);
          ra_cur = lane < cnt ? A.run_a[p0 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
          pk_cur = lane < cnt ? A.c.nb_pack[p0 + lane] : 0u;
        }
      }
      {
        int np0 = p0 + 32, nend = iend;
        if (np0 >= nend) {
          const int in = i + astep;
          np0 = in < N ? start[in] : 0;
          nend = in < N ? end_of(in) : 0;
        }
        prefetch(np0, nend);
      }
      if constexpr (kRunsOK) {
        if (runs && lane < cnt) {
          // a pair run record: u and t on the shared grid, the segment in the key
          PairRec<T> R;
          const uint32_t pk = static_cast<uint32_t>(rb_cur.x);
          const int j = static_cast<int>(pk & 0xFFFFFu), img = static_cast<int>(pk >> 20);
          const int tj = rb_cur.y >> kRunKeyBits, e = rb_cur.y & ((1 << kRunKeyBits) - 1);
          const int cross = want_stress && img != home;
          const T t = ra_cur.w, u[3] = {ra_cur.x, ra_cur.y, ra_cur.z};
          R.jw.jc = static_cast<int>(static_cast<uint32_t>(j) | (cross ? 0x80000000u : 0u));
          for (int s = 0; s < 4; ++s) {
            R.s[s].g = R.s[s].c = 0;
            R.s[s].t = R.s[s].w = T(0);
          }
          T dgi = T(0), dgj = T(0), cFj = T(0), v[6] = {0, 0, 0, 0, 0, 0};
          if (u[0] != T(0) || u[1] != T(0) || u[2] != T(0)) { // (coincident atoms: no pair term)
            if (cross) {
              const T s0 = static_cast<T>(shift[3 * img]), s1 = static_cast<T>(shift[3 * img + 1]),
                      s2 = static_cast<T>(shift[3 * img + 2]);
              v[0] = s0 * u[0];
              v[1] = s1 * u[1];
              v[2] = s2 * u[2];
              v[3] = s0 * u[1];
              v[4] = s0 * u[2];
              v[5] = s1 * u[2];
            }
            auto set_slot = [&](int sl, const STab<T> &tb, int sg, T wgt) {
              R.s[sl].g = sg * kWin;
              R.s[sl].c = tb.cmap0 + segws[sg];
              R.s[sl].t = t;
              R.s[sl].w = wgt * tb.inv_h;
            };
            const STab<T> &tp = tabs[pair_ord(ti, tj, nt)], &gj = tabs[np + tj], &gi_ = tabs[np + ti];
            set_slot(0, tp, tp.seg0 + e, T(1));
            const T gFj = gFa[j];
            cFj = cFa[j];
            set_slot(1, gj, gj.seg0 + e, tj == ti ? gFi + gFj : gFi);
            dgj = seg_der<T>(seg[gj.seg0 + e], t, gj.inv_h);
            if (tj == ti) {
              dgi = dgj;
            } else {
              dgi = seg_der<T>(seg[gi_.seg0 + e], t, gi_.inv_h);
              set_slot(2, gi_, gi_.seg0 + e, gFj);
            }
            const STab<T> &te = tabs[np + nt + tj];
            R.s[3].c = te.cmap0 + wsFa[j];
            R.s[3].w = dgi;
          }
          R.uv = {u[0], u[1], u[2], v[0]};
          R.vv = {v[1], v[2], v[3], v[4]};
          R.vyz = v[5];
          R.jw.w = cFj * dgi;
          rec[lane] = R;
          for (int a = 0; a < 3; ++a) V[a] += dgj * u[a];
          for (int a = 0; a < 6; ++a) P[a] += dgj * v[a];
        }
      }
      if (!runs && lane < cnt) {
        PairRec<T> R;
        int j;
        T d[3];
        const uint32_t pk = pk_cur;
        pair_vec(wpos, shift, i, pk, j, d[0], d[1], d[2]);
        const T r = sqrt_t(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const int tj = typ[j];
        const int img = static_cast<int>(pk >> 20);
        const int cross = want_stress && img != home; // the pair leaves the cell: image shift s ≠ 0
        R.jw.jc = static_cast<int>(static_cast<uint32_t>(j) | (cross ? 0x80000000u : 0u));
        for (int s = 0; s < 4; ++s) {
          R.s[s].g = R.s[s].c = 0;
          R.s[s].t = R.s[s].w = T(0);
        }
        T dgi = T(0), cFj = T(0), u[3] = {0, 0, 0}, v[6] = {0, 0, 0, 0, 0, 0};
        T dgj = T(0);
        if (r >= T(1e-14)) {
          const T ir = T(1) / r;
          for (int a = 0; a < 3; ++a) u[a] = d[a] * ir;
          if (cross) { // v = s ⊗ u in the order xx, yy, zz, xy, xz, yz
            const T s0 = static_cast<T>(shift[3 * img]), s1 = static_cast<T>(shift[3 * img + 1]),
                    s2 = static_cast<T>(shift[3 * img + 2]);
            v[0] = s0 * u[0];
            v[1] = s1 * u[1];
            v[2] = s2 * u[2];
            v[3] = s0 * u[1];
            v[4] = s0 * u[2];
            v[5] = s1 * u[2];
          }
          const auto r64 = [=] { return pair_len64(wpos, shift, i, pk); };
          auto set_slot = [&](int s, const STab<T> &tb, int e, T t, T wgt) {
            R.s[s].g = e * kWin;
            R.s[s].c = tb.cmap0 + segws[e];
            R.s[s].t = t;
            R.s[s].w = wgt * tb.inv_h;
          };
          const STab<T> &tp = tabs[pair_ord(ti, tj, nt)];
          T tq;
          const int ep = gate_seg<EAM>(tp, r, tq, r64);
          if (ep >= 0) set_slot(0, tp, ep, tq, T(1));
          if constexpr (EAM) {
            const STab<T> &gj = tabs[np + tj], &gi_ = tabs[np + ti];
            const T gFj = gFa[j];
            cFj = cFa[j];
            T tj_;
            const int ej = gate_seg(gj, r, tj_, r64);
            if (ej >= 0) {
              set_slot(1, gj, ej, tj_, tj == ti ? gFi + gFj : gFi);
              dgj = seg_der<T>(seg[ej], tj_, gj.inv_h);
            }
            if (tj == ti) {
              dgi = dgj; // the same table at the same distance
            } else {
              T ti_;
              const int ei = gate_seg(gi_, r, ti_, r64);
              if (ei >= 0) {
                dgi = seg_der<T>(seg[ei], ti_, gi_.inv_h);
                set_slot(2, gi_, ei, ti_, gFj);
              }
            }
            // F_j window: coefficient dgd_j[q]·ρ'_{ti}(r)
            const STab<T> &te = tabs[np + nt + tj];
            const int wsj = wsFa[j];
            R.s[3].c = te.cmap0 + wsj;
            R.s[3].w = dgi;
          }
        }
        R.uv = {u[0], u[1], u[2], v[0]};
        R.vv = {v[1], v[2], v[3], v[4]};
        R.vyz = v[5];
        R.jw.w = cFj * dgi;
        rec[lane] = R;
        for (int a = 0; a < 3; ++a) V[a] += dgj * u[a];
        for (int a = 0; a < 6; ++a) P[a] += dgj * v[a];
      }
      __syncwarp();
      // sparse knot-window scatter, 24 lanes = 4 slots × 6 knots per pair.
      // kPairStep pairs per step: their columns, coefficients and the dense
      // ρ-chain terms are computed together (independent work), then the
      // read-modify-writes of the row buffer go one pair at a time (windows
      // of different pairs may share columns across lanes).  Unused slots add
      // zero to the spare column D.
#pragma unroll 1
      for (int k0 = 0; k0 < cnt; k0 += kPairStep) {
        int col[kPairStep];
        T cf[kPairStep], dv[kPairStep];
        bool st[kPairStep];
        T4 uvs[kPairStep];
        T dval[kPairStep][2], dwgt[kPairStep], fwin[kPairStep];
        bool crs[kPairStep];
        if constexpr (EAM) {
          // per-atom loads go out first: the F-window terms ∂F'_j/∂y_q (slot 3
          // lanes) and the dense ρ-chain's ∂ρ_j/∂y, used after the row updates
#pragma unroll
          for (int u = 0; u < kPairStep; ++u) {
            const bool live = k0 + u < cnt;
            const JW<T> jw = rec[live ? k0 + u : k0].jw;
            const int jj = jw.jc & 0x7FFFFFFF;
            crs[u] = jw.jc < 0;
            fwin[u] = slot_c == 3 ? dgda[jj * kWin + q] : T(0);
            dwgt[u] = live ? jw.w : T(0);
            const T *drj = drho + jj * dstr;
#pragma unroll
            for (int s2 = 0; s2 < 2; ++s2) {
              const int m = lane + 32 * s2;
              dval[u][s2] = (m < nd && dwgt[u] != T(0)) ? drj[m] : T(0);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < kPairStep; ++u) {
          const bool live = k0 + u < cnt;
          const PairRec<T> &R = rec[live ? k0 + u : k0];
          const SlotRec<T> sr = R.s[slot_c];
          const int c0 = cmap[sr.c + q]; // −1: no term (padding, fixed knot, unused slot)
          const T tt = sr.t;
          const T4 G = G4[sr.g + q];
          if constexpr (!EAM) crs[u] = R.jw.jc < 0;
          const T g0 = G.x, g1 = G.y, g2 = G.z, g3 = G.w;
          T base = g1 + tt * (T(2) * g2 + T(3) * tt * g3);
          if constexpr (EAM)
            if (slot_c == 3) base = fwin[u]; // F window of j: ∂F'_j/∂y_q
          const bool use = live && lane_ok && c0 >= 0;
          col[u] = use ? c0 : D;
          cf[u] = use ? sr.w * base : T(0);
          dv[u] = (use && slot == 0) ? half_we * (g0 + tt * (g1 + tt * (g2 + tt * g3))) : T(0);
          st[u] = use && crs[u] && slot < 3; // the F window carries no stress term here
          uvs[u] = R.uv;
        }
#pragma unroll
        for (int u = 0; u < kPairStep; ++u) {
          const int cu = col[u];
          T4 fr = frow[cu];
          fr.x += cf[u] * uvs[u].x;
          fr.y += cf[u] * uvs[u].y;
          fr.z += cf[u] * uvs[u].z;
          fr.w += dv[u];
          frow[cu] = fr;
          if (st[u]) { // stress scatter: pairs that leave the cell only
            const PairRec<T> &R = rec[k0 + u];
            const T4 vv = R.vv;
            const T v5 = R.vyz, c = cf[u];
            T2 s0 = srow[3 * cu], s1 = srow[3 * cu + 1], s2 = srow[3 * cu + 2];
            s0.x += c * uvs[u].w;
            s0.y += c * vv.x;
            s1.x += c * vv.y;
            s1.y += c * vv.z;
            s2.x += c * vv.w;
            s2.y += c * v5;
            srow[3 * cu] = s0;
            srow[3 * cu + 1] = s1;
            srow[3 * cu + 2] = s2;
          }
          __syncwarp();
        }
        if constexpr (EAM) {
          // dense ρ-chain: Σ_j F''_j ρ'_{ti}(r) u drho_j[m]
#pragma unroll
          for (int u = 0; u < kPairStep; ++u)
#pragma unroll
            for (int s2 = 0; s2 < 2; ++s2) {
              const T dd = dwgt[u] * dval[u][s2];
              dacc[s2][0] += dd * uvs[u].x;
              dacc[s2][1] += dd * uvs[u].y;
              dacc[s2][2] += dd * uvs[u].z;
            }
        }
      }
      __syncwarp();
    }
    for (int a = 0; a < 3; ++a) V[a] = warp_sum_group(V[a], 32);
    for (int a = 0; a < 6; ++a) P[a] = warp_sum_group(P[a], 32);
    if constexpr (EAM) {
      const T *dri = drho + i * dstr;
      for (int s2 = 0; s2 < 2; ++s2) {
        const int m = lane + 32 * s2;
        if (m < nd) {
          const T gim = cFi * dri[m];
          const int col = A.dens_c0 + m;
          T4 fr = frow[col];
          fr.x += dacc[s2][0] + gim * V[0];
          fr.y += dacc[s2][1] + gim * V[1];
          fr.z += dacc[s2][2] + gim * V[2];
          frow[col] = fr;
          if (want_stress) {
            const T g2 = T(2) * gim;
            srow[3 * col].x += g2 * P[0];
            srow[3 * col].y += g2 * P[1];
            srow[3 * col + 1].x += g2 * P[2];
            srow[3 * col + 1].y += g2 * P[3];
            srow[3 * col + 2].x += g2 * P[4];
            srow[3 * col + 2].y += g2 * P[5];
          }
        }
      }
      __syncwarp();
      if (lane < kWin) {
        const STab<T> &te = tabs[np + nt + ti];
        const int knot = wsFi + lane;
        const int col = knot < te.n ? cmap[te.cmap0 + knot] : -1;
        const T dg = dgda[i * kWin + lane];
        if (col >= 0 && dg != T(0)) {
          T4 fr = frow[col];
          fr.x += dg * V[0];
          fr.y += dg * V[1];
          fr.z += dg * V[2];
          frow[col] = fr;
          if (want_stress) {
            const T g2 = T(2) * dg;
            srow[3 * col].x += g2 * P[0];
            srow[3 * col].y += g2 * P[1];
            srow[3 * col + 1].x += g2 * P[2];
            srow[3 * col + 1].y += g2 * P[3];
            srow[3 * col + 2].x += g2 * P[4];
            srow[3 * col + 2].y += g2 * P[5];
          }
        }
      }
    }
    __syncwarp();
    const double F0 = A.F[row0 + 3 * i], F1 = A.F[row0 + 3 * i + 1], F2 = A.F[row0 + 3 * i + 2];
    const T x0 = static_cast<T>(-2.0 * (wpos[3 * i] - ctr[0])), x1 = static_cast<T>(-2.0 * (wpos[3 * i + 1] - ctr[1])),
            x2 = static_cast<T>(-2.0 * (wpos[3 * i + 2] - ctr[2]));
    // Streaming stores: J is written once here and read once by JᵀJ, so it
    // should not evict the ∂ρ/∂y rows this kernel rereads from L2.  Row-major
    // J: each of the atom's 3 rows is one coalesced store per 32 columns.
    // Column-major J: the atom's 3 rows of a column in two stores, a pair on
    // its even row (ld is a multiple of 32, so the row parity is the address
    // parity).
    const bool rowm = A.cs == 1;
    const bool even = ((row0 + 3 * i) & 1) == 0;
    T *Ji = A.J + (row0 + 3 * i) * A.rs;
    for (int col = lane; col < D; col += 32) {
      const T4 fr = frow[col];
      if (rowm) {
        __stcs(Ji + col, fr.x);
        __stcs(Ji + A.rs + col, fr.y);
        __stcs(Ji + 2 * A.rs + col, fr.z);
      } else {
        T *Jc = Ji + static_cast<int64_t>(col) * A.cs;
        if (even) {
          __stcs(reinterpret_cast<T2 *>(Jc), T2{fr.x, fr.y});
          __stcs(Jc + 2, fr.z);
        } else {
          __stcs(Jc, fr.x);
          __stcs(reinterpret_cast<T2 *>(Jc + 1), T2{fr.y, fr.z});
        }
      }
      erow[col] += fr.w;
      jtr[col] += static_cast<double>(fr.x) * F0 + static_cast<double>(fr.y) * F1 + static_cast<double>(fr.z) * F2;
      if (want_stress) { // −2 (x_i − c) ⊗ ∂F_i/∂y: the in-cell part of Σ_pairs d ⊗ ∂f/∂y
        T2 s0 = srow[3 * col], s1 = srow[3 * col + 1], s2 = srow[3 * col + 2];
        s0.x += x0 * fr.x;
        s0.y += x1 * fr.y;
        s1.x += x2 * fr.z;
        s1.y += x0 * fr.y;
        s2.x += x0 * fr.z;
        s2.y += x1 * fr.z;
        srow[3 * col] = s0;
        srow[3 * col + 1] = s1;
        srow[3 * col + 2] = s2;
      }
    }
    __syncwarp();
  }
  __syncthreads();
  for (int col = threadIdx.x; col < D; col += blockDim.x) {
    double e = 0.0, jr = 0.0, s[6] = {0, 0, 0, 0, 0, 0};
    for (int ww = 0; ww < warps; ++ww) {
      e += static_cast<double>(erow_all[static_cast<size_t>(ww) * D + col]);
      jr += jtr_all[static_cast<size_t>(ww) * D + col];
    }
    if (want_stress)
      for (int ww = 0; ww < warps; ++ww) {
        const T2 *sr = srow_all + static_cast<size_t>(ww) * 3 * D + 3 * col;
        s[0] += static_cast<double>(sr[0].x);
        s[1] += static_cast<double>(sr[0].y);
        s[2] += static_cast<double>(sr[1].x);
        s[3] += static_cast<double>(sr[1].y);
        s[4] += static_cast<double>(sr[2].x);
        s[5] += static_cast<double>(sr[2].y);
      }
    if (A.halves == 1) {
      finish_cfg_column<T, EAM>(A, c, col, e, s, jr);
    } else { // the combine kernel adds the halves in order and finishes the column
      double *hp = A.half_part + (static_cast<int64_t>(c) * 2 + half) * 8 * D + col;
      hp[0] = e;
      for (int v = 0; v < 6; ++v) hp[(1 + v) * D] = s[v];
      hp[7 * D] = jr;
    }
  }
}

// halves = 2: configuration blockIdx.x's columns from its two CTAs' sums
template <class T, bool EAM> __global__ void __launch_bounds__(256) jac_halves_combine(JacArgs<T> A) {
  const int c = blockIdx.x, D = A.D;
  const double *h0 = A.half_part + static_cast<int64_t>(c) * 2 * 8 * D, *h1 = h0 + 8 * D;
  for (int col = threadIdx.x; col < D; col += blockDim.x) {
    double s[6];
    for (int v = 0; v < 6; ++v) s[v] = h0[(1 + v) * D + col] + h1[(1 + v) * D + col];
    finish_cfg_column<T, EAM>(A, c, col, h0[col] + h1[col], s, h0[7 * D + col] + h1[7 * D + col]);
  }
}

__global__ void jtr_reduce_kernel(const double *__restrict__ part, int n_cfg, int D, double *__restrict__ Jtr) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= D) return;
  double s = 0.0;
  for (int c = 0; c < n_cfg; ++c) s += part[static_cast<int64_t>(c) * D + col];
  Jtr[col] = s;
}

int choose_lpa(const fs_gpu *h) {
  if (h->lanes_per_atom) return h->lanes_per_atom;
  if (h->tuned_lpa) return h->tuned_lpa;
  const double avg = h->n_atoms ? static_cast<double>(h->n_pairs) / h->n_atoms : 0.0;
  if (avg > 24) return 16;
  if (avg > 10) return 8;
  return 4;
}

template <class T, int LPA, bool EAM> int launch_residual_t(fs_gpu *h, double w_e, double w_s) {
  using T4 = typename Vec4T<T>::type;
  ResArgs<T> a;
  a.c = make_common<T>(h);
  a.seg_a = static_cast<const T4 *>(h->d_seg_a);
  a.w_e = w_e;
  a.w_s = w_s;
  a.F = h->d_F;
  a.forces = h->d_forces;
  a.energy = h->d_energy;
  a.stress9 = h->d_stress9;
  a.limit = h->d_limit;
  a.obj_part = h->d_obj_part;
  const size_t sm = residual_smem<T>(a.c.n_tables, h->n_segs, h->max_natoms, max_images(h));
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "residual: configuration too large for shared memory");
  bool analytic = false;
  for (const HostTable &t : h->tables) analytic = analytic || t.kind == FS_TABLE_ANALYTIC;
  auto k = analytic ? residual_kernel<T, LPA, EAM, true> : residual_kernel<T, LPA, EAM, false>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, 256, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  sum_kernel<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

template <class T, bool EAM> int launch_residual_lpa(fs_gpu *h, double w_e, double w_s) {
  switch (choose_lpa(h)) {
  case 4: return launch_residual_t<T, 4, EAM>(h, w_e, w_s);
  case 8: return launch_residual_t<T, 8, EAM>(h, w_e, w_s);
  case 16: return launch_residual_t<T, 16, EAM>(h, w_e, w_s);
  default: return launch_residual_t<T, 32, EAM>(h, w_e, w_s);
  }
}

template <class X> int grow(fs_gpu *h, X **p, size_t n, size_t &have) {
  if (have >= n && *p) return FS_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(X)) != cudaSuccess)
    return set_error(h, FS_ERR_NOMEM, "cudaMalloc (Jacobian)");
  have = n;
  return FS_OK;
}

template <class T> int launch_jacobian_t(fs_gpu *h, double w_e, double w_s) {
  using T4 = typename Vec4T<T>::type;
  const bool eam = h->family == FS_FAMILY_EAM;
  const int64_t M = rows_of(h, w_s);
  const int D = h->D;
  // J, rows rounded up to 32 (padding rows stay zero).  When the tensor cores
  // form JᵀJ (FP32, 48 < D ≤ 256): row-major with the row stride rounded up to 4
  // columns (16 bytes, as a TMA stride needs), so that an atom's rows are
  // contiguous and its stores coalesce.  Otherwise column-major with the
  // leading dimension the padded row count.
  const bool rowmajor = gram_on_tensor_cores(h->precision, D);
  const int64_t rows = (M + 31) / 32 * 32;
  const int64_t ldj = rowmajor ? (D + 3) / 4 * 4 : rows;
  const size_t jn = static_cast<size_t>(rowmajor ? rows * ldj : ldj * D);
  if (static_cast<size_t>(h->jac_alloc) != jn || h->ldj != ldj || !h->d_J || h->j_rowmajor != rowmajor) {
    if (h->d_J) cudaFree(h->d_J);
    h->d_J = nullptr;
    if (cudaMalloc(&h->d_J, std::max<size_t>(jn, 1) * sizeof(T)) != cudaSuccess)
      return set_error(h, FS_ERR_NOMEM, "cudaMalloc (J)");
    FS_CUDA(cudaMemsetAsync(h->d_J, 0, std::max<size_t>(jn, 1) * sizeof(T), h->stream));
    h->jac_alloc = static_cast<int64_t>(jn);
    h->ldj = ldj;
    h->j_rowmajor = rowmajor;
  }
  {
    const size_t need = static_cast<size_t>(h->n_cfg) * D;
    if (h->jtr_part_alloc < need || !h->d_jtr_part) {
      if (h->d_jtr_part) cudaFree(h->d_jtr_part);
      h->d_jtr_part = nullptr;
      FS_CUDA(cudaMalloc(&h->d_jtr_part, std::max<size_t>(need, 1) * sizeof(double)));
      h->jtr_part_alloc = need;
    }
  }
  if (!h->d_JtJ) {
    FS_CUDA(cudaMalloc(&h->d_JtJ, std::max(D * D, 1) * sizeof(double)));
    FS_CUDA(cudaMalloc(&h->d_Jtr, std::max(D, 1) * sizeof(double)));
  }
  // density columns: tables [np, np+nt) are contiguous in the column space
  const int nt = h->ntypes, np = npair_of(nt);
  int dens_c0 = 0, ndens = 0;
  if (eam) {
    int lo = 1 << 30, hi = -1;
    for (int t = np; t < np + nt; ++t)
      for (int col : h->tables[t].cols)
        if (col >= 0) {
          lo = std::min(lo, col);
          hi = std::max(hi, col);
        }
    if (hi >= 0) {
      dens_c0 = lo;
      ndens = hi - lo + 1;
    }
    if (ndens > 64) return set_error(h, FS_ERR_UNSUPPORTED, "Jacobian: more than 64 free density knots");
    const size_t na = static_cast<size_t>(h->n_atoms);
    if (static_cast<size_t>(h->atom_scratch_alloc) < na || !h->d_atom_scalars) {
      size_t dummy = 0;
      if (h->d_atom_scalars) cudaFree(h->d_atom_scalars);
      if (h->d_drho) cudaFree(h->d_drho);
      if (h->d_dgd) cudaFree(h->d_dgd);
      if (h->d_wsF) cudaFree(h->d_wsF);
      h->d_atom_scalars = h->d_drho = h->d_dgd = nullptr;
      h->d_wsF = nullptr;
      FS_TRY(grow(h, reinterpret_cast<T **>(&h->d_atom_scalars), 4 * na, dummy));
      dummy = 0;
      FS_TRY(grow(h, reinterpret_cast<T **>(&h->d_drho), 64 * na, dummy));
      dummy = 0;
      FS_TRY(grow(h, reinterpret_cast<T **>(&h->d_dgd), kWin * na, dummy));
      dummy = 0;
      FS_TRY(grow(h, &h->d_wsF, na, dummy));
      h->atom_scratch_alloc = static_cast<int64_t>(na);
    }
  }
  JacArgs<T> a;
  a.c = make_common<T>(h);
  a.seg_a = static_cast<const T4 *>(h->d_seg_a);
  a.seg_g = static_cast<const T *>(h->d_seg_g);
  a.seg_ws = h->d_seg_ws;
  a.w_e = w_e;
  a.w_s = w_s;
  a.M = M;
  a.cs = rowmajor ? 1 : ldj;
  a.rs = rowmajor ? ldj : 1;
  a.halves = 1;
  a.half_part = nullptr;
  a.D = D;
  a.F = h->d_F;
  a.jtr_part = h->d_jtr_part;
  a.dens_c0 = dens_c0;
  a.ndens = ndens;
  a.J = static_cast<T *>(h->d_J);
  {
    T *sc = static_cast<T *>(h->d_atom_scalars);
    const size_t na = static_cast<size_t>(h->n_atoms);
    a.gF = sc;
    a.cF = sc ? sc + na : nullptr;
    a.over = sc ? sc + 2 * na : nullptr;
  }
  a.drho = static_cast<T *>(h->d_drho);
  a.dgd = static_cast<T *>(h->d_dgd);
  a.wsF = h->d_wsF;
  a.run_a = h->d_run_a;
  a.run_b = h->d_run_b;
  a.run_cnt = h->d_run_cnt;
  a.runs = 0;
  if constexpr (std::is_same_v<T, float>) {
    RunGrid rg;
    a.runs = eam && h->runs_valid && pair_runs_grid(h, &rg) ? 1 : 0;
  }
  a.stage = 0;
  const size_t common = jac_common_smem<T>(a.c.n_tables, h->n_segs, h->n_cmap, h->max_natoms, max_images(h));
  if (eam) {
    const size_t sm1 = common + align16(2 * D * sizeof(double)) + atom_stage_smem<T>(h->max_natoms, ndens) + 64;
    if (sm1 > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "Jacobian: configuration too large");
    FS_CUDA(cudaFuncSetAttribute(jac_atoms_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sm1)));
    jac_atoms_kernel<T><<<h->n_cfg, 256, sm1, h->stream>>>(a);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  mark(h, 2);
  if (h->join_pending) { // the residual (side stream) must be done: F feeds Jᵀr here
    FS_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    h->join_pending = false;
  }
  // per-warp buffers + (optionally) the configuration's staged per-atom data;
  // prefer the most warps that fit with staging, else the most without
  auto k2_smem = [&](int wp) {
    return common + align16(static_cast<size_t>(wp) * (D + 1) * 4 * sizeof(T)) +
           align16(static_cast<size_t>(wp) * 3 * D * 2 * sizeof(T)) + align16(static_cast<size_t>(wp) * D * sizeof(T)) +
           align16(static_cast<size_t>(wp) * 32 * sizeof(PairRec<T>)) +
           align16(static_cast<size_t>(wp) * D * sizeof(double)) +
           align16(static_cast<size_t>(h->max_natoms + 1) * sizeof(int32_t)) + 112;
  };
  // staging levels (EAM): 2 = per-atom scalars + ∂ρ/∂y rows, 1 = scalars only
  const size_t stage_sz[3] = {0, eam ? atom_scalar_stage_smem<T>(h->max_natoms) : 0,
                              eam ? atom_scalar_stage_smem<T>(h->max_natoms) +
                                        align16(static_cast<size_t>(h->max_natoms) * (ndens + 1) * sizeof(T)) + 16
                                  : 0};
  const size_t cap = 227 * 1024;
  int warps = 0;
  size_t sm2 = 0;
  const int max_wp = kMaxK2Warps<T>;
  // the given warp count with the most staging that fits
  auto fit = [&](int wp) {
    for (int lv = eam ? 2 : 0; lv >= 0; --lv)
      if (k2_smem(wp) + stage_sz[lv] <= cap) {
        warps = wp;
        sm2 = k2_smem(wp) + stage_sz[lv];
        a.stage = lv;
        return true;
      }
    return false;
  };
  if (h->tuned_k2_warps > 0) fit(std::min(h->tuned_k2_warps, max_wp));
  if (eam) // untuned: the most warps with full staging, else the most warps
    for (int wp = max_wp; wp >= 4 && !warps; --wp)
      if (k2_smem(wp) + stage_sz[2] <= cap) fit(wp);
  for (int wp = max_wp; wp >= 1 && !warps; --wp) fit(wp);
  if (warps < 1) return set_error(h, FS_ERR_UNSUPPORTED, "Jacobian: configuration too large");
  auto k2 = eam ? (a.stage == 2   ? jac_forces_kernel<T, true, 2>
                   : a.stage == 1 ? jac_forces_kernel<T, true, 1>
                                  : jac_forces_kernel<T, true, 0>)
                : jac_forces_kernel<T, false, 0>;
  FS_CUDA(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm2)));
  // Two CTAs per configuration when that fills the SMs' waves clearly better
  // (e.g. 500 configurations on 148 SMs, one CTA each: 3.38 of 4 waves busy,
  // 84 %; 1000 half-size CTAs: 6.76 of 7, 97 %), and every CTA keeps atoms.
  {
    int per_sm = 0, nsm = 0;
    FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2, 32 * warps, sm2));
    FS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    const int64_t slots = static_cast<int64_t>(std::max(per_sm, 1)) * std::max(nsm, 1);
    auto fill = [&](int64_t ctas) { return static_cast<double>(ctas) / (((ctas + slots - 1) / slots) * slots); };
    int min_atoms = 1 << 30;
    for (const CfgDev &cd : h->cfg_host) min_atoms = std::min(min_atoms, cd.natoms);
    if (min_atoms >= 2 * warps && fill(2 * static_cast<int64_t>(h->n_cfg)) > fill(h->n_cfg) + 0.05) {
      const size_t need = static_cast<size_t>(h->n_cfg) * 2 * 8 * D;
      if (h->half_part_alloc < need || !h->d_half_part) {
        if (h->d_half_part) cudaFree(h->d_half_part);
        h->d_half_part = nullptr;
        FS_CUDA(cudaMalloc(&h->d_half_part, need * sizeof(double)));
        h->half_part_alloc = need;
      }
      a.halves = 2;
      a.half_part = h->d_half_part;
    }
  }
  k2<<<h->n_cfg * a.halves, 32 * warps, sm2, h->stream>>>(a, warps);
  FS_CUDA(cudaGetLastError());
  if (a.halves == 2) {
    auto comb = eam ? jac_halves_combine<T, true> : jac_halves_combine<T, false>;
    comb<<<h->n_cfg, 256, 0, h->stream>>>(a);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  jtr_reduce_kernel<<<(D + 127) / 128, 128, 0, h->stream>>>(h->d_jtr_part, h->n_cfg, D, h->d_Jtr);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  mark(h, 3);
  return FS_OK;
}


// Per-trial makima segments for the population kernel: block (table, trial)
// rebuilds the knot values from the trial vector (fixed knots from the model)
// and computes the slopes and power-basis coefficients with the same
// arithmetic as the single-model setup.
template <class T>
__global__ void pop_setup_kernel(const TableDesc *__restrict__ desc, const int *__restrict__ spl,
                                 const double *__restrict__ vals, const int32_t *__restrict__ cmap,
                                 const double *__restrict__ xs, int D, int n_segs,
                                 typename Vec4T<T>::type *__restrict__ pop_seg) {
  using T4 = typename Vec4T<T>::type;
  const TableDesc td = desc[spl[blockIdx.x]];
  const int k = blockIdx.y, n = td.n;
  __shared__ double y[512], s[512];
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int col = cmap[td.cmap0 + q];
    y[q] = col >= 0 ? xs[static_cast<int64_t>(k) * D + col] : vals[td.pv0 + q];
  }
  __syncthreads();
  const double h = td.h;
  auto sec = [&](int q) { return (y[q + 1] - y[q]) / h; };
  auto wgt = [](double u, double v) { return fabs(u - v) + fabs(u + v) / 2; };
  auto slope = [&](double p1, double p2, double p3, double p4) {
    const double w1 = wgt(p4, p3), w2 = wgt(p2, p1);
    const double r = (w1 * p2 + w2 * p3) / (w1 + w2);
    return (isnan(r) || w1 + w2 == 0.0) ? 0.0 : r;
  };
  if (n >= 4)
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
      double v;
      if (q == 0 || q == 1) {
        const double m0 = sec(0), m1 = sec(1);
        const double mm1 = 2.0 * m0 + -1.0 * m1;
        v = q == 0 ? slope(2.0 * mm1 + -1.0 * m0, mm1, m0, m1) : slope(mm1, m0, m1, sec(2));
      } else if (q >= n - 2) {
        const double mnm3 = sec(n - 3), mnm2 = sec(n - 2);
        const double mnm1 = 2.0 * mnm2 + -1.0 * mnm3;
        v = q == n - 2 ? slope(sec(n - 4), mnm3, mnm2, mnm1) : slope(mnm3, mnm2, mnm1, 2.0 * mnm1 + -1.0 * mnm2);
      } else {
        v = slope(sec(q - 2), sec(q - 1), sec(q), sec(q + 1));
      }
      s[q] = v;
    }
  __syncthreads();
  for (int e = threadIdx.x; e <= n; e += blockDim.x) {
    double a[4] = {0, 0, 0, 0};
    if (e == 0) {
      a[0] = y[0];
      a[1] = y[1] - y[0];
    } else if (e == n) {
      a[0] = y[n - 1];
      a[1] = y[n - 1] - y[n - 2];
    } else {
      const int i = e - 1;
      if (n < 4) {
        a[0] = y[i];
        a[1] = y[i + 1] - y[i];
      } else {
        const double s0 = s[i], s1 = s[i + 1];
        a[0] = y[i];
        a[1] = h * s0;
        a[2] = -3.0 * y[i] - 2.0 * h * s0 + 3.0 * y[i + 1] - h * s1;
        a[3] = 2.0 * y[i] + h * s0 - 2.0 * y[i + 1] + h * s1;
      }
    }
    T4 o;
    o.x = static_cast<T>(a[0]);
    o.y = static_cast<T>(a[1]);
    o.z = static_cast<T>(a[2]);
    o.w = static_cast<T>(a[3]);
    pop_seg[static_cast<int64_t>(k) * n_segs + td.seg0 + e] = o;
  }
}

__global__ void pop_reduce_kernel(const double *__restrict__ part, int n_cfg, int NP, double *__restrict__ obj) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NP) return;
  double s = 0.0;
  for (int c = 0; c < n_cfg; ++c) s += part[static_cast<int64_t>(k) * n_cfg + c];
  obj[k] = s;
}

template <class T, int LPA, bool EAM>
int launch_population_t(fs_gpu *h, double w_e, double w_s, const double *d_xs, int NP, double *d_obj) {
  using T4 = typename Vec4T<T>::type;
  ResArgs<T> a;
  a.c = make_common<T>(h);
  a.seg_a = nullptr;
  a.w_e = w_e;
  a.w_s = w_s;
  a.F = a.forces = a.energy = a.stress9 = a.limit = a.obj_part = nullptr;
  // layout: config order (n_cfg int32, fixed offset 0) | per-trial segments | per-(trial, config) Σ rows²
  const size_t ordb = (h->n_cfg * sizeof(int32_t) + 255) / 256 * 256;
  const size_t segb = (static_cast<size_t>(NP) * h->n_segs * sizeof(T4) + 255) / 256 * 256;
  const size_t partb = static_cast<size_t>(NP) * h->n_cfg * sizeof(double);
  const size_t need = ordb + segb + partb;
  if (static_cast<size_t>(h->pop_alloc) < need || !h->d_pop_seg_a) {
    if (h->d_pop_seg_a) cudaFree(h->d_pop_seg_a);
    h->d_pop_seg_a = nullptr;
    FS_CUDA(cudaMalloc(&h->d_pop_seg_a, need));
    h->pop_alloc = static_cast<int64_t>(need);
    // configurations in decreasing atom count (largest work items first)
    std::vector<int32_t> ord(h->n_cfg);
    for (int c = 0; c < h->n_cfg; ++c) ord[c] = c;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return h->natoms[x] > h->natoms[y]; });
    FS_CUDA(cudaMemcpy(h->d_pop_seg_a, ord.data(), h->n_cfg * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  const int32_t *order = static_cast<const int32_t *>(h->d_pop_seg_a);
  T4 *pop_seg = reinterpret_cast<T4 *>(static_cast<char *>(h->d_pop_seg_a) + ordb);
  double *part = reinterpret_cast<double *>(static_cast<char *>(h->d_pop_seg_a) + ordb + segb);
  std::vector<int> spl;
  for (int t = 0; t < static_cast<int>(h->desc.size()); ++t)
    if (h->desc[t].kind == FS_TABLE_SPLINE) spl.push_back(t);
  if (h->pop_spl_count != static_cast<int>(spl.size()) || !h->d_pop_spl) {
    if (h->d_pop_spl) cudaFree(h->d_pop_spl);
    FS_CUDA(cudaMalloc(&h->d_pop_spl, std::max<size_t>(spl.size(), 1) * sizeof(int)));
    FS_CUDA(cudaMemcpy(h->d_pop_spl, spl.data(), spl.size() * sizeof(int), cudaMemcpyHostToDevice));
    h->pop_spl_count = static_cast<int>(spl.size());
  }
  if (!spl.empty()) {
    dim3 g(static_cast<unsigned>(spl.size()), static_cast<unsigned>(NP));
    pop_setup_kernel<T><<<g, 32, 0, h->stream>>>(h->d_desc, h->d_pop_spl, h->d_vals, h->d_cmap, d_xs, h->D,
                                                 h->n_segs, pop_seg);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  if constexpr (std::is_same_v<T, float>) {
    // one lane per trial when the largest configuration fits in shared memory
    const int np_ = npair_of(h->ntypes);
    const int nseg_pd = EAM ? h->desc[np_ + h->ntypes].seg0 : h->n_segs;
    const size_t sml = pop_lanes_smem(a.c.n_tables, nseg_pd, h->max_natoms, max_images(h), EAM);
    if (sml <= 227 * 1024) {
      PopArgs pa;
      pa.c = a.c;
      pa.pop_seg = pop_seg;
      pa.NP = NP;
      pa.n_tiles = (NP + kPopLanes - 1) / kPopLanes;
      // about four waves of one CTA per SM (or the tuned number)
      const int waves = h->tuned_pop_waves > 0 ? h->tuned_pop_waves : 4;
      pa.n_chunks = std::max(1, std::min(h->n_cfg, (waves * 148 + pa.n_tiles - 1) / pa.n_tiles));
      pa.nseg_pd = nseg_pd;
      pa.max_atoms = h->max_natoms;
      pa.max_img = max_images(h);
      pa.order = order;
      pa.part = part;
      pa.w_e = w_e;
      pa.w_s = w_s;
      pa.run_a = h->d_run_a;
      pa.run_b = h->d_run_b;
      pa.run_r = h->d_run_r;
      pa.run_cnt = h->d_run_cnt;
      pa.runs = 0;
      const bool stress = w_s > 0.0;
      auto kl = stress ? pop_lanes_kernel<EAM, false, true> : pop_lanes_kernel<EAM, false, false>;
      if constexpr (EAM) {
        RunGrid rg;
        if (h->runs_valid && pair_runs_grid(h, &rg)) {
          kl = stress ? pop_lanes_kernel<EAM, true, true> : pop_lanes_kernel<EAM, true, false>;
          pa.runs = 1;
        }
      }
      FS_CUDA(cudaFuncSetAttribute(kl, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sml)));
      kl<<<static_cast<unsigned>(pa.n_chunks) * pa.n_tiles, kPopWarps * 32, sml, h->stream>>>(pa);
      FS_CUDA(cudaGetLastError());
      pop_reduce_kernel<<<(NP + 127) / 128, 128, 0, h->stream>>>(part, h->n_cfg, NP, d_obj);
      FS_CUDA(cudaGetLastError());
      h->launches += 2;
      return FS_OK;
    }
  }
  const int tile = std::max(1, std::min(16, NP));
  const int n_tiles = (NP + tile - 1) / tile;
  const size_t sm = residual_smem<T>(a.c.n_tables, h->n_segs, h->max_natoms, max_images(h));
  auto k = pop_eval_kernel<T, LPA, EAM>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<static_cast<unsigned>(h->n_cfg) * n_tiles, 256, sm, h->stream>>>(a, pop_seg, NP, tile, n_tiles, order, part);
  FS_CUDA(cudaGetLastError());
  pop_reduce_kernel<<<(NP + 127) / 128, 128, 0, h->stream>>>(part, h->n_cfg, NP, d_obj);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

template <class T, bool EAM> int launch_population_lpa(fs_gpu *h, double w_e, double w_s, const double *xs, int NP, double *obj) {
  switch (choose_lpa(h)) {
  case 4: return launch_population_t<T, 4, EAM>(h, w_e, w_s, xs, NP, obj);
  case 8: return launch_population_t<T, 8, EAM>(h, w_e, w_s, xs, NP, obj);
  case 16: return launch_population_t<T, 16, EAM>(h, w_e, w_s, xs, NP, obj);
  default: return launch_population_t<T, 32, EAM>(h, w_e, w_s, xs, NP, obj);
  }
}

// ---------------------------------------------------------------------------
// Population objective with caller-owned buffers and no allocation
// (fs_gpu_eval_population_noalloc).  The same kernels as the allocating
// path; its scratch — configuration order, spline-table list, per-trial
// segments and per-(trial, configuration) partial sums — lives in one
// fixed-size device array, g_noalloc_scratch below.

__global__ void iota_kernel(int32_t *__restrict__ v, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

struct NoAllocLayout {
  size_t ord, spl, seg, part, total;
};

template <class T> NoAllocLayout noalloc_layout(const fs_gpu *h, int NP) {
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  NoAllocLayout L;
  L.ord = 0;
  L.spl = L.ord + up(h->n_cfg * sizeof(int32_t));
  L.seg = L.spl + up(h->desc.size() * sizeof(int32_t));
  L.part = L.seg + up(static_cast<size_t>(NP) * h->n_segs * sizeof(typename Vec4T<T>::type));
  L.total = L.part + static_cast<size_t>(NP) * h->n_cfg * sizeof(double);
  return L;
}

// Launches of launch_population_t with every buffer taken from `scratch`.
template <class T, int LPA, bool EAM>
int launch_population_static(fs_gpu *h, double w_e, double w_s, const double *d_xs, int NP, double *d_obj,
                             unsigned char *scratch) {
  using T4 = typename Vec4T<T>::type;
  const NoAllocLayout L = noalloc_layout<T>(h, NP);
  int32_t *order = reinterpret_cast<int32_t *>(scratch + L.ord);
  int32_t *spl = reinterpret_cast<int32_t *>(scratch + L.spl);
  T4 *pop_seg = reinterpret_cast<T4 *>(scratch + L.seg);
  double *part = reinterpret_cast<double *>(scratch + L.part);
  const int n_tables = static_cast<int>(h->desc.size());
  // every table is a spline here, so the table list is 0..n_tables−1.  The
  // configurations go heaviest first, in the order the context already keeps
  // for its 3-body kernels (pairs + neighbour pairs per configuration, built
  // with the neighbour lists); the order only balances the work, since the
  // partial sums are indexed by configuration and added in a fixed order
  if (h->d_cfg_by_work) {
    FS_CUDA(cudaMemcpyAsync(order, h->d_cfg_by_work, h->n_cfg * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                            h->stream));
  } else {
    iota_kernel<<<(h->n_cfg + 255) / 256, 256, 0, h->stream>>>(order, h->n_cfg);
    ++h->launches;
  }
  iota_kernel<<<1, 256, 0, h->stream>>>(spl, n_tables);
  FS_CUDA(cudaGetLastError());
  dim3 g(static_cast<unsigned>(n_tables), static_cast<unsigned>(NP));
  pop_setup_kernel<T><<<g, 32, 0, h->stream>>>(h->d_desc, spl, h->d_vals, h->d_cmap, d_xs, h->D, h->n_segs, pop_seg);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  ResArgs<T> a;
  a.c = make_common<T>(h);
  a.seg_a = nullptr;
  a.w_e = w_e;
  a.w_s = w_s;
  a.F = a.forces = a.energy = a.stress9 = a.limit = a.obj_part = nullptr;
  if constexpr (std::is_same_v<T, float>) {
    const int np_ = npair_of(h->ntypes);
    const int nseg_pd = EAM ? h->desc[np_ + h->ntypes].seg0 : h->n_segs;
    const size_t sml = pop_lanes_smem(a.c.n_tables, nseg_pd, h->max_natoms, max_images(h), EAM);
    if (sml <= 227 * 1024) {
      PopArgs pa;
      pa.c = a.c;
      pa.pop_seg = pop_seg;
      pa.NP = NP;
      pa.n_tiles = (NP + kPopLanes - 1) / kPopLanes;
      // the allocating path's wave count (tuned by fs_gpu_autotune, else 4)
      const int waves = h->tuned_pop_waves > 0 ? h->tuned_pop_waves : 4;
      pa.n_chunks = std::max(1, std::min(h->n_cfg, (waves * 148 + pa.n_tiles - 1) / pa.n_tiles));
      pa.nseg_pd = nseg_pd;
      pa.max_atoms = h->max_natoms;
      pa.max_img = max_images(h);
      pa.order = order;
      pa.part = part;
      pa.w_e = w_e;
      pa.w_s = w_s;
      pa.run_a = h->d_run_a;
      pa.run_b = h->d_run_b;
      pa.run_r = h->d_run_r;
      pa.run_cnt = h->d_run_cnt;
      pa.runs = 0;
      const bool stress = w_s > 0.0;
      auto kl = stress ? pop_lanes_kernel<EAM, false, true> : pop_lanes_kernel<EAM, false, false>;
      if constexpr (EAM) {
        RunGrid rg;
        if (h->runs_valid && pair_runs_grid(h, &rg)) {
          kl = stress ? pop_lanes_kernel<EAM, true, true> : pop_lanes_kernel<EAM, true, false>;
          pa.runs = 1;
        }
      }
      FS_CUDA(cudaFuncSetAttribute(kl, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sml)));
      kl<<<static_cast<unsigned>(pa.n_chunks) * pa.n_tiles, kPopWarps * 32, sml, h->stream>>>(pa);
      FS_CUDA(cudaGetLastError());
      pop_reduce_kernel<<<(NP + 127) / 128, 128, 0, h->stream>>>(part, h->n_cfg, NP, d_obj);
      FS_CUDA(cudaGetLastError());
      h->launches += 2;
      return FS_OK;
    }
  }
  const int tile = std::max(1, std::min(16, NP));
  const int n_tiles = (NP + tile - 1) / tile;
  const size_t sm = residual_smem<T>(a.c.n_tables, h->n_segs, h->max_natoms, max_images(h));
  if (sm > 227 * 1024) return set_error(h, FS_ERR_UNSUPPORTED, "population: configuration too large for shared memory");
  auto k = pop_eval_kernel<T, LPA, EAM>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<static_cast<unsigned>(h->n_cfg) * n_tiles, 256, sm, h->stream>>>(a, pop_seg, NP, tile, n_tiles, order, part);
  FS_CUDA(cudaGetLastError());
  pop_reduce_kernel<<<(NP + 127) / 128, 128, 0, h->stream>>>(part, h->n_cfg, NP, d_obj);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

template <class T, bool EAM>
int launch_population_static_lpa(fs_gpu *h, double w_e, double w_s, const double *xs, int NP, double *obj,
                                 unsigned char *scratch) {
  switch (choose_lpa(h)) {
  case 4: return launch_population_static<T, 4, EAM>(h, w_e, w_s, xs, NP, obj, scratch);
  case 8: return launch_population_static<T, 8, EAM>(h, w_e, w_s, xs, NP, obj, scratch);
  case 16: return launch_population_static<T, 16, EAM>(h, w_e, w_s, xs, NP, obj, scratch);
  default: return launch_population_static<T, 32, EAM>(h, w_e, w_s, xs, NP, obj, scratch);
  }
}

} // namespace

int eval_residual(fs_gpu *h, double w_e, double w_s) {
  if (h->family != FS_FAMILY_EAM && h->family != FS_FAMILY_PAIR) {
    extern int eval_residual_other(fs_gpu * h, double w_e, double w_s);
    return eval_residual_other(h, w_e, w_s);
  }
  const bool eam = h->family == FS_FAMILY_EAM;
  if (h->precision == FS_PREC_FP64)
    return eam ? launch_residual_lpa<double, true>(h, w_e, w_s) : launch_residual_lpa<double, false>(h, w_e, w_s);
  return eam ? launch_residual_lpa<float, true>(h, w_e, w_s) : launch_residual_lpa<float, false>(h, w_e, w_s);
}

int eval_jacobian(fs_gpu *h, double w_e, double w_s) {
  if (h->family != FS_FAMILY_EAM && h->family != FS_FAMILY_PAIR) {
    extern int eval_jacobian_other(fs_gpu * h, double w_e, double w_s);
    return eval_jacobian_other(h, w_e, w_s);
  }
  // every table analytic: the reference's analytic chain rule
  // (forcesmith_functor.cpp:265-277); analytic and spline tables mixed: the
  // reference's central differences (fd_jacobian.hpp:37-49), FP64 contexts only
  // a free global parameter: central differences too, as the reference
  // (analytic_jacobian_available, param_jacobian.hpp:44-57)
  if (h->shared_cols) {
    extern int eval_jacobian_fd(fs_gpu * h, double w_e, double w_s);
    return eval_jacobian_fd(h, w_e, w_s);
  }
  int n_an = 0;
  for (const HostTable &t : h->tables) n_an += t.kind == FS_TABLE_ANALYTIC;
  if (n_an == static_cast<int>(h->tables.size())) {
    extern int eval_jacobian_analytic(fs_gpu * h, double w_e, double w_s);
    return eval_jacobian_analytic(h, w_e, w_s);
  }
  if (n_an > 0) {
    extern int eval_jacobian_fd(fs_gpu * h, double w_e, double w_s);
    return eval_jacobian_fd(h, w_e, w_s);
  }
  return h->precision == FS_PREC_FP64 ? launch_jacobian_t<double>(h, w_e, w_s)
                                      : launch_jacobian_t<float>(h, w_e, w_s);
}

} // namespace fsg

namespace fsg {
// FP64 segments of every spline table at the parameter vector d_x1 (D
// values on the device), whatever the working precision: the per-trial setup
// with one trial.  seg holds n_segs entries.
int spline_segments_fp64(fs_gpu *h, const double *d_x1, double4 *seg) {
  if (h->n_spl == 0) return FS_OK;
  pop_setup_kernel<double><<<dim3(static_cast<unsigned>(h->n_spl), 1), 32, 0, h->stream>>>(
      h->d_desc, h->d_spl, h->d_vals, h->d_cmap, d_x1, h->D, h->n_segs, seg);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  return FS_OK;
}

// Σ‖F(x_k)‖² for NP device-resident trial vectors (EAM / pair families).
int eval_population_device(fs_gpu *h, double w_e, double w_s, const double *d_xs, int NP, double *d_obj) {
  if (h->family != FS_FAMILY_EAM && h->family != FS_FAMILY_PAIR)
    return set_error(h, FS_ERR_UNSUPPORTED, "population kernel: EAM and pair families");
  for (const HostTable &t : h->tables)
    if (t.kind != FS_TABLE_SPLINE) return set_error(h, FS_ERR_UNSUPPORTED, "population kernel: spline tables");
  const bool eam = h->family == FS_FAMILY_EAM;
  if (h->precision == FS_PREC_FP64)
    return eam ? launch_population_lpa<double, true>(h, w_e, w_s, d_xs, NP, d_obj)
               : launch_population_lpa<double, false>(h, w_e, w_s, d_xs, NP, d_obj);
  return eam ? launch_population_lpa<float, true>(h, w_e, w_s, d_xs, NP, d_obj)
             : launch_population_lpa<float, false>(h, w_e, w_s, d_xs, NP, d_obj);
}
} // namespace fsg

// ---------------------------------------------------------------------------
// fs_gpu_eval_population_noalloc: the scratch array and its device address.

namespace fsg {

// 8 MiB of device memory in the library image: every GPU that loads the
// library holds it until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kMaxDevices] = {};

// The array's device address on h's device (looked up once per device, with
// that device current).  The host-side symbol itself is not a device address.
} // namespace

// Forget the cached address of `device` (fs_gpu_create calls this): a
// context created after a cudaDeviceReset looks the array up again in the
// device's new CUDA context instead of using the old address.
void noalloc_forget(int device) {
  if (device < 0 || device >= kMaxDevices) return;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  g_noalloc_addr[device] = nullptr;
}

namespace {
int noalloc_scratch(fs_gpu *h, unsigned char **out) {
  if (h->device < 0 || h->device >= kMaxDevices) return set_error(h, FS_ERR_ARG, "eval_population_noalloc: device ordinal");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[h->device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(h, FS_ERR_CUDA, std::string("eval_population_noalloc: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e));
    g_noalloc_addr[h->device] = p;
  }
  *out = static_cast<unsigned char *>(g_noalloc_addr[h->device]);
  return FS_OK;
}

bool on_device(const void *p, int device) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == device;
}
} // namespace
} // namespace fsg

extern "C" int fs_gpu_eval_population_noalloc(fs_gpu *h, double w_e, double w_s, const double *xs_dev, int32_t NP,
                                              double *obj_dev) {
  using namespace fsg;
  if (!h) return FS_ERR_ARG;
  if (!xs_dev || !obj_dev || NP < 1) return set_error(h, FS_ERR_ARG, "eval_population_noalloc: bad arguments");
  if (h->n_cfg == 0 || !h->have_model) return set_error(h, FS_ERR_STATE, "eval_population_noalloc: no configurations or model");
  if (h->rcut_built < 0 || model_max_cutoff(h) > h->rcut_built)
    return set_error(h, FS_ERR_STATE, "eval_population_noalloc: neighbour lists not built for the model; call fs_gpu_prepare");
  if (h->family != FS_FAMILY_EAM && h->family != FS_FAMILY_PAIR)
    return set_error(h, FS_ERR_UNSUPPORTED, "eval_population_noalloc: EAM and pair families");
  for (const HostTable &t : h->tables)
    if (t.kind != FS_TABLE_SPLINE) return set_error(h, FS_ERR_UNSUPPORTED, "eval_population_noalloc: spline tables");
  if (cudaSetDevice(h->device) != cudaSuccess) return set_error(h, FS_ERR_CUDA, "eval_population_noalloc: cudaSetDevice");
  if (!on_device(xs_dev, h->device) || !on_device(obj_dev, h->device))
    return set_error(h, FS_ERR_ARG, "eval_population_noalloc: xs and obj must be device memory of the context's GPU");
  const bool fp64 = h->precision == FS_PREC_FP64;
  const size_t need = fp64 ? noalloc_layout<double>(h, NP).total : noalloc_layout<float>(h, NP).total;
  if (need > kNoAllocScratchBytes) {
    // the largest NP whose layout fits, by bisection on the same layout the
    // check uses (0 when not even one trial fits)
    auto fits = [&](long long np) {
      return (fp64 ? noalloc_layout<double>(h, static_cast<int>(np)).total
                   : noalloc_layout<float>(h, static_cast<int>(np)).total) <= kNoAllocScratchBytes;
    };
    long long lo = 0, hi = NP; // fits(lo) or lo == 0; !fits(hi)
    while (hi - lo > 1) {
      const long long mid = lo + (hi - lo) / 2;
      (mid > 0 && fits(mid) ? lo : hi) = mid;
    }
    const long long max_np = lo;
    return set_error(h, FS_ERR_ARG,
                     "eval_population_noalloc: NP = " + std::to_string(NP) + " needs " + std::to_string(need) +
                         " bytes of scratch; the fixed maximum is " + std::to_string(kNoAllocScratchBytes) +
                         " bytes (NP <= " + std::to_string(max_np) + " for these configurations and model)");
  }
  unsigned char *scratch = nullptr;
  FS_TRY(noalloc_scratch(h, &scratch));
  const bool eam = h->family == FS_FAMILY_EAM;
  if (fp64)
    return eam ? launch_population_static_lpa<double, true>(h, w_e, w_s, xs_dev, NP, obj_dev, scratch)
               : launch_population_static_lpa<double, false>(h, w_e, w_s, xs_dev, NP, obj_dev, scratch);
  return eam ? launch_population_static_lpa<float, true>(h, w_e, w_s, xs_dev, NP, obj_dev, scratch)
             : launch_population_static_lpa<float, false>(h, w_e, w_s, xs_dev, NP, obj_dev, scratch);
}
