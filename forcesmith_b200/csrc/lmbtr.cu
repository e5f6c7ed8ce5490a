// LMBTR descriptors with a linear energy head per species, on the device.
//
//   LMBTR::get_descriptor (src/force/lmbtr.cpp:64-121): for a central atom i,
//   the neighbours with 1e-14 ≤ r < rcut (descriptor_neighbor,
//   include/forcesmith/force/ml_force.hpp:85-97); for each neighbour j a
//   Gaussian of width σ2 at r_ij with weight e^{−r_ij/ws} on the k2 grid of
//   j's species; for each neighbour pair j < k (list order) a Gaussian of
//   width σ3 at cos θ_jik, clamped to [−1, 1], with weight
//   e^{−(r_ij + r_ik + r_jk)/ws} on the k3 grid of the species pair.  Each
//   Gaussian is scaled by 1/(σ√(2π)) and added to the grid bins within 5σ of
//   its centre (broaden, lmbtr.cpp:31-55); then u/‖u‖ (normalize_l2).
//   LinearHead: E_i = w_{t_i}·D_i + b_{t_i}.
//
// Forces.  The reference has no analytic descriptor gradient (analytic_grads()
// is false, include/forcesmith/potentials/lmbtr.hpp:48) and forms ∂D/∂d_ij by
// central differences of the whole descriptor, h = 1e-4, one neighbour
// displacement component at a time (MLBase::descriptor_with_grad,
// ml_force.hpp:544-572).  Here the derivative of the same function is exact:
// each Gaussian's bin window is the one of the evaluation point, and the
// normalisation enters as ∂v/∂u = (I − v vᵀ)/‖u‖.  The two agree to the
// central difference's truncation error, except where a displacement of ±h
// moves a neighbour across rcut or a bin across a window edge (where the
// descriptor itself jumps by e^{−12.5} of a Gaussian's peak).
//
// Jacobian with respect to the head coefficients (exact: the model is linear
// in them): ∂E/∂w_s = Σ_i v_s(i), ∂E/∂b = atom count, and the force rows
// −∂v_s/∂x, formed per neighbour q of atom i as the dense 3 × S block
// ∂v/∂d_q = (P_q − v (v·P_q))/‖u‖ with P_q = ∂u/∂d_q.
//
// One CTA per configuration; each warp takes one central atom at a time.
// Its neighbours inside rcut are compacted (in list order) into the warp's
// shared-memory slice; u is accumulated there with the lanes over a
// Gaussian's bins, in the reference's term order; the force pass puts the
// lanes over neighbours (k2) and neighbour pairs (k3), each lane summing its
// Gaussian's bins against ∂E/∂u.
#include "jtr.cuh"
#include "kern_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fsg {
namespace {

constexpr int kLmMaxWarps = 16;

// exp: the hardware approximation in FP32, IEEE in FP64
__device__ __forceinline__ float lm_exp(float x) { return __expf(x); }
__device__ __forceinline__ double lm_exp(double x) { return exp(x); }

// One broadening grid: n bins from lo in steps of step; s2 = 2σ², inv =
// 1/(σ√(2π)), rad = 5σ/step (make_kernel, lmbtr.cpp:21-29).
template <class T> struct LmGrid {
  int n;
  T lo, step, is2, inv, rad;
  __device__ void init(const double *v) { // {n, min, max, sigma}
    n = static_cast<int>(v[0]);
    const double sig = v[3];
    const double st = n > 1 ? (v[2] - v[1]) / (n - 1) : 0.0;
    lo = static_cast<T>(v[1]);
    step = static_cast<T>(st);
    is2 = static_cast<T>(1.0 / (2.0 * sig * sig));
    inv = static_cast<T>(1.0 / (sig * sqrt(2.0 * 3.14159265358979323846)));
    rad = static_cast<T>(n > 1 ? 5.0 * sig / st : 0.0);
  }
  // bins [b0, b1] within 5σ of geom (b0 > b1: none); one bin on a 1-bin grid
  __device__ __forceinline__ void window(T geom, int &b0, int &b1) const {
    if (n <= 1) {
      b0 = b1 = 0;
      return;
    }
    const T center = (geom - lo) / step;
    b0 = max(0, static_cast<int>(ceil(center - rad)));
    b1 = min(n - 1, static_cast<int>(floor(center + rad)));
  }
  __device__ __forceinline__ T x(int b) const { return lo + static_cast<T>(b) * step; }
};

template <class T> struct LmArgs {
  Common c;
  const double *vals;
  double w_e, w_s;
  double *F, *forces, *energy, *stress9, *limit, *obj_part;
  const int32_t *order;
  T *J;
  int64_t ld;
  int D, smj, std_on;
  int kmax; // the longest neighbour list of the context
  double *desc; // MODE 2: per-atom descriptors [atom][S]
};

// Per-warp shared-memory slice: the compacted neighbours (d, r), their atoms
// and species, u (then v), ∂E/∂u, the staged neighbour pairs, and in the
// Jacobian mode P (3 × S), atom i's own rows (3 × S) and its stress rows
// (6 × S).
template <class T> struct LmWarp {
  T *nd;  // [kmax][4]: dx, dy, dz, r
  int *nj, *ns;
  T *u, *g;
  T *sc, *sa; // staged pairs: Gaussian centre and scale
  int *sb0, *sb1, *sblk;
  T *sU, *sV; // staged pairs (Jacobian): [32][3] each
  T *P, *Mi, *St;
};

template <class T> size_t lm_warp_bytes(int kmax, int S, bool jac) {
  size_t b = align16(static_cast<size_t>(kmax) * 4 * sizeof(T)) + 2 * align16(static_cast<size_t>(kmax) * sizeof(int)) +
             2 * align16(static_cast<size_t>(S) * sizeof(T)) + 2 * align16(32 * sizeof(T)) +
             3 * align16(32 * sizeof(int)) + 2 * align16(96 * sizeof(T));
  if (jac) b += align16(static_cast<size_t>(12) * S * sizeof(T));
  return b + 64;
}

template <class T> __device__ LmWarp<T> lm_take(Smem &S, int kmax, int Sz, bool jac) {
  LmWarp<T> w;
  w.nd = S.take<T>(static_cast<size_t>(kmax) * 4);
  w.nj = S.take<int>(kmax);
  w.ns = S.take<int>(kmax);
  w.u = S.take<T>(Sz);
  w.g = S.take<T>(Sz);
  w.sc = S.take<T>(32);
  w.sa = S.take<T>(32);
  w.sb0 = S.take<int>(32);
  w.sb1 = S.take<int>(32);
  w.sblk = S.take<int>(32);
  w.sU = S.take<T>(96);
  w.sV = S.take<T>(96);
  w.P = jac ? S.take<T>(static_cast<size_t>(12) * Sz) : nullptr;
  w.Mi = jac ? w.P + 3 * Sz : nullptr;
  w.St = jac ? w.P + 6 * Sz : nullptr;
  return w;
}

template <class T> __device__ __forceinline__ T warp_sum_t(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One CTA per configuration.  MODE 0: residual; 1: Jacobian rows; 2: each
// atom's descriptor into desc (for the standardization statistics).
// Standardized heads (the head sees (D − mean) ⊙ inv_std) act as heads of raw
// descriptors with w' = w ⊙ inv_std and b' = b − Σ w·inv_std·mean; in the
// Jacobian, w_k's column is inv_std_k times the raw one, and its energy row
// also gets −w_e·inv_std_k·mean_k per atom of the species.
template <class T, int MODE> __global__ void __launch_bounds__(kLmMaxWarps * 32) lmbtr_kernel(LmArgs<T> A) {
  constexpr bool JAC = MODE == 1, DESC = MODE == 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = A.order ? A.order[blockIdx.x] : blockIdx.x;
  const CfgDev &cd = A.c.cfg[c];
  const int N = cd.natoms, nt = A.c.ntypes;
  const int nimg = (2 * cd.sx + 1) * (2 * cd.sy + 1) * (2 * cd.sz + 1);
  const double *spec = A.vals + A.c.desc[0].pv0;
  const double rcut = spec[0];
  const T iws = static_cast<T>(1.0 / spec[1]);
  const bool normalize = spec[2] != 0.0;
  LmGrid<T> G2, G3;
  G2.init(spec + 3);
  G3.init(spec + 7);
  const int n2 = G2.n, n3 = G3.n, base3 = nt * n2;
  const int S = base3 + nt * (nt + 1) / 2 * n3;
  Smem sm(smem_raw);
  T *W = sm.take<T>(nt * (S + 1));        // heads: w[S], b per species
  int *col = sm.take<int>(nt * (S + 1));  // head value → J column (−1 fixed)
  double *wpos = sm.take<double>(3 * N);
  double *shift = sm.take<double>(3 * nimg);
  uint8_t *typ = sm.take<uint8_t>(N);
  T *Fs = sm.take<T>(3 * N);
  double *red = sm.take<double>(8 * 32);
  T *ivs = (JAC && A.std_on) ? sm.take<T>(nt * S) : nullptr;
  int *ntyp = (JAC && A.std_on) ? sm.take<int>(nt) : nullptr;
  T *Jb = (JAC && A.smj) ? sm.take<T>(static_cast<size_t>(3 * N) * A.D) : nullptr;
  double *E64 = JAC ? sm.take<double>(static_cast<size_t>(7) * A.D) : nullptr;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int k = 0; k < warp; ++k) lm_take<T>(sm, A.kmax, S, JAC);
  const LmWarp<T> wp = lm_take<T>(sm, A.kmax, S, JAC);
  if (E64)
    for (int k = threadIdx.x; k < 7 * A.D; k += blockDim.x) E64[k] = 0.0;
  if (Jb)
    for (int k = threadIdx.x; k < 3 * N * A.D; k += blockDim.x) Jb[k] = T(0);
  for (int k = threadIdx.x; k < nt * (S + 1); k += blockDim.x) {
    const int t = k / (S + 1), q = k % (S + 1);
    const TableDesc &td = A.c.desc[1 + t];
    const double *w = A.vals + td.pv0;
    double v = w[q];
    if (A.std_on) { // w ⊙ inv_std; b − Σ w·inv_std·mean
      const double *st = A.vals + A.c.desc[1 + nt + t].pv0; // mean[S], inv_std[S]
      if (q < S) {
        v = w[q] * st[S + q];
      } else {
        for (int u = 0; u < S; ++u) v -= w[u] * st[S + u] * st[u];
      }
    }
    W[k] = static_cast<T>(v);
    col[k] = A.c.cmap[td.cmap0 + q];
  }
  if (ivs) {
    for (int k = threadIdx.x; k < nt * S; k += blockDim.x)
      ivs[k] = static_cast<T>(A.vals[A.c.desc[1 + nt + k / S].pv0 + S + k % S]);
    for (int k = threadIdx.x; k < nt; k += blockDim.x) ntyp[k] = 0;
  }
  for (int k = threadIdx.x; k < 3 * N; k += blockDim.x) Fs[k] = T(0);
  stage_geometry(cd, A.c, wpos, shift, typ);
  __syncthreads();
  const int32_t *nbs = A.c.nb_start + cd.atom0;
  const int64_t rows_per_extra = 2 + (A.w_s > 0.0 ? 6 : 0);
  const int64_t row0 = 3 * static_cast<int64_t>(cd.atom0) + static_cast<int64_t>(c) * rows_per_extra;
  const int64_t rowE = row0 + 3 * N;
  const T sw = static_cast<T>(A.w_s / cd.volume);
  const int nrow = A.w_s > 0.0 ? 7 : 1;
  double e_acc = 0.0, sg[6] = {0, 0, 0, 0, 0, 0}; // xx, yy, zz, xy, xz, yz
  // J entry (local row r: 3N force rows, then E, 6 stress) in column cl
  auto jadd = [&](int cl, int r, T v) {
    if (Jb) atomicAdd(&Jb[r * A.D + cl], v);
    else atomicAdd(&A.J[static_cast<int64_t>(cl) * A.ld + row0 + r], v);
  };
  for (int i = warp; i < N; i += nw) {
    // ---- neighbours inside rcut, compacted in list order (the FP64 length
    // decides the gate in both precisions)
    int K = 0;
    for (int32_t pb = nbs[i]; pb < nbs[i + 1]; pb += 32) {
      const int32_t p = pb + lane;
      bool ok = false;
      T dx = T(0), dy = T(0), dz = T(0);
      int j = 0;
      double r64 = 0.0;
      if (p < nbs[i + 1]) {
        r64 = pair_vec_len<T>(wpos, shift, i, A.c.nb_pack[p], j, dx, dy, dz);
        ok = r64 >= 1e-14 && r64 < rcut;
      }
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const int q = K + __popc(m & ((1u << lane) - 1u));
        wp.nd[4 * q] = dx;
        wp.nd[4 * q + 1] = dy;
        wp.nd[4 * q + 2] = dz;
        wp.nd[4 * q + 3] = static_cast<T>(r64);
        wp.nj[q] = j;
        wp.ns[q] = typ[j];
      }
      K += __popc(m);
    }
    __syncwarp();
    // ---- u: the lanes over each Gaussian's bins, terms in the reference's order
    T *u = wp.u;
    for (int s = lane; s < S; s += 32) u[s] = T(0);
    __syncwarp();
    if (n2 > 0)
      for (int q = 0; q < K; ++q) {
        const T r = wp.nd[4 * q + 3];
        int b0, b1;
        G2.window(r, b0, b1);
        const T a = G2.inv * lm_exp(-r * iws);
        T *blk = u + wp.ns[q] * n2;
        for (int b = b0 + lane; b <= b1; b += 32) {
          const T dx = G2.x(b) - r;
          blk[b] += a * lm_exp(-dx * dx * G2.is2);
        }
        __syncwarp();
      }
    const int npr = K * (K - 1) / 2;
    if (n3 > 0)
      for (int pb = 0; pb < npr; pb += 32) {
        const int p = pb + lane;
        if (p < npr) { // stage the pair's centre, scale, window and block
          int uu = p, a0 = 0;
          pair_row(K, uu, a0);
          const T *dj = wp.nd + 4 * a0, *dk = wp.nd + 4 * (a0 + 1 + uu);
          T cth = (dj[0] * dk[0] + dj[1] * dk[1] + dj[2] * dk[2]) / (dj[3] * dk[3]);
          cth = cth > T(1) ? T(1) : (cth < T(-1) ? T(-1) : cth);
          const T ex = dk[0] - dj[0], ey = dk[1] - dj[1], ez = dk[2] - dj[2];
          const T rjk = sqrt(ex * ex + ey * ey + ez * ez);
          int b0, b1;
          G3.window(cth, b0, b1);
          wp.sc[lane] = cth;
          wp.sa[lane] = G3.inv * lm_exp(-(dj[3] + dk[3] + rjk) * iws);
          wp.sb0[lane] = b0;
          wp.sb1[lane] = b1;
          wp.sblk[lane] = base3 + pair_ord(wp.ns[a0], wp.ns[a0 + 1 + uu], nt) * n3;
        }
        __syncwarp();
        const int cnt = min(32, npr - pb);
        for (int t = 0; t < cnt; ++t) {
          const T cc = wp.sc[t], a = wp.sa[t];
          T *blk = u + wp.sblk[t];
          for (int b = wp.sb0[t] + lane; b <= wp.sb1[t]; b += 32) {
            const T dx = G3.x(b) - cc;
            blk[b] += a * lm_exp(-dx * dx * G3.is2);
          }
          __syncwarp();
        }
      }
    // ---- normalisation (normalize_l2, lmbtr.cpp:57-62) and the energy
    T ss = T(0);
    for (int s = lane; s < S; s += 32) ss += u[s] * u[s];
    ss = warp_sum_t(ss);
    const T nu = sqrt(ss);
    const bool nz = normalize && nu > T(0) && static_cast<double>(nu) > 1e-300;
    const T inv_nu = nz ? T(1) / nu : T(1);
    const int ti = typ[i];
    const T *w_ = W + ti * (S + 1);
    T ev = T(0);
    for (int s = lane; s < S; s += 32) {
      const T v = nz ? u[s] / nu : u[s];
      u[s] = v;
      ev += w_[s] * v;
    }
    ev = warp_sum_t(ev);
    __syncwarp();
    if constexpr (DESC) {
      for (int s = lane; s < S; s += 32)
        A.desc[(static_cast<int64_t>(cd.atom0) + i) * S + s] = static_cast<double>(u[s]);
      continue;
    }
    if constexpr (JAC) {
      // ---- Jacobian: energy row Σ_i v; per neighbour q the block
      // ∂v/∂d_q = (P_q − v (v·P_q))/‖u‖, −block on q's rows, +block summed
      // on i's rows, −sw d_q ⊗ block on the stress rows
      const T *iv = ivs ? ivs + ti * S : nullptr;
      const int *cl_ = col + ti * (S + 1);
      T *P = wp.P, *Mi = wp.Mi, *St = wp.St;
      for (int s = lane; s < S; s += 32) {
        const int cc = cl_[s];
        if (cc >= 0) atomicAdd(&E64[cc], A.w_e * static_cast<double>(iv ? u[s] * iv[s] : u[s]));
#pragma unroll
        for (int x = 0; x < 3; ++x) Mi[x * S + s] = T(0);
#pragma unroll
        for (int v = 0; v < 6; ++v) St[v * S + s] = T(0);
      }
      for (int q = 0; q < K; ++q) {
        const T *dq = wp.nd + 4 * q;
        const T rq = dq[3], irq = T(1) / rq;
        const T hq[3] = {dq[0] * irq, dq[1] * irq, dq[2] * irq};
        for (int s = lane; s < 3 * S; s += 32) P[s] = T(0);
        __syncwarp();
        if (n2 > 0) { // q's k2 Gaussian: ∂/∂d_q = (∂/∂r) d̂_q
          int b0, b1;
          G2.window(rq, b0, b1);
          const T a = G2.inv * lm_exp(-rq * iws);
          const int blk = wp.ns[q] * n2;
          for (int b = b0 + lane; b <= b1; b += 32) {
            const T dx = G2.x(b) - rq;
            const T t = a * lm_exp(-dx * dx * G2.is2) * (T(2) * G2.is2 * dx - iws);
            P[blk + b] += t * hq[0];
            P[S + blk + b] += t * hq[1];
            P[2 * S + blk + b] += t * hq[2];
          }
          __syncwarp();
        }
        if (n3 > 0)
          for (int kb = 0; kb < K; kb += 32) { // the k3 Gaussians of the pairs (q, k), k ≠ q
            const int k = kb + lane;
            if (k < K) {
              if (k == q) {
                wp.sb0[lane] = 1;
                wp.sb1[lane] = 0;
              } else {
                const T *dk = wp.nd + 4 * k;
                const T rk = dk[3];
                const T raw = (dq[0] * dk[0] + dq[1] * dk[1] + dq[2] * dk[2]) / (rq * rk);
                const bool clamped = raw > T(1) || raw < T(-1);
                const T cth = raw > T(1) ? T(1) : (raw < T(-1) ? T(-1) : raw);
                const T e[3] = {dk[0] - dq[0], dk[1] - dq[1], dk[2] - dq[2]};
                const T rqk = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
                const T irqk = rqk > T(1e-14) ? T(1) / rqk : T(0);
                int b0, b1;
                G3.window(cth, b0, b1);
                wp.sc[lane] = cth;
                wp.sa[lane] = G3.inv * lm_exp(-(rq + rk + rqk) * iws);
                wp.sb0[lane] = b0;
                wp.sb1[lane] = b1;
                wp.sblk[lane] = base3 + pair_ord(wp.ns[q], wp.ns[k], nt) * n3;
                const T irk = T(1) / rk;
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                  // ∂(r_q + r_k + r_qk)/∂d_q and ∂cos θ/∂d_q
                  wp.sU[3 * lane + x] = -iws * (hq[x] - e[x] * irqk);
                  wp.sV[3 * lane + x] = clamped ? T(0) : (dk[x] * irk - cth * hq[x]) * irq;
                }
              }
            }
            __syncwarp();
            const int cnt = min(32, K - kb);
            for (int t = 0; t < cnt; ++t) {
              const int b0 = wp.sb0[t], b1 = wp.sb1[t];
              if (b0 > b1) continue;
              const T cc = wp.sc[t], a = wp.sa[t];
              const int blk = wp.sblk[t];
              const T U0 = wp.sU[3 * t], U1 = wp.sU[3 * t + 1], U2 = wp.sU[3 * t + 2];
              const T V0 = wp.sV[3 * t], V1 = wp.sV[3 * t + 1], V2 = wp.sV[3 * t + 2];
              for (int b = b0 + lane; b <= b1; b += 32) {
                const T dx = G3.x(b) - cc;
                const T base = a * lm_exp(-dx * dx * G3.is2), bv = T(2) * G3.is2 * dx;
                P[blk + b] += base * (U0 + bv * V0);
                P[S + blk + b] += base * (U1 + bv * V1);
                P[2 * S + blk + b] += base * (U2 + bv * V2);
              }
              __syncwarp();
            }
            __syncwarp();
          }
        T vP0 = T(0), vP1 = T(0), vP2 = T(0);
        if (nz) {
          for (int s = lane; s < S; s += 32) {
            vP0 += u[s] * P[s];
            vP1 += u[s] * P[S + s];
            vP2 += u[s] * P[2 * S + s];
          }
          vP0 = warp_sum_t(vP0);
          vP1 = warp_sum_t(vP1);
          vP2 = warp_sum_t(vP2);
        }
        const int jq = wp.nj[q];
        for (int s = lane; s < S; s += 32) {
          const int cc = cl_[s];
          if (cc < 0) continue;
          const T sv = iv ? iv[s] : T(1);
          T m[3];
          m[0] = (nz ? (P[s] - u[s] * vP0) * inv_nu : P[s]) * sv;
          m[1] = (nz ? (P[S + s] - u[s] * vP1) * inv_nu : P[S + s]) * sv;
          m[2] = (nz ? (P[2 * S + s] - u[s] * vP2) * inv_nu : P[2 * S + s]) * sv;
#pragma unroll
          for (int x = 0; x < 3; ++x) {
            jadd(cc, 3 * jq + x, -m[x]);
            Mi[x * S + s] += m[x];
          }
          St[s] -= sw * dq[0] * m[0];
          St[S + s] -= sw * dq[1] * m[1];
          St[2 * S + s] -= sw * dq[2] * m[2];
          St[3 * S + s] -= sw * dq[0] * m[1];
          St[4 * S + s] -= sw * dq[0] * m[2];
          St[5 * S + s] -= sw * dq[1] * m[2];
        }
        __syncwarp();
      }
      for (int s = lane; s < S; s += 32) {
        const int cc = cl_[s];
        if (cc < 0) continue;
#pragma unroll
        for (int x = 0; x < 3; ++x) jadd(cc, 3 * i + x, Mi[x * S + s]);
        for (int v = 1; v < nrow; ++v) atomicAdd(&E64[v * A.D + cc], static_cast<double>(St[(v - 1) * S + s]));
      }
      __syncwarp();
      continue;
    }
    // ---- residual: ∂E/∂u = (w − (w·v) v)/‖u‖
    if (lane == 0) e_acc += static_cast<double>(ev) + static_cast<double>(w_[S]);
    T *g = wp.g;
    for (int s = lane; s < S; s += 32) g[s] = nz ? (w_[s] - ev * u[s]) * inv_nu : w_[s];
    __syncwarp();
    T fi[3] = {T(0), T(0), T(0)};
    // a term's ∂E/∂d for neighbour q: +f on i, −f on q's atom, σ −= d ⊗ f
    auto put = [&](const T *d, int j, const T (&f)[3]) {
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        fi[x] += f[x];
        atomicAdd(&Fs[3 * j + x], -f[x]);
      }
      sg[0] -= static_cast<double>(d[0] * f[0]);
      sg[1] -= static_cast<double>(d[1] * f[1]);
      sg[2] -= static_cast<double>(d[2] * f[2]);
      sg[3] -= static_cast<double>(d[0] * f[1]);
      sg[4] -= static_cast<double>(d[0] * f[2]);
      sg[5] -= static_cast<double>(d[1] * f[2]);
    };
    if (n2 > 0)
      for (int q = lane; q < K; q += 32) { // a lane per neighbour
        const T *d = wp.nd + 4 * q;
        const T r = d[3];
        int b0, b1;
        G2.window(r, b0, b1);
        if (b0 > b1) continue;
        const T *gb = g + wp.ns[q] * n2;
        T sA = T(0), sB = T(0);
        for (int b = b0; b <= b1; ++b) {
          const T dx = G2.x(b) - r;
          const T gg = gb[b] * lm_exp(-dx * dx * G2.is2);
          sA += gg;
          sB += gg * dx;
        }
        const T a = G2.inv * lm_exp(-r * iws);
        const T s_ = a * (T(2) * G2.is2 * sB - iws * sA) / r;
        const T f[3] = {s_ * d[0], s_ * d[1], s_ * d[2]};
        put(d, wp.nj[q], f);
      }
    if (n3 > 0)
      for (int p = lane; p < npr; p += 32) { // a lane per neighbour pair
        int uu = p, a0 = 0;
        pair_row(K, uu, a0);
        const int jq = a0, kq = a0 + 1 + uu;
        const T *dj = wp.nd + 4 * jq, *dk = wp.nd + 4 * kq;
        const T rj = dj[3], rk = dk[3];
        const T raw = (dj[0] * dk[0] + dj[1] * dk[1] + dj[2] * dk[2]) / (rj * rk);
        const bool clamped = raw > T(1) || raw < T(-1);
        const T cth = raw > T(1) ? T(1) : (raw < T(-1) ? T(-1) : raw);
        int b0, b1;
        G3.window(cth, b0, b1);
        if (b0 > b1) continue;
        const T e[3] = {dk[0] - dj[0], dk[1] - dj[1], dk[2] - dj[2]};
        const T rjk = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        const T *gb = g + base3 + pair_ord(wp.ns[jq], wp.ns[kq], nt) * n3;
        T sA = T(0), sB = T(0);
        for (int b = b0; b <= b1; ++b) {
          const T dx = G3.x(b) - cth;
          const T gg = gb[b] * lm_exp(-dx * dx * G3.is2);
          sA += gg;
          sB += gg * dx;
        }
        const T a = G3.inv * lm_exp(-(rj + rk + rjk) * iws);
        const T cA = -a * iws * sA;                                 // ∂/∂(r_j + r_k + r_jk)
        const T cB = clamped ? T(0) : a * T(2) * G3.is2 * sB;     // ∂/∂cos θ
        const T irjk = rjk > T(1e-14) ? T(1) / rjk : T(0), irj = T(1) / rj, irk = T(1) / rk;
        T Gj[3], Gk[3];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
          const T hj = dj[x] * irj, hk = dk[x] * irk, ex = e[x] * irjk;
          Gj[x] = cA * (hj - ex) + cB * (hk - cth * hj) * irj;
          Gk[x] = cA * (hk + ex) + cB * (hj - cth * hk) * irk;
        }
        put(dj, wp.nj[jq], Gj);
        put(dk, wp.nj[kq], Gk);
      }
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      const T t = warp_sum_t(fi[x]);
      if (lane == 0) atomicAdd(&Fs[3 * i + x], t);
    }
    __syncwarp();
  }
  if constexpr (DESC) return;
  if constexpr (JAC) {
    // biases: one per atom
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const int ti = typ[i];
      const int cb = col[ti * (S + 1) + S];
      if (cb >= 0) atomicAdd(&E64[cb], A.w_e);
      if (ntyp) atomicAdd(&ntyp[ti], 1);
    }
    __syncthreads();
    if (ivs) // standardized: ∂E/∂w_k also holds −inv_std_k·mean_k per atom of the species
      for (int q = threadIdx.x; q < nt * S; q += blockDim.x) {
        const int t = q / S, kk = q % S;
        const int ck = col[t * (S + 1) + kk];
        if (ck < 0 || ntyp[t] == 0) continue;
        const double mu = A.vals[A.c.desc[1 + nt + t].pv0 + kk];
        atomicAdd(&E64[ck], -A.w_e * static_cast<double>(ivs[q]) * mu * ntyp[t]);
      }
    __syncthreads();
    for (int q = threadIdx.x; q < nrow * A.D; q += blockDim.x) {
      const int m = q / A.D, cl = q % A.D;
      A.J[static_cast<int64_t>(cl) * A.ld + rowE + m] = static_cast<T>(E64[q]);
    }
    if (!Jb) return;
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
    const double E = sums[0], ivol = 1.0 / cd.volume;
    double st[6];
    for (int a = 0; a < 6; ++a) st[a] = sums[1 + a] * ivol;
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
    if (A.stress9) { // symmetric virial: upper triangle mirrored
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

__global__ void lm_sum_parts(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double r[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += part[k];
  s = block_sum(s, r);
  if (threadIdx.x == 0) *out = s;
}

int lm_size(const fs_gpu *h) {
  const double *v = h->tables[0].v.data();
  const int nt = h->ntypes;
  return nt * static_cast<int>(v[3]) + nt * (nt + 1) / 2 * static_cast<int>(v[7]);
}

// The longest neighbour list (an upper bound on the neighbours inside rcut).
// The neighbour build records it; this recount from the list offsets (a
// synchronising copy) is only a fallback for lists built without it.
int lm_kmax(fs_gpu *h) {
  if (h->max_list >= 0) return FS_OK;
  std::vector<int32_t> st(static_cast<size_t>(h->n_atoms) + 1);
  FS_CUDA(cudaMemcpyAsync(st.data(), h->d_nb_start, st.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  int m = 0;
  for (int64_t a = 0; a < h->n_atoms; ++a) m = std::max(m, st[a + 1] - st[a]);
  h->max_list = m;
  return FS_OK;
}

// mode 0: residual; 1: Jacobian rows (+ Jᵀr); 2: descriptors into desc
template <class T> int launch_lmbtr(fs_gpu *h, double w_e, double w_s, int mode, double *desc = nullptr) {
  const bool jac = mode == 1;
  FS_TRY(lm_kmax(h));
  LmArgs<T> a;
  a.c = make_common<T>(h);
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
  a.kmax = std::max(1, h->max_list);
  a.desc = desc;
  const int S = lm_size(h), nt = h->ntypes, N = h->max_natoms, D = h->D;
  const size_t cta = align16(nt * (S + 1) * sizeof(T)) + align16(nt * (S + 1) * sizeof(int)) +
                     align16(3 * N * sizeof(double)) + align16(3 * max_images(h) * sizeof(double)) + align16(N) +
                     align16(3 * N * sizeof(T)) + align16(8 * 32 * sizeof(double)) + align16(nt * S * sizeof(T)) +
                     align16(nt * sizeof(int)) + (jac ? align16(static_cast<size_t>(7) * D * sizeof(double)) : 0) +
                     64;
  const size_t per_warp = lm_warp_bytes<T>(a.kmax, S, jac);
  constexpr size_t kBudget = 227 * 1024;
  if (cta + per_warp > kBudget)
    return set_error(h, FS_ERR_UNSUPPORTED,
                     "LMBTR: " + std::to_string(cta + per_warp) + " bytes of shared memory for S = " +
                         std::to_string(S) + ", " + std::to_string(a.kmax) + " neighbours and " + std::to_string(N) +
                         " atoms in the largest configuration (the limit is 232448)");
  size_t sm = cta;
  int nw = static_cast<int>(std::min<size_t>(kLmMaxWarps, (kBudget - cta) / per_warp));
  const int64_t M = rows_of(h, w_s);
  if (jac) {
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
    // the configuration's force rows in shared memory when four warps still fit
    const size_t jb = align16(static_cast<size_t>(3 * N) * D * sizeof(T));
    if (D > 0 && cta + jb + 4 * per_warp <= kBudget) {
      a.smj = 1;
      sm += jb;
      nw = static_cast<int>(std::min<size_t>(kLmMaxWarps, (kBudget - sm) / per_warp));
    }
  }
  sm += nw * per_warp;
  auto k = mode == 1 ? lmbtr_kernel<T, 1> : mode == 2 ? lmbtr_kernel<T, 2> : lmbtr_kernel<T, 0>;
  FS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)));
  k<<<h->n_cfg, nw * 32, sm, h->stream>>>(a);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  if (mode == 2) return FS_OK;
  if (jac) {
    if (D > 0) FS_TRY(launch_jtr<T>(h, static_cast<const T *>(h->d_J), h->ldj, M, D, h->d_F, h->d_Jtr));
  } else {
    lm_sum_parts<<<1, 1024, 0, h->stream>>>(h->d_obj_part, h->n_cfg, h->d_obj);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  return FS_OK;
}

} // namespace

int eval_residual_lmbtr(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_lmbtr<double>(h, w_e, w_s, 0) : launch_lmbtr<float>(h, w_e, w_s, 0);
}
int eval_jacobian_lmbtr(fs_gpu *h, double w_e, double w_s) {
  return h->precision == FS_PREC_FP64 ? launch_lmbtr<double>(h, w_e, w_s, 1) : launch_lmbtr<float>(h, w_e, w_s, 1);
}
// every atom's descriptor, [atom][S], into desc (zeroed by the caller)
int lmbtr_descriptors(fs_gpu *h, double *desc) {
  return h->precision == FS_PREC_FP64 ? launch_lmbtr<double>(h, 1.0, 0.0, 2, desc)
                                      : launch_lmbtr<float>(h, 1.0, 0.0, 2, desc);
}

} // namespace fsg
