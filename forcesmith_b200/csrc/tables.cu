// Model tables on the device: the parameter-vector layout (table order, free
// values only — force_calculator_concept.hpp:171-208) and, for every makima
// spline, the per-segment power-basis coefficients and knot derivatives
// rebuilt in FP64 after each parameter scatter (the reference's
// scatter_params → recompute_slopes_, src/potentials/spline.cpp:43-103,196-203).
#include "internal.cuh"

#include <algorithm>
#include <cmath>

namespace fsg {

double model_max_cutoff(const fs_gpu *h) {
  // max span end over RADIAL tables (force_calculator_concept.hpp:210-221);
  // SW: max(a1, a2) (stiweb_force.cpp:234-239)
  const int nt = h->ntypes, np = npair_of(nt);
  double m = 0.0;
  if (h->family == FS_FAMILY_SW) {
    for (int p = 0; p < np; ++p) m = std::max(m, std::max(h->tables[p].v[5], h->tables[p].v[7]));
    return m;
  }
  if (h->family == FS_FAMILY_ACSF) return h->tables[0].v[0]; // descriptor_cutoff (acsf.hpp:73)
  if (h->family == FS_FAMILY_LMBTR) return h->tables[0].v[0]; // descriptor_cutoff (lmbtr.hpp:47)
  if (h->family == FS_FAMILY_TERSOFF) { // max S over pair slots (tersoff_force.cpp:259-265)
    for (int p = 0; p < np; ++p) m = std::max(m, h->tables[p].v[10]);
    return m;
  }
  for (int t = 0; t < static_cast<int>(h->desc.size()); ++t) {
    const bool emb = (h->family == FS_FAMILY_EAM || h->family == FS_FAMILY_ADP) && t >= np + nt &&
                     t < np + 2 * nt;
    const bool ang = h->family == FS_FAMILY_ANGULAR && t >= 2 * np; // cos θ tables are not radial
    if (!emb && !ang) m = std::max(m, h->desc[t].xmax);
  }
  return m;
}

namespace {

template <class X> int realloc_dev(fs_gpu *h, X **p, size_t n) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (n == 0) n = 1;
  if (cudaMalloc(reinterpret_cast<void **>(p), n * sizeof(X)) != cudaSuccess)
    return set_error(h, FS_ERR_NOMEM, "cudaMalloc (tables)");
  return FS_OK;
}

// One makima weight |u − v| + |u + v|/2 and the sign of a difference, with
// sign(0) = 0 (the central-difference limit at a kink).
__device__ __forceinline__ double mk_w(double u, double v) { return fabs(u - v) + fabs(u + v) / 2; }
__device__ __forceinline__ double sgn(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); }

// A linear combination of secants: value and gradient over the knot window
// [k-3, k+5) of the slope being built.
struct Lin {
  double v;
  double g[8];
};

__device__ void lin_sec(Lin &p, const double *y, double x0, double h, int q, int base) {
  const double ih = 1.0 / h;
  p.v = (y[q + 1] - y[q]) / h;
  for (int k = 0; k < 8; ++k) p.g[k] = 0.0;
  p.g[q - base] -= ih;
  p.g[q + 1 - base] += ih;
  (void)x0;
}
__device__ void lin_comb(Lin &o, double a, const Lin &p, double b, const Lin &q) {
  o.v = a * p.v + b * q.v;
  for (int k = 0; k < 8; ++k) o.g[k] = a * p.g[k] + b * q.g[k];
}

// s = (w1·p2 + w2·p3)/(w1 + w2), w1 = W(p4, p3), w2 = W(p2, p1): the makima
// slope of spline.cpp:58-101, with its gradient over the window.
__device__ double slope_and_grad(const Lin &p1, const Lin &p2, const Lin &p3, const Lin &p4, double *g) {
  const double w1 = mk_w(p4.v, p3.v), w2 = mk_w(p2.v, p1.v);
  const double W = w1 + w2;
  double s = (w1 * p2.v + w2 * p3.v) / W;
  for (int k = 0; k < 8; ++k) g[k] = 0.0;
  if (isnan(s) || W == 0.0) return 0.0;
  const double ds_dw1 = (p2.v - s) / W, ds_dw2 = (p3.v - s) / W;
  const double c1 = ds_dw2 * (-sgn(p2.v - p1.v) + 0.5 * sgn(p2.v + p1.v));
  const double c2 = w1 / W + ds_dw2 * (sgn(p2.v - p1.v) + 0.5 * sgn(p2.v + p1.v));
  const double c3 = w2 / W + ds_dw1 * (-sgn(p4.v - p3.v) + 0.5 * sgn(p4.v + p3.v));
  const double c4 = ds_dw1 * (sgn(p4.v - p3.v) + 0.5 * sgn(p4.v + p3.v));
  for (int k = 0; k < 8; ++k) g[k] = c1 * p1.g[k] + c2 * p2.g[k] + c3 * p3.g[k] + c4 * p4.g[k];
  return s;
}

constexpr int kMaxKnotsSmem = 512;

// One block per spline table.  smem: y, s, dS (5 per knot).
template <class T>
__global__ void spline_setup_kernel(const TableDesc *__restrict__ desc, const int *__restrict__ spl,
                                    const double *__restrict__ vals, T *__restrict__ seg_a,
                                    T *__restrict__ seg_g, int32_t *__restrict__ seg_ws) {
  const TableDesc td = desc[spl[blockIdx.x]];
  const int n = td.n;
  __shared__ double y[kMaxKnotsSmem];
  __shared__ double s[kMaxKnotsSmem];
  __shared__ double dS[kMaxKnotsSmem][5];
  for (int k = threadIdx.x; k < n; k += blockDim.x) y[k] = vals[td.pv0 + k];
  __syncthreads();
  const double h = td.h;
  const bool cubic = n >= 4;
  if (cubic) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int base = k - 3;
      Lin p1, p2, p3, p4;
      if (k == 0 || k == 1 || k >= n - 2) {
        Lin m0, m1, m2, a, b;
        if (k <= 1) {
          lin_sec(m0, y, td.x0, h, 0, base);
          lin_sec(m1, y, td.x0, h, 1, base);
          lin_comb(a, 2.0, m0, -1.0, m1); // mm1 = 2 m0 − m1
          if (k == 0) {
            lin_comb(b, 2.0, a, -1.0, m0); // mm2 = 2 mm1 − m0
            p1 = b; p2 = a; p3 = m0; p4 = m1;
          } else {
            lin_sec(m2, y, td.x0, h, 2, base);
            p1 = a; p2 = m0; p3 = m1; p4 = m2;
          }
        } else {
          Lin mnm4, mnm3, mnm2, mnm1, mn;
          lin_sec(mnm3, y, td.x0, h, n - 3, base);
          lin_sec(mnm2, y, td.x0, h, n - 2, base);
          lin_comb(mnm1, 2.0, mnm2, -1.0, mnm3);
          if (k == n - 2) {
            lin_sec(mnm4, y, td.x0, h, n - 4, base);
            p1 = mnm4; p2 = mnm3; p3 = mnm2; p4 = mnm1;
          } else {
            lin_comb(mn, 2.0, mnm1, -1.0, mnm2);
            p1 = mnm3; p2 = mnm2; p3 = mnm1; p4 = mn;
          }
        }
      } else {
        lin_sec(p1, y, td.x0, h, k - 2, base);
        lin_sec(p2, y, td.x0, h, k - 1, base);
        lin_sec(p3, y, td.x0, h, k, base);
        lin_sec(p4, y, td.x0, h, k + 1, base);
      }
      double g[8];
      s[k] = slope_and_grad(p1, p2, p3, p4, g);
      // compress to the 5-knot window starting at clamp(k-2, 0, n-5)
      const int wsk = max(0, min(k - 2, n - 5));
      for (int q = 0; q < 5; ++q) {
        const int knot = wsk + q;
        const int gi = knot - base;
        dS[k][q] = (knot < n && gi >= 0 && gi < 8) ? g[gi] : 0.0;
      }
    }
  }
  __syncthreads();
  const int W = n < kWin ? n : kWin;
  for (int e = threadIdx.x; e <= n; e += blockDim.x) {
    double a[4] = {0, 0, 0, 0};
    double G[4][kWin];
    for (int r = 0; r < 4; ++r)
      for (int q = 0; q < kWin; ++q) G[r][q] = 0.0;
    int ws = 0;
    if (e == 0) { // r <= x0: y0 + (y1 − y0)·t
      a[0] = y[0];
      a[1] = y[1] - y[0];
      G[0][0] = 1.0;
      G[1][0] = -1.0;
      G[1][1] = 1.0;
    } else if (e == n) { // r >= x_{n-1}: y_{n-1} + (y_{n-1} − y_{n-2})·t
      ws = n - W;
      const int ql = n - 1 - ws;
      a[0] = y[n - 1];
      a[1] = y[n - 1] - y[n - 2];
      G[0][ql] = 1.0;
      G[1][ql] = 1.0;
      G[1][ql - 1] = -1.0;
    } else {
      const int i = e - 1;
      ws = n >= kWin ? max(0, min(i - 2, n - kWin)) : 0;
      if (!cubic) {
        a[0] = y[i];
        a[1] = y[i + 1] - y[i];
        G[0][i - ws] = 1.0;
        G[1][i - ws] = -1.0;
        G[1][i + 1 - ws] = 1.0;
      } else {
        const double s0 = s[i], s1 = s[i + 1];
        a[0] = y[i];
        a[1] = h * s0;
        a[2] = -3.0 * y[i] - 2.0 * h * s0 + 3.0 * y[i + 1] - h * s1;
        a[3] = 2.0 * y[i] + h * s0 - 2.0 * y[i + 1] + h * s1;
        const int w0 = max(0, min(i - 2, n - 5)), w1 = max(0, min(i - 1, n - 5));
        for (int q = 0; q < W; ++q) {
          const int knot = ws + q;
          const double di = (knot == i) ? 1.0 : 0.0, di1 = (knot == i + 1) ? 1.0 : 0.0;
          const double g0 = (knot >= w0 && knot < w0 + 5) ? dS[i][knot - w0] : 0.0;
          const double g1 = (knot >= w1 && knot < w1 + 5) ? dS[i + 1][knot - w1] : 0.0;
          G[0][q] = di;
          G[1][q] = h * g0;
          G[2][q] = -3.0 * di - 2.0 * h * g0 + 3.0 * di1 - h * g1;
          G[3][q] = 2.0 * di + h * g0 - 2.0 * di1 + h * g1;
        }
      }
    }
    const int sg = td.seg0 + e;
    for (int r = 0; r < 4; ++r) seg_a[4 * sg + r] = static_cast<T>(a[r]);
    for (int r = 0; r < 4; ++r)
      for (int q = 0; q < kWin; ++q) seg_g[(4 * sg + r) * kWin + q] = static_cast<T>(G[r][q]);
    seg_ws[sg] = ws;
  }
}

} // namespace

// A pinned host buffer of at least n doubles (kept between calls).
int ensure_pinned(fs_gpu *h, double **buf, size_t *cap, size_t n) {
  if (*cap >= n && *buf) return FS_OK;
  if (*buf) cudaFreeHost(*buf);
  *buf = nullptr;
  *cap = 0;
  FS_CUDA(cudaMallocHost(buf, std::max<size_t>(n, 1) * sizeof(double)));
  *cap = std::max<size_t>(n, 1);
  return FS_OK;
}

int upload_tables(fs_gpu *h) {
  const int nt = static_cast<int>(h->tables.size());
  std::vector<TableDesc> desc(nt);
  // column map: a leading block of kWin entries −1 (a window that adds
  // nothing reads there), then each table's knots followed by kWin entries −1
  // (a window that runs past the table's last knot reads −1 there)
  std::vector<int32_t> cmap(kWin, -1);
  std::vector<double> vals;
  int segs = 0;
  for (int t = 0; t < nt; ++t) {
    const HostTable &ht = h->tables[t];
    TableDesc &d = desc[t];
    d = TableDesc{};
    d.kind = ht.kind;
    d.form = ht.form;
    d.n = ht.n;
    d.cmap0 = static_cast<int>(cmap.size());
    d.pv0 = static_cast<int>(vals.size());
    d.seg0 = -1;
    d.rmin = ht.rmin;
    d.rmax = ht.rmax;
    if (ht.kind == FS_TABLE_SPLINE) {
      if (ht.n > 512) return set_error(h, FS_ERR_UNSUPPORTED, "spline with more than 512 knots");
      d.seg0 = segs;
      segs += ht.n + 1;
      // potential_reader.cpp:178-182: x_k = rmin + k·h, h = (rmax − rmin)/(n − 1)
      d.h = (ht.rmax - ht.rmin) / static_cast<double>(ht.n - 1);
      d.x0 = ht.rmin + 0.0 * d.h;
      d.xmax = ht.rmin + static_cast<double>(ht.n - 1) * d.h;
      d.inv_h = 1.0 / d.h;
    } else if (ht.kind == FS_TABLE_ANALYTIC) {
      // closed form on its gate span [rmin, rmax] (the reference's range gate)
      d.x0 = ht.rmin;
      d.xmax = ht.rmax;
      d.h = d.inv_h = 1.0;
    }
    cmap.insert(cmap.end(), ht.cols.begin(), ht.cols.end());
    cmap.insert(cmap.end(), kWin, -1);
    vals.insert(vals.end(), ht.v.begin(), ht.v.end());
  }
  if (segs > kMaxSegs) return set_error(h, FS_ERR_UNSUPPORTED, "model has too many spline segments");
  const bool structure_changed = static_cast<int>(h->desc.size()) != nt || h->n_segs != segs ||
                                 h->n_cmap != static_cast<int>(cmap.size());
  h->desc = desc;
  if (structure_changed || !h->d_desc) {
    FS_TRY(realloc_dev(h, &h->d_desc, nt));
    FS_TRY(realloc_dev(h, &h->d_cmap, cmap.size()));
    FS_TRY(realloc_dev(h, &h->d_vals, vals.size()));
    const size_t es = h->precision == FS_PREC_FP64 ? sizeof(double) : sizeof(float);
    if (h->d_seg_a) cudaFree(h->d_seg_a);
    if (h->d_seg_g) cudaFree(h->d_seg_g);
    h->d_seg_a = h->d_seg_g = nullptr;
    if (cudaMalloc(&h->d_seg_a, std::max(segs, 1) * 4 * es) != cudaSuccess ||
        cudaMalloc(&h->d_seg_g, std::max(segs, 1) * 4 * kWin * es) != cudaSuccess)
      return set_error(h, FS_ERR_NOMEM, "cudaMalloc (segments)");
    FS_TRY(realloc_dev(h, &h->d_seg_ws, segs));
    FS_TRY(realloc_dev(h, &h->d_x, std::max(h->D, 1)));
  }
  h->n_segs = segs;
  h->n_cmap = static_cast<int>(cmap.size());
  h->n_vals = static_cast<int>(vals.size());
  FS_CUDA(cudaMemcpyAsync(h->d_desc, desc.data(), nt * sizeof(TableDesc), cudaMemcpyHostToDevice, h->stream));
  FS_CUDA(cudaMemcpyAsync(h->d_cmap, cmap.data(), cmap.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                          h->stream));
  FS_CUDA(cudaMemcpyAsync(h->d_vals, vals.data(), vals.size() * sizeof(double), cudaMemcpyHostToDevice,
                          h->stream));
  // pinned staging for the parameter values and the normal equations, sized
  // here (model set-up) rather than on a fit's first step
  FS_TRY(ensure_pinned(h, &h->h_vals_pin, &h->h_vals_pin_n, vals.size()));
  FS_TRY(ensure_pinned(h, &h->h_ne_pin, &h->h_ne_pin_n,
                       static_cast<size_t>(h->D) * h->D + h->D + 1));
  std::vector<int32_t> spl;
  for (int t = 0; t < nt; ++t)
    if (desc[t].kind == FS_TABLE_SPLINE) spl.push_back(t);
  if (h->d_spl) cudaFree(h->d_spl);
  h->d_spl = nullptr;
  h->n_spl = static_cast<int>(spl.size());
  if (!spl.empty()) {
    FS_CUDA(cudaMalloc(&h->d_spl, spl.size() * sizeof(int32_t)));
    FS_CUDA(cudaMemcpyAsync(h->d_spl, spl.data(), spl.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            h->stream));
  }
  FS_CUDA(cudaStreamSynchronize(h->stream));
  return FS_OK;
}

// New values of an unchanged model: one copy from a pinned buffer, ordered on
// the context's stream, no host wait (unless the previous upload from the
// buffer is still in flight).
int upload_values(fs_gpu *h) {
  size_t n = 0;
  for (const HostTable &ht : h->tables) n += ht.v.size();
  if (!h->d_vals || static_cast<int>(n) != h->n_vals) return upload_tables(h);
  FS_CUDA(cudaEventSynchronize(h->vals_ev)); // the previous upload from the buffer is done
  FS_TRY(ensure_pinned(h, &h->h_vals_pin, &h->h_vals_pin_n, n));
  size_t k = 0;
  for (const HostTable &ht : h->tables)
    for (double v : ht.v) h->h_vals_pin[k++] = v;
  FS_CUDA(cudaMemcpyAsync(h->d_vals, h->h_vals_pin, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  FS_CUDA(cudaEventRecord(h->vals_ev, h->stream));
  return FS_OK;
}

int refresh_segments(fs_gpu *h) {
  if (h->n_spl == 0) return FS_OK;
  if (h->precision == FS_PREC_FP64)
    spline_setup_kernel<double><<<h->n_spl, 128, 0, h->stream>>>(
        h->d_desc, h->d_spl, h->d_vals, static_cast<double *>(h->d_seg_a), static_cast<double *>(h->d_seg_g),
        h->d_seg_ws);
  else
    spline_setup_kernel<float><<<h->n_spl, 128, 0, h->stream>>>(
        h->d_desc, h->d_spl, h->d_vals, static_cast<float *>(h->d_seg_a), static_cast<float *>(h->d_seg_g),
        h->d_seg_ws);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  return FS_OK;
}

} // namespace fsg
