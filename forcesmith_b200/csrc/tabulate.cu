// Tabulation: value and d/dr of one radial table of the current model at
// given points, in FP64 whatever the working precision.
//
// The reference's writers sample each RadialPotential on a uniform grid of
// its span, p.eval(r) and p.deriv(r) (output_writer.cpp:22-40 for the native
// JSON, 266-289 for LAMMPS, 291-310 for IMD).  Here the sampling runs the
// same device code the evaluation kernels run: the makima segment (rebuilt in
// FP64 from the current parameter vector) or the analytic form, with the
// extended linear segments outside a spline's knot span.
#include "internal.cuh"
#include "spline_dev.cuh"

using namespace fsg;

namespace fsg {
namespace {

__global__ void __launch_bounds__(256) tabulate_kernel(TableDesc td, const double4 *__restrict__ seg,
                                                       const double *__restrict__ vals, const double *__restrict__ r,
                                                       int n, double *__restrict__ v, double *__restrict__ dv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  STab<double> tb;
  load_stab(tb, td);
  const VD<double> o = tab_vd<double, true>(tb, seg, vals, r[i]);
  v[i] = o.v;
  dv[i] = o.d;
}

} // namespace
} // namespace fsg

extern "C" int fs_gpu_tabulate(fs_gpu *h, int32_t table, int32_t n, const double *r, double *value, double *deriv) {
  if (!h || n < 0 || (n > 0 && (!r || !value || !deriv))) return FS_ERR_ARG;
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "tabulate: no model");
  if (table < 0 || table >= static_cast<int>(h->tables.size()))
    return set_error(h, FS_ERR_ARG, "tabulate: table index out of range");
  const HostTable &ht = h->tables[table];
  if (ht.kind != FS_TABLE_SPLINE && ht.kind != FS_TABLE_ANALYTIC)
    return set_error(h, FS_ERR_ARG, "tabulate: table " + std::to_string(table) + " is not a radial table");
  if (n == 0) return FS_OK;
  for (int k = 0; k < n; ++k)
    if (!std::isfinite(r[k])) return set_error(h, FS_ERR_ARG, "tabulate: non-finite sample point");
  cudaSetDevice(h->device);
  // the current parameter vector, from the host copy of the tables
  std::vector<double> x(std::max(h->D, 1), 0.0);
  for (const HostTable &t : h->tables)
    for (int k = 0; k < t.n; ++k)
      if (t.cols[k] >= 0) x[t.cols[k]] = t.v[k];
  // every block starts on a 256-byte boundary (double4 loads need 16)
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t nx = x.size() * sizeof(double), np = static_cast<size_t>(n) * sizeof(double); // bytes copied
  const size_t bx = up(nx), bs = up(std::max(h->n_segs, 1) * sizeof(double4)), bp = up(np);   // blocks
  char *buf = nullptr;
  if (cudaMalloc(&buf, bx + bs + 3 * bp) != cudaSuccess) return set_error(h, FS_ERR_NOMEM, "tabulate: cudaMalloc");
  double *d_x1 = reinterpret_cast<double *>(buf);
  double4 *d_seg = reinterpret_cast<double4 *>(buf + bx);
  double *d_r = reinterpret_cast<double *>(buf + bx + bs);
  double *d_v = reinterpret_cast<double *>(buf + bx + bs + bp);
  double *d_dv = reinterpret_cast<double *>(buf + bx + bs + 2 * bp);
  int rc = FS_OK;
  auto cuda_ok = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && rc == FS_OK) rc = set_error(h, FS_ERR_CUDA, std::string("tabulate: ") + what);
    return rc == FS_OK;
  };
  if (cuda_ok(cudaMemcpyAsync(d_x1, x.data(), nx, cudaMemcpyHostToDevice, h->stream), "copy x") &&
      cuda_ok(cudaMemcpyAsync(d_r, r, np, cudaMemcpyHostToDevice, h->stream), "copy r")) {
    if (ht.kind == FS_TABLE_SPLINE) rc = spline_segments_fp64(h, d_x1, d_seg);
    if (rc == FS_OK) {
      tabulate_kernel<<<(n + 255) / 256, 256, 0, h->stream>>>(h->desc[table], d_seg, h->d_vals, d_r, n, d_v, d_dv);
      if (cuda_ok(cudaGetLastError(), "launch")) {
        ++h->launches;
        if (cuda_ok(cudaMemcpyAsync(value, d_v, np, cudaMemcpyDeviceToHost, h->stream), "copy values") &&
            cuda_ok(cudaMemcpyAsync(deriv, d_dv, np, cudaMemcpyDeviceToHost, h->stream), "copy derivatives"))
          rc = sync_checked(h);
      }
    }
  }
  cudaStreamSynchronize(h->stream);
  cudaFree(buf);
  return rc;
}
