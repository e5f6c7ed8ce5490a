// Normal-equation product JᵀJ (D × D) with FP64 accumulation, an input of
// NormalEquationsSolver and the LM step (src/optimization/solver.cpp:242-266);
// Jᵀr is accumulated in FP64 by the Jacobian kernels themselves.
//
// SIMT paths.  D ≤ 48: a row-slab kernel over the upper triangle.  Otherwise
// (FP64 mode, or D > 256): 64 × 64 output tiles (upper triangle only) × a
// split of the rows.
// Each 32-row slab is multiplied in the working precision and folded into
// FP64 accumulators, so the FP32 partial sums never exceed 32 terms.
// Split partials are reduced in a fixed order (deterministic result).
#include "internal.cuh"

#include <algorithm>

namespace fsg {
namespace {

constexpr int TB = 64, KS = 32;

template <class T>
__global__ void __launch_bounds__(256) gram_partial_kernel(const T *__restrict__ J, int64_t ld, int64_t M, int D,
                                                           int64_t rows_per_split, const int2 *__restrict__ tiles,
                                                           double *__restrict__ part) {
  __shared__ T As[KS][TB + 1];
  __shared__ T Bs[KS][TB + 1];
  const int2 tp = tiles[blockIdx.x];
  const int split = blockIdx.y;
  const int a0 = tp.x * TB, b0 = tp.y * TB;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t r_begin = static_cast<int64_t>(split) * rows_per_split;
  const int64_t r_end = min(M, r_begin + rows_per_split);
  double acc[4][4];
  for (int x = 0; x < 4; ++x)
    for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
  for (int64_t r0 = r_begin; r0 < r_end; r0 += KS) {
    // load As[k][c] = J[r0+k, a0+c]; column-major: consecutive k are contiguous
    for (int idx = threadIdx.x; idx < KS * TB; idx += blockDim.x) {
      const int k = idx % KS, cc = idx / KS;
      const int64_t r = r0 + k;
      const int ca = a0 + cc, cb = b0 + cc;
      As[k][cc] = (r < r_end && ca < D) ? J[static_cast<int64_t>(ca) * ld + r] : T(0);
      Bs[k][cc] = (r < r_end && cb < D) ? J[static_cast<int64_t>(cb) * ld + r] : T(0);
    }
    __syncthreads();
    T s[4][4];
    for (int x = 0; x < 4; ++x)
      for (int y = 0; y < 4; ++y) s[x][y] = T(0);
#pragma unroll 8
    for (int k = 0; k < KS; ++k) {
      T av[4], bv[4];
      for (int x = 0; x < 4; ++x) av[x] = As[k][tx * 4 + x];
      for (int y = 0; y < 4; ++y) bv[y] = Bs[k][ty * 4 + y];
      for (int x = 0; x < 4; ++x)
        for (int y = 0; y < 4; ++y) s[x][y] += av[x] * bv[y];
    }
    for (int x = 0; x < 4; ++x)
      for (int y = 0; y < 4; ++y) acc[x][y] += static_cast<double>(s[x][y]);
    __syncthreads();
  }
  double *P = part + static_cast<size_t>(split) * D * D;
  for (int x = 0; x < 4; ++x)
    for (int y = 0; y < 4; ++y) {
      const int a = a0 + tx * 4 + x, b = b0 + ty * 4 + y;
      if (a < D && b < D) P[static_cast<size_t>(a) * D + b] = acc[x][y];
    }
}

// Small D (≤ kGramSmallD): CTA = a slab of rows, staged 32 rows at a time.
// With P = D(D+1)/2 upper-triangle entries: P ≥ 256, thread t owns entries
// t, t + 256, …; P < 256, the threads form G = ⌊256 / P⌋ row groups, thread
// t owning entry t mod P over the slab rows ≡ ⌊t / P⌋ (mod G), and the groups'
// sums are added in order at the end.  Each thread's sums over a staged slab
// are in the working precision, folded into FP64.
constexpr int kSmallPer = (kGramSmallD * (kGramSmallD + 1) / 2 + 255) / 256;

template <class T>
__global__ void __launch_bounds__(256) gram_small_kernel(const T *__restrict__ J, int64_t ld, int64_t M, int D,
                                                         int64_t rows_per_cta, double *__restrict__ part) {
  __shared__ T S[KS][kGramSmallD + 1];
  __shared__ double red[256];
  const int npairs = D * (D + 1) / 2;
  const int G = npairs >= 256 ? 1 : 256 / npairs;
  const int g = G > 1 ? static_cast<int>(threadIdx.x) / npairs : 0;
  const bool mine = G == 1 || static_cast<int>(threadIdx.x) < G * npairs;
  const int nper = G > 1 ? 1 : kSmallPer;
  int pa[kSmallPer], pb[kSmallPer];
  double acc[kSmallPer];
#pragma unroll
  for (int u = 0; u < kSmallPer; ++u) {
    int p = G > 1 ? static_cast<int>(threadIdx.x) % npairs : static_cast<int>(threadIdx.x) + 256 * u, a = 0;
    if (p >= npairs) p = 0;
    while (p >= D - a) { // row a of the upper triangle holds D − a entries
      p -= D - a;
      ++a;
    }
    pa[u] = a;
    pb[u] = a + p;
    acc[u] = 0.0;
  }
  const int64_t r_begin = static_cast<int64_t>(blockIdx.x) * rows_per_cta;
  const int64_t r_end = min(M, r_begin + rows_per_cta);
  for (int64_t r0 = r_begin; r0 < r_end; r0 += KS) {
    for (int idx = threadIdx.x; idx < KS * D; idx += blockDim.x) { // contiguous along the rows
      const int k = idx % KS, c = idx / KS;
      const int64_t r = r0 + k;
      S[k][c] = r < r_end ? J[static_cast<int64_t>(c) * ld + r] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kSmallPer; ++u)
      if (u < nper) {
        T s = T(0);
        for (int k = g; k < KS; k += G) s += S[k][pa[u]] * S[k][pb[u]];
        acc[u] += static_cast<double>(s);
      }
    __syncthreads();
  }
  double *P = part + static_cast<size_t>(blockIdx.x) * D * D;
  if (G == 1) {
#pragma unroll
    for (int u = 0; u < kSmallPer; ++u)
      if (static_cast<int>(threadIdx.x) + 256 * u < npairs) P[static_cast<size_t>(pa[u]) * D + pb[u]] = acc[u];
  } else {
    red[threadIdx.x] = mine ? acc[0] : 0.0; // index g·P + entry
    __syncthreads();
    if (static_cast<int>(threadIdx.x) < npairs) {
      double t = 0.0;
      for (int gg = 0; gg < G; ++gg) t += red[gg * npairs + threadIdx.x];
      P[static_cast<size_t>(pa[0]) * D + pb[0]] = t;
    }
  }
}

__global__ void gram_reduce_kernel(const double *__restrict__ part, int splits, int D, double *__restrict__ JtJ) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < D * D) {
    const int a = idx / D, b = idx % D;
    if (a <= b) { // upper triangle, mirrored: JᵀJ is exactly symmetric
      double s = 0.0;
      for (int k = 0; k < splits; ++k) s += part[static_cast<size_t>(k) * D * D + idx];
      JtJ[idx] = s;
      JtJ[static_cast<size_t>(b) * D + a] = s;
    }
  }
}

} // namespace

int gram(fs_gpu *h, int64_t M, double *JtJ, double *) {
  const int D = h->D;
  if (D == 0) return FS_OK;
  if (gram_on_tensor_cores(h->precision, D)) return gram_tc(h, M, JtJ);
  if (D <= kGramSmallD) {
    int ncta = 4 * 148;
    int64_t rpc = (M + ncta - 1) / ncta;
    rpc = (rpc + KS - 1) / KS * KS;
    ncta = static_cast<int>((M + rpc - 1) / rpc);
    const size_t need = static_cast<size_t>(ncta) * D * D;
    if (h->gram_part_alloc < need || !h->d_gram_part) {
      if (h->d_gram_part) cudaFree(h->d_gram_part);
      h->d_gram_part = nullptr;
      FS_CUDA(cudaMalloc(&h->d_gram_part, need * sizeof(double)));
      h->gram_part_alloc = need;
    }
    if (h->precision == FS_PREC_FP64)
      gram_small_kernel<double><<<ncta, 256, 0, h->stream>>>(static_cast<const double *>(h->d_J), h->ldj, M, D, rpc,
                                                              h->d_gram_part);
    else
      gram_small_kernel<float><<<ncta, 256, 0, h->stream>>>(static_cast<const float *>(h->d_J), h->ldj, M, D, rpc,
                                                             h->d_gram_part);
    FS_CUDA(cudaGetLastError());
    gram_reduce_kernel<<<(D * D + 255) / 256, 256, 0, h->stream>>>(h->d_gram_part, ncta, D, JtJ);
    FS_CUDA(cudaGetLastError());
    h->launches += 2;
    return FS_OK;
  }
  const int T = (D + TB - 1) / TB;
  std::vector<int2> tiles;
  for (int a = 0; a < T; ++a)
    for (int b = a; b < T; ++b) tiles.push_back(make_int2(a, b));
  const int nt = static_cast<int>(tiles.size());
  int splits = std::max(1, (4 * 148) / nt);
  int64_t rps = (M + splits - 1) / splits;
  rps = (rps + KS - 1) / KS * KS;
  splits = static_cast<int>((M + rps - 1) / rps);
  const size_t need = static_cast<size_t>(splits) * D * D + 2 * nt;
  if (h->gram_part_alloc < need || !h->d_gram_part) {
    if (h->d_gram_part) cudaFree(h->d_gram_part);
    h->d_gram_part = nullptr;
    FS_CUDA(cudaMalloc(&h->d_gram_part, need * sizeof(double)));
    h->gram_part_alloc = need;
  }
  double *part = h->d_gram_part;
  int2 *d_tiles = reinterpret_cast<int2 *>(part + static_cast<size_t>(splits) * D * D);
  FS_CUDA(cudaMemcpyAsync(d_tiles, tiles.data(), nt * sizeof(int2), cudaMemcpyHostToDevice, h->stream));
  dim3 grid(nt, splits);
  if (h->precision == FS_PREC_FP64)
    gram_partial_kernel<double><<<grid, 256, 0, h->stream>>>(static_cast<const double *>(h->d_J), h->ldj, M, D,
                                                              rps, d_tiles, part);
  else
    gram_partial_kernel<float><<<grid, 256, 0, h->stream>>>(static_cast<const float *>(h->d_J), h->ldj, M, D, rps,
                                                            d_tiles, part);
  FS_CUDA(cudaGetLastError());
  gram_reduce_kernel<<<(D * D + 255) / 256, 256, 0, h->stream>>>(part, splits, D, JtJ);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

} // namespace fsg
