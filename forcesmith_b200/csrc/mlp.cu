// Surrogate objective model: MLP  D → 256 → 256 → 1  with GELU, BF16
// operands and FP32 accumulation on the 5th-generation tensor cores,
// trained with Adam by the kernels in this file.
//
// GEMM: C[m, n] = Σ_k A[m, k]·B[n, k] (both operands K-major BF16, N ≤ 256)
//   one CTA per 128-row tile of C (and per K split):
//   - a TMA thread streams 128×64 A tiles and 256×64 B tiles (128-byte
//     swizzle) through a 4-stage mbarrier ring (48 KB per stage);
//   - one thread issues tcgen05.mma.kind::f16 (BF16 × BF16 → FP32 in TMEM,
//     M = 128, N = 256, K = 16 per instruction);
//   - four warps drain the 128 × 256 FP32 accumulator (tcgen05.ld) to
//     global memory; K splits write partials that a second kernel sums in a
//     fixed order.
//   TMA fills rows ≥ M, rows ≥ N and columns ≥ K with zeros.  Waits are
//   bounded (error word, TMEM freed, return).
//
// Layers (rows = samples):
//   Z1 = X W1ᵀ + b1,  H1 = GELU(Z1)                     GEMM K = Dp
//   Z2 = H1 W2ᵀ + b2, H2 = GELU(Z2), y = H2·w3 + b3      GEMM K = 256, head by warps
// Backward of L = (1/B) Σ (y − t)²:
//   dy = 2(y − t)/B, dZ2 = dy·w3 ⊙ GELU′(Z2)
//   dW2 = dZ2ᵀ H1 (GEMM, K = B), dH1 = dZ2 W2 (GEMM with W2ᵀ), dZ1 = dH1 ⊙ GELU′(Z1)
//   dW1 = dZ1ᵀ X (GEMM, K = B), biases / w3 by column sums.
// BF16 rounding points: X, W1, W2, H1, dZ2 and dZ1 as GEMM operands; all
// other arithmetic is FP32.  GELU is the erf form x·Φ(x).
#include "internal.cuh"
#include "tc_common.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace fsg {
namespace {
using namespace tc;
using bf16 = __nv_bfloat16;

constexpr int kH = 256;
constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kGStages = 4;
constexpr uint32_t kABytes = kBM * kBK * 2;
constexpr uint32_t kBBytes = kH * kBK * 2;
constexpr uint32_t kGStageBytes = kABytes + kBBytes;
constexpr size_t kGemmSmem = kGStages * kGStageBytes + 1024 + 256;

__global__ void __launch_bounds__(128, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap bmap, int M,
                     int N, int K, int kper, float *__restrict__ out, int ldc, int32_t *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base =
      reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(base + kGStages * kGStageBytes);
  uint64_t *empty = full + kGStages;
  uint64_t *done = empty + kGStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
  __shared__ volatile int failed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM;
  const int k0 = blockIdx.y * kper;
  const int k1 = min(K, k0 + kper);
  const int nchunks = k1 > k0 ? (k1 - k0 + kBK - 1) / kBK : 0;
  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < kGStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kH)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    for (int kc = 0; kc < nchunks; ++kc) {
      const int s = kc % kGStages;
      if (kc >= kGStages && !mbar_wait(&empty[s], ((kc / kGStages) - 1) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      unsigned char *st = base + static_cast<size_t>(s) * kGStageBytes;
      mbar_expect_tx(&full[s], kGStageBytes);
      tma_load_2d(st, &amap, &full[s], k0 + kc * kBK, m0);
      tma_load_2d(st + kABytes, &bmap, &full[s], k0 + kc * kBK, 0);
    }
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = idesc_bf16(kBM, kH);
    for (int kc = 0; kc < nchunks; ++kc) {
      const int s = kc % kGStages;
      if (!mbar_wait(&full[s], (kc / kGStages) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(base + static_cast<size_t>(s) * kGStageBytes);
      const uint32_t sb = sa + kABytes;
#pragma unroll
      for (int ks = 0; ks < kBK / 16; ++ks) {
        const uint32_t k_off = ks * 32; // 16 BF16 of K = 32 bytes inside the swizzle row
        umma_bf16(tmem, desc_sw128(sa + k_off), desc_sw128(sb + k_off), idesc, (kc > 0 || ks > 0) ? 1u : 0u);
      }
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  __syncwarp();
  const bool ok = mbar_wait(done, 0);
  if (!ok) atomicExch(const_cast<int *>(&failed), 1);
  tc_fence_after();
  __syncthreads();
  if (!failed) {
    const int row = m0 + 32 * warp + lane;
    float *o = out + static_cast<size_t>(blockIdx.y) * M * ldc + static_cast<size_t>(row) * ldc;
    const uint32_t lane_base = static_cast<uint32_t>(32 * warp) << 16;
    float v[32];
    for (int c = 0; c < kH / 32; ++c) {
      if (c * 32 >= N) break; // warp-uniform
      tmem_ld_32(tmem + lane_base + c * 32, v);
      if (row < M) {
        if (nchunks == 0)
          for (int k = 0; k < 32; ++k) v[k] = 0.f;
        if (c * 32 + 32 <= N && (ldc & 3) == 0) {
#pragma unroll
          for (int k = 0; k < 32; k += 4)
            *reinterpret_cast<float4 *>(o + c * 32 + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
        } else {
          for (int k = 0; k < 32; ++k)
            if (c * 32 + k < N) o[c * 32 + k] = v[k];
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 2);
  }
  tc_fence_before();
  __syncthreads();
  if (failed && warp == 0 && lane == 0)
    for (int s = 0; s < kGStages; ++s) mbar_wait(&full[s], 0);
  __syncthreads();
  if (warp == 2)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kH) : "memory");
}

__global__ void split_sum_kernel(const float *__restrict__ part, int splits, int64_t n, float *__restrict__ out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < splits; ++k) s += part[k * n + i];
    out[i] = s;
  }
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Z = C + b; H = GELU(Z) (BF16, row-major and optionally transposed)
__global__ void bias_gelu_kernel(const float *__restrict__ C, const float *__restrict__ b, int rows,
                                 float *__restrict__ Z, bf16 *__restrict__ Hb, bf16 *__restrict__ HT) {
  const int64_t n = static_cast<int64_t>(rows) * kH;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(i % kH);
    const float z = C[i] + b[j];
    if (Z) Z[i] = z;
    const bf16 h = __float2bfloat16(gelu(z));
    Hb[i] = h;
    if (HT) HT[static_cast<int64_t>(j) * rows + i / kH] = h;
  }
}

// y = GELU(C + b2)·w3 + b3, one warp per row
__global__ void head_kernel(const float *__restrict__ C, const float *__restrict__ b2, const float *__restrict__ w3,
                            const float *__restrict__ b3, int rows, float *__restrict__ Z2, float *__restrict__ H2,
                            float *__restrict__ y) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;
  float acc = 0.f;
  for (int j = lane; j < kH; j += 32) {
    const int64_t i = static_cast<int64_t>(row) * kH + j;
    const float z = C[i] + b2[j];
    const float h = gelu(z);
    if (Z2) Z2[i] = z;
    if (H2) H2[i] = h;
    acc += h * w3[j];
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) y[row] = acc + b3[0];
}

// dy = 2(y − t)/B;  dZ2 = dy·w3 ⊙ GELU′(Z2) (FP32 + BF16 row-major + BF16 transposed); loss partial per row
__global__ void loss_back_kernel(const float *__restrict__ y, const float *__restrict__ t, int rows,
                                 const float *__restrict__ Z2, const float *__restrict__ w3, float *__restrict__ dy,
                                 float *__restrict__ dZ2, bf16 *__restrict__ dZ2b, bf16 *__restrict__ dZ2T,
                                 float *__restrict__ sq) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;
  const float e = y[row] - t[row];
  const float d = 2.f * e / static_cast<float>(rows);
  if (lane == 0) {
    dy[row] = d;
    sq[row] = e * e;
  }
  for (int j = lane; j < kH; j += 32) {
    const int64_t i = static_cast<int64_t>(row) * kH + j;
    const float g = d * w3[j] * gelu_d(Z2[i]);
    dZ2[i] = g;
    const bf16 gb = __float2bfloat16(g);
    dZ2b[i] = gb;
    dZ2T[static_cast<int64_t>(j) * rows + row] = gb;
  }
}

// dZ1 = dH1 ⊙ GELU′(Z1) (FP32 + BF16 transposed)
__global__ void gelu_back_kernel(const float *__restrict__ dH, const float *__restrict__ Z1, int rows,
                                 float *__restrict__ dZ1, bf16 *__restrict__ dZ1T) {
  const int64_t n = static_cast<int64_t>(rows) * kH;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float g = dH[i] * gelu_d(Z1[i]);
    dZ1[i] = g;
    dZ1T[(i % kH) * rows + i / kH] = __float2bfloat16(g);
  }
}

// out[j] = Σ_r X[r·ncols + j]·(s ? s[r] : 1), fixed order.  A block of
// kColsumRows × 32 threads takes 32 columns: thread (x, y) sums rows
// y, y + kColsumRows, … of column x (coalesced across x), and the partial
// sums meet in shared memory in the order of y.
constexpr int kColsumRows = 8;
__global__ void __launch_bounds__(32 * kColsumRows) colsum_kernel(const float *__restrict__ X,
                                                                  const float *__restrict__ s, int rows, int ncols,
                                                                  float *__restrict__ out) {
  __shared__ float part[kColsumRows][33];
  const int x = threadIdx.x & 31, y = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + x;
  float acc = 0.f;
  if (j < ncols)
    for (int r = y; r < rows; r += kColsumRows) acc += X[static_cast<int64_t>(r) * ncols + j] * (s ? s[r] : 1.f);
  part[y][x] = acc;
  __syncthreads();
  if (y == 0 && j < ncols) {
    float t = 0.f;
    for (int q = 0; q < kColsumRows; ++q) t += part[q][x];
    out[j] = t;
  }
}

__global__ void sum_kernel_f(const float *__restrict__ v, int n, float *__restrict__ out) {
  __shared__ float red[32];
  float acc = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += v[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) t += red[k];
    *out = t;
  }
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// BF16 operand copies of W1 (256 × Dp), W2 (256 × 256) and W2ᵀ
__global__ void pack_kernel(const float *__restrict__ W1, const float *__restrict__ W2, int Dp,
                            bf16 *__restrict__ W1b, bf16 *__restrict__ W2b, bf16 *__restrict__ W2T) {
  const int64_t n1 = static_cast<int64_t>(kH) * Dp;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n1 + kH * kH;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (i < n1) {
      W1b[i] = __float2bfloat16(W1[i]);
    } else {
      const int64_t k = i - n1;
      const bf16 w = __float2bfloat16(W2[k]);
      W2b[k] = w;
      W2T[(k % kH) * kH + k / kH] = w;
    }
  }
}

// X = BF16 rows of an FP32 host-normalised sample matrix (row stride Dp, zero pad)
__global__ void pack_x_kernel(const float *__restrict__ xs, int rows, int D, int Dp, bf16 *__restrict__ X,
                              bf16 *__restrict__ XT) {
  const int64_t n = static_cast<int64_t>(rows) * Dp;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / Dp;
    const int j = static_cast<int>(i % Dp);
    const bf16 v = __float2bfloat16(j < D ? xs[r * D + j] : 0.f);
    X[i] = v;
    if (XT) XT[static_cast<int64_t>(j) * rows + r] = v;
  }
}

inline int grid_for(int64_t n, int threads = 256) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16)));
}

bool make_map(CUtensorMap *map, const void *ptr, int64_t inner, int64_t outer, int64_t ld_elems, int box_outer) {
  auto enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t gdim[2] = {static_cast<cuuint64_t>(inner), static_cast<cuuint64_t>(outer)};
  const cuuint64_t gstride[1] = {static_cast<cuuint64_t>(ld_elems) * 2};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), static_cast<cuuint32_t>(box_outer)};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), gdim, gstride, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace

// ---------------------------------------------------------------------------
// the model state
struct Mlp {
  int D = 0, Dp = 0, cap = 0;
  int64_t n_dev = 0;            // flat device parameters (W1 padded to Dp columns)
  int64_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, ow3 = 0, ob3 = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16 *W1b = nullptr, *W2b = nullptr, *W2T = nullptr;
  bf16 *X = nullptr, *XT = nullptr, *H1 = nullptr, *H1T = nullptr, *dZ2b = nullptr, *dZ2T = nullptr,
       *dZ1T = nullptr;
  float *xs = nullptr, *C = nullptr, *Z1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *y = nullptr, *t = nullptr,
        *dy = nullptr, *dZ2 = nullptr, *dZ1 = nullptr, *part = nullptr, *sq = nullptr, *loss = nullptr;
  int64_t part_cap = 0;
  int64_t step = 0;
  float lr = 1e-3f, beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  bool packed = false;
};

namespace {

template <class T> int alloc(T **p, int64_t n) {
  return cudaMalloc(reinterpret_cast<void **>(p), std::max<int64_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : 1;
}

void free_rows(Mlp *s) {
  for (void *q : {(void *)s->X, (void *)s->XT, (void *)s->H1, (void *)s->H1T, (void *)s->dZ2b, (void *)s->dZ2T,
                  (void *)s->dZ1T, (void *)s->xs, (void *)s->C, (void *)s->Z1, (void *)s->Z2, (void *)s->H2,
                  (void *)s->y, (void *)s->t, (void *)s->dy, (void *)s->dZ2, (void *)s->dZ1, (void *)s->sq})
    cudaFree(q);
  s->X = s->XT = s->H1 = s->H1T = s->dZ2b = s->dZ2T = s->dZ1T = nullptr;
  s->xs = s->C = s->Z1 = s->Z2 = s->H2 = s->y = s->t = s->dy = s->dZ2 = s->dZ1 = s->sq = nullptr;
  s->cap = 0;
}

int ensure_rows(fs_gpu *h, Mlp *s, int rows) {
  if (rows <= s->cap) return FS_OK;
  free_rows(s);
  const int cap = (rows + 127) / 128 * 128;
  const int64_t rh = static_cast<int64_t>(cap) * kH, rd = static_cast<int64_t>(cap) * s->Dp;
  int bad = 0;
  bad |= alloc(&s->X, rd) | alloc(&s->XT, rd) | alloc(&s->H1, rh) | alloc(&s->H1T, rh) | alloc(&s->dZ2b, rh);
  bad |= alloc(&s->dZ2T, rh) | alloc(&s->dZ1T, rh) | alloc(&s->xs, static_cast<int64_t>(cap) * s->D);
  bad |= alloc(&s->C, rh) | alloc(&s->Z1, rh) | alloc(&s->Z2, rh) | alloc(&s->H2, rh) | alloc(&s->y, cap);
  bad |= alloc(&s->t, cap) | alloc(&s->dy, cap) | alloc(&s->dZ2, rh) | alloc(&s->dZ1, rh) | alloc(&s->sq, cap);
  if (bad) {
    free_rows(s);
    return set_error(h, FS_ERR_NOMEM, "surrogate: cudaMalloc");
  }
  s->cap = cap;
  return FS_OK;
}

int gemm(fs_gpu *h, Mlp *s, const bf16 *A, int64_t lda, const bf16 *B, int64_t ldb, int M, int N, int K, float *out,
         int ldc, int splits) {
  if (N > kH || M <= 0 || K <= 0 || (lda % 8) || (ldb % 8))
    return set_error(h, FS_ERR_ARG, "surrogate gemm: shape");
  CUtensorMap am, bm;
  if (!make_map(&am, A, K, M, lda, kBM) || !make_map(&bm, B, K, N, ldb, kH))
    return set_error(h, FS_ERR_CUDA, "surrogate gemm: tensor map");
  const int kchunks = (K + kBK - 1) / kBK;
  splits = std::max(1, std::min(splits, kchunks));
  const int kper = (kchunks + splits - 1) / splits * kBK;
  splits = (K + kper - 1) / kper;
  float *dst = out;
  if (splits > 1) {
    const int64_t need = static_cast<int64_t>(splits) * M * ldc;
    if (need > s->part_cap) {
      cudaFree(s->part);
      s->part = nullptr;
      if (alloc(&s->part, need)) return set_error(h, FS_ERR_NOMEM, "surrogate: cudaMalloc");
      s->part_cap = need;
    }
    dst = s->part;
  }
  if (!h->d_err) {
    FS_CUDA(cudaMalloc(&h->d_err, sizeof(int32_t)));
    FS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int32_t), h->stream));
  }
  FS_CUDA(cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(kGemmSmem)));
  dim3 grid((M + kBM - 1) / kBM, splits);
  gemm_bf16_kernel<<<grid, 128, kGemmSmem, h->stream>>>(am, bm, M, N, K, kper, dst, ldc, h->d_err);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  if (splits > 1) {
    const int64_t n = static_cast<int64_t>(M) * ldc;
    split_sum_kernel<<<grid_for(n), 256, 0, h->stream>>>(s->part, splits, n, out);
    FS_CUDA(cudaGetLastError());
    ++h->launches;
  }
  return FS_OK;
}

int pack_weights(fs_gpu *h, Mlp *s) {
  pack_kernel<<<grid_for(static_cast<int64_t>(kH) * (s->Dp + kH)), 256, 0, h->stream>>>(
      s->p + s->oW1, s->p + s->oW2, s->Dp, s->W1b, s->W2b, s->W2T);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  s->packed = true;
  return FS_OK;
}

} // namespace

void mlp_free(Mlp *s) {
  if (!s) return;
  free_rows(s);
  for (void *q : {(void *)s->p, (void *)s->g, (void *)s->m, (void *)s->v, (void *)s->W1b, (void *)s->W2b,
                  (void *)s->W2T, (void *)s->part, (void *)s->loss})
    cudaFree(q);
  delete s;
}

int64_t mlp_param_count(int D) { return static_cast<int64_t>(kH) * D + kH + kH * kH + kH + kH + 1; }

// Host layout (W1 [256 × D], b1, W2 [256 × 256], b2, w3, b3) ↔ device layout (W1 padded to Dp).
static void host_to_dev(const Mlp *s, const float *hp, std::vector<float> &dv) {
  dv.assign(s->n_dev, 0.f);
  for (int r = 0; r < kH; ++r)
    std::memcpy(&dv[s->oW1 + static_cast<int64_t>(r) * s->Dp], hp + static_cast<int64_t>(r) * s->D,
                s->D * sizeof(float));
  std::memcpy(&dv[s->ob1], hp + static_cast<int64_t>(kH) * s->D, (mlp_param_count(s->D) - kH * s->D) * sizeof(float));
}
static void dev_to_host(const Mlp *s, const std::vector<float> &dv, float *hp) {
  for (int r = 0; r < kH; ++r)
    std::memcpy(hp + static_cast<int64_t>(r) * s->D, &dv[s->oW1 + static_cast<int64_t>(r) * s->Dp],
                s->D * sizeof(float));
  std::memcpy(hp + static_cast<int64_t>(kH) * s->D, &dv[s->ob1], (mlp_param_count(s->D) - kH * s->D) * sizeof(float));
}

int mlp_create(fs_gpu *h, int D, uint64_t seed, float lr, Mlp **out) {
  if (D < 1 || D > kH) return set_error(h, FS_ERR_UNSUPPORTED, "surrogate: 1 <= D <= 256 parameters");
  Mlp *s = new Mlp();
  s->D = D;
  s->Dp = (D + 7) / 8 * 8;
  s->oW1 = 0;
  s->ob1 = static_cast<int64_t>(kH) * s->Dp;
  s->oW2 = s->ob1 + kH;
  s->ob2 = s->oW2 + kH * kH;
  s->ow3 = s->ob2 + kH;
  s->ob3 = s->ow3 + kH;
  s->n_dev = s->ob3 + 1;
  s->lr = lr;
  if (alloc(&s->p, s->n_dev) | alloc(&s->g, s->n_dev) | alloc(&s->m, s->n_dev) | alloc(&s->v, s->n_dev) |
      alloc(&s->W1b, static_cast<int64_t>(kH) * s->Dp) | alloc(&s->W2b, kH * kH) | alloc(&s->W2T, kH * kH) |
      alloc(&s->loss, 1)) {
    mlp_free(s);
    return set_error(h, FS_ERR_NOMEM, "surrogate: cudaMalloc");
  }
  // uniform(±1/√fan_in) initial weights from a seeded SplitMix64 stream; biases 0
  std::vector<float> hp(mlp_param_count(D), 0.f);
  uint64_t z = seed;
  auto u = [&]() {
    z += 0x9E3779B97F4A7C15ull;
    uint64_t q = z;
    q = (q ^ (q >> 30)) * 0xBF58476D1CE4E5B9ull;
    q = (q ^ (q >> 27)) * 0x94D049BB133111EBull;
    q ^= q >> 31;
    return static_cast<float>((q >> 11) * (1.0 / 9007199254740992.0));
  };
  const float a1 = 1.f / std::sqrt(static_cast<float>(D)), a2 = 1.f / 16.f;
  int64_t o = 0;
  for (int64_t k = 0; k < static_cast<int64_t>(kH) * D; ++k) hp[o++] = a1 * (2.f * u() - 1.f);
  o += kH;
  for (int64_t k = 0; k < kH * kH; ++k) hp[o++] = a2 * (2.f * u() - 1.f);
  o += kH;
  for (int64_t k = 0; k < kH; ++k) hp[o++] = a2 * (2.f * u() - 1.f);
  std::vector<float> dv;
  host_to_dev(s, hp.data(), dv);
  if (cudaMemcpyAsync(s->p, dv.data(), s->n_dev * sizeof(float), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
      cudaMemsetAsync(s->m, 0, s->n_dev * sizeof(float), h->stream) != cudaSuccess ||
      cudaMemsetAsync(s->v, 0, s->n_dev * sizeof(float), h->stream) != cudaSuccess ||
      cudaMemsetAsync(s->g, 0, s->n_dev * sizeof(float), h->stream) != cudaSuccess) {
    mlp_free(s);
    return set_error(h, FS_ERR_CUDA, "surrogate: upload");
  }
  int rc = pack_weights(h, s);
  if (rc != FS_OK) {
    mlp_free(s);
    return rc;
  }
  *out = s;
  return FS_OK;
}

int mlp_set_params(fs_gpu *h, Mlp *s, const float *hp) {
  std::vector<float> dv;
  host_to_dev(s, hp, dv);
  FS_CUDA(cudaMemcpyAsync(s->p, dv.data(), s->n_dev * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  return pack_weights(h, s);
}

int mlp_get(fs_gpu *h, Mlp *s, const float *dev, float *hp) {
  std::vector<float> dv(s->n_dev);
  FS_CUDA(cudaMemcpyAsync(dv.data(), dev, s->n_dev * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  FS_CUDA(cudaStreamSynchronize(h->stream));
  dev_to_host(s, dv, hp);
  return FS_OK;
}

float *mlp_param_ptr(Mlp *s) { return s->p; }
float *mlp_grad_ptr(Mlp *s) { return s->g; }
float *mlp_rows_x(Mlp *s) { return s->xs; }
float *mlp_rows_t(Mlp *s) { return s->t; }
float *mlp_rows_y(Mlp *s) { return s->y; }
int mlp_capacity(Mlp *s) { return s->cap; }
int mlp_reserve(fs_gpu *h, Mlp *s, int rows) { return ensure_rows(h, s, rows); }

// y = f(xs) for `rows` samples already in s->xs (FP32, row-major D).
int mlp_forward_dev(fs_gpu *h, Mlp *s, int rows) {
  FS_TRY(ensure_rows(h, s, rows));
  pack_x_kernel<<<grid_for(static_cast<int64_t>(rows) * s->Dp), 256, 0, h->stream>>>(s->xs, rows, s->D, s->Dp, s->X,
                                                                                     nullptr);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  FS_TRY(gemm(h, s, s->X, s->Dp, s->W1b, s->Dp, rows, kH, s->Dp, s->C, kH, 1));
  bias_gelu_kernel<<<grid_for(static_cast<int64_t>(rows) * kH), 256, 0, h->stream>>>(s->C, s->p + s->ob1, rows,
                                                                                      nullptr, s->H1, nullptr);
  FS_CUDA(cudaGetLastError());
  FS_TRY(gemm(h, s, s->H1, kH, s->W2b, kH, rows, kH, kH, s->C, kH, 1));
  head_kernel<<<(rows + 7) / 8, 256, 0, h->stream>>>(s->C, s->p + s->ob2, s->p + s->ow3, s->p + s->ob3, rows,
                                                     nullptr, nullptr, s->y);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

// Gradient of the mean squared error over `rows` samples (xs, t in the row
// buffers) into s->g; loss into s->loss.  rows must be a multiple of 8.
int mlp_gradient_dev(fs_gpu *h, Mlp *s, int rows) {
  if (rows % 8) return set_error(h, FS_ERR_ARG, "surrogate: training batch must be a multiple of 8");
  FS_TRY(ensure_rows(h, s, rows));
  const int64_t rh = static_cast<int64_t>(rows) * kH;
  pack_x_kernel<<<grid_for(static_cast<int64_t>(rows) * s->Dp), 256, 0, h->stream>>>(s->xs, rows, s->D, s->Dp, s->X,
                                                                                     s->XT);
  FS_CUDA(cudaGetLastError());
  FS_TRY(gemm(h, s, s->X, s->Dp, s->W1b, s->Dp, rows, kH, s->Dp, s->C, kH, 1));
  bias_gelu_kernel<<<grid_for(rh), 256, 0, h->stream>>>(s->C, s->p + s->ob1, rows, s->Z1, s->H1, s->H1T);
  FS_CUDA(cudaGetLastError());
  FS_TRY(gemm(h, s, s->H1, kH, s->W2b, kH, rows, kH, kH, s->C, kH, 1));
  head_kernel<<<(rows + 7) / 8, 256, 0, h->stream>>>(s->C, s->p + s->ob2, s->p + s->ow3, s->p + s->ob3, rows, s->Z2,
                                                     s->H2, s->y);
  FS_CUDA(cudaGetLastError());
  loss_back_kernel<<<(rows + 7) / 8, 256, 0, h->stream>>>(s->y, s->t, rows, s->Z2, s->p + s->ow3, s->dy, s->dZ2,
                                                          s->dZ2b, s->dZ2T, s->sq);
  FS_CUDA(cudaGetLastError());
  const int splits = std::max(1, std::min(16, rows / 256));
  // dW2 = dZ2ᵀ H1
  FS_TRY(gemm(h, s, s->dZ2T, rows, s->H1T, rows, kH, kH, rows, s->g + s->oW2, kH, splits));
  // dH1 = dZ2 W2  (B operand W2ᵀ)
  FS_TRY(gemm(h, s, s->dZ2b, kH, s->W2T, kH, rows, kH, kH, s->C, kH, 1));
  gelu_back_kernel<<<grid_for(rh), 256, 0, h->stream>>>(s->C, s->Z1, rows, s->dZ1, s->dZ1T);
  FS_CUDA(cudaGetLastError());
  // dW1 = dZ1ᵀ X  (columns padded to Dp; the pad columns of X are zero)
  FS_TRY(gemm(h, s, s->dZ1T, rows, s->XT, rows, kH, s->Dp, rows, s->g + s->oW1, s->Dp, splits));
  const unsigned cb = (kH + 31) / 32;
  colsum_kernel<<<cb, 32 * kColsumRows, 0, h->stream>>>(s->dZ1, nullptr, rows, kH, s->g + s->ob1);
  colsum_kernel<<<cb, 32 * kColsumRows, 0, h->stream>>>(s->dZ2, nullptr, rows, kH, s->g + s->ob2);
  colsum_kernel<<<cb, 32 * kColsumRows, 0, h->stream>>>(s->H2, s->dy, rows, kH, s->g + s->ow3);
  colsum_kernel<<<1, 32 * kColsumRows, 0, h->stream>>>(s->dy, nullptr, rows, 1, s->g + s->ob3);
  sum_kernel_f<<<1, 256, 0, h->stream>>>(s->sq, rows, s->loss);
  FS_CUDA(cudaGetLastError());
  h->launches += 10;
  return FS_OK;
}

int mlp_adam_dev(fs_gpu *h, Mlp *s) {
  s->step += 1;
  const float c1 = 1.f - std::pow(s->beta1, static_cast<float>(s->step));
  const float c2 = 1.f - std::pow(s->beta2, static_cast<float>(s->step));
  adam_kernel<<<grid_for(s->n_dev), 256, 0, h->stream>>>(s->p, s->g, s->m, s->v, s->n_dev, s->lr, s->beta1, s->beta2,
                                                         s->eps, c1, c2);
  FS_CUDA(cudaGetLastError());
  ++h->launches;
  return pack_weights(h, s);
}

float *mlp_loss_ptr(Mlp *s) { return s->loss; }

} // namespace fsg
