// JᵀJ on the 5th-generation tensor cores (tcgen05.mma, kind::tf32).
//
// J is column-major (ld × D, FP32), i.e. Jᵀ is row-major with the residual
// rows as the contraction dimension K — K-major for both operands.  Each CTA
// owns a contiguous slab of rows (split-K over 148 SMs):
//   - a TMA producer thread streams 32-row × 256-column tiles of Jᵀ
//     (32 KB, 128-byte swizzle) through a 3-stage mbarrier ring;
//   - two warps split every landed tile into hi = TF32(x) (round to nearest)
//     in place and lo = x − hi beside it (3×TF32: hi·hi + hi·lo + lo·hi keeps
//     ≈ 2⁻²¹ relative accuracy, where plain TF32 truncation biases JᵀJ by
//     ≈ −1e-3);
//   - one thread issues the MMAs: rows [0,128) of Jᵀ against all 256 columns
//     (M=128, N=256) and rows [128,256) against columns [128,256) (M=128,
//     N=128) — the lower-left block is the transpose of the upper-right;
//     both accumulators live in TMEM (384 of 512 columns), FP32;
//   - all four warps drain TMEM (tcgen05.ld) into an FP64 per-CTA partial;
//     a second kernel sums the partials in a fixed order (FP64 accumulation
//     across slabs, deterministic) and mirrors the lower-left block.
// Columns ≥ D and rows ≥ M are zero (TMA out-of-bounds fill / zeroed pad).
// Every mbarrier wait is bounded: on expiry the kernel sets an error word,
// skips the remaining work, frees its TMEM and returns.
#include "internal.cuh"
#include "tc_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

namespace fsg {
namespace {
using namespace tc;

constexpr int kStages = 3;
constexpr int kKChunk = 32;                                  // rows of J per stage (128 B of FP32)
constexpr int kTileN = 256;                                  // columns of J per stage
constexpr uint32_t kTileBytes = kKChunk * kTileN * 4;        // 32 KB landed by TMA (then hi)
constexpr uint32_t kStageBytes = 2 * kTileBytes;             // + 32 KB lo
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 512;

__global__ void __launch_bounds__(kThreads, 1)
    gram_tc_kernel(const __grid_constant__ CUtensorMap tmap, int D, int64_t rows_per_cta, int64_t ld,
                   double *__restrict__ part, int32_t *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base =
      reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char *stage = base;
  uint64_t *full = reinterpret_cast<uint64_t *>(base + kStages * kStageBytes);
  uint64_t *empty = full + kStages;
  uint64_t *conv = empty + kStages;
  uint64_t *done = conv + kStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
  __shared__ volatile int failed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * rows_per_cta;
  const int64_t r1 = min(ld, r0 + rows_per_cta);
  const int nchunks = static_cast<int>((r1 - r0 + kKChunk - 1) / kKChunk);
  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
      mbar_init(&conv[s], 2);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // TMA producer
    for (int kc = 0; kc < nchunks; ++kc) {
      const int s = kc % kStages;
      if (kc >= kStages && !mbar_wait(&empty[s], ((kc / kStages) - 1) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      mbar_expect_tx(&full[s], kTileBytes);
      tma_load_2d(stage + static_cast<size_t>(s) * kStageBytes, &tmap, &full[s],
                  static_cast<int>(r0 + static_cast<int64_t>(kc) * kKChunk), 0);
    }
  } else if (warp >= 2) {
    // hi/lo split of every landed tile (element-wise, so the swizzle is kept)
    for (int kc = 0; kc < nchunks && !failed; ++kc) {
      const int s = kc % kStages;
      if (!mbar_wait(&full[s], (kc / kStages) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      float4 *hi = reinterpret_cast<float4 *>(stage + static_cast<size_t>(s) * kStageBytes);
      float4 *lo = reinterpret_cast<float4 *>(stage + static_cast<size_t>(s) * kStageBytes + kTileBytes);
      for (int k = threadIdx.x - 64; k < static_cast<int>(kTileBytes / 16); k += 64) {
        const float4 x = hi[k];
        float4 a, b;
        const float *xs = &x.x;
        float *as = &a.x, *bs = &b.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float h = __uint_as_float((__float_as_uint(xs[e]) + 0x1000u) & 0xFFFFE000u);
          as[e] = h;
          bs[e] = xs[e] - h;
        }
        hi[k] = a;
        lo[k] = b;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&conv[s]);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: per 8-element K step, hi·hi + hi·lo + lo·hi for both blocks
    constexpr uint32_t id_full = idesc_tf32(128, 256), id_half = idesc_tf32(128, 128);
    for (int kc = 0; kc < nchunks; ++kc) {
      const int s = kc % kStages;
      if (!mbar_wait(&conv[s], (kc / kStages) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      tc_fence_after();
      const uint32_t sh = smem_u32(stage + static_cast<size_t>(s) * kStageBytes);
      const uint32_t sl = sh + kTileBytes;
#pragma unroll
      for (int ks = 0; ks < kKChunk / 8; ++ks) {
        const uint32_t k_off = ks * 32; // 8 TF32 elements of K = 32 bytes inside the swizzle row
        const uint32_t acc = (kc > 0 || ks > 0) ? 1u : 0u;
        umma_tf32(tmem, desc_sw128(sh + k_off), desc_sw128(sh + k_off), id_full, acc);
        umma_tf32(tmem, desc_sw128(sh + k_off), desc_sw128(sl + k_off), id_full, 1u);
        umma_tf32(tmem, desc_sw128(sl + k_off), desc_sw128(sh + k_off), id_full, 1u);
        umma_tf32(tmem + 256, desc_sw128(sh + 16384 + k_off), desc_sw128(sh + 16384 + k_off), id_half, acc);
        umma_tf32(tmem + 256, desc_sw128(sh + 16384 + k_off), desc_sw128(sl + 16384 + k_off), id_half, 1u);
        umma_tf32(tmem + 256, desc_sw128(sl + 16384 + k_off), desc_sw128(sh + 16384 + k_off), id_half, 1u);
      }
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  __syncwarp();
  // epilogue: every warp drains its 32 TMEM lanes
  const bool ok = mbar_wait(done, 0);
  if (!ok) atomicExch(const_cast<int *>(&failed), 1);
  tc_fence_after();
  __syncthreads();
  if (!failed) {
    double *P = part + static_cast<size_t>(blockIdx.x) * D * D;
    const uint32_t lane_base = static_cast<uint32_t>(32 * warp) << 16;
    float v[32];
    const int row0 = 32 * warp + lane;
    for (int c = 0; c < 8; ++c) { // rows [0,128) × columns [0,256)
      tmem_ld_32(tmem + lane_base + c * 32, v);
      if (row0 < D)
        for (int k = 0; k < 32; ++k) {
          const int col = c * 32 + k;
          if (col < D) P[static_cast<size_t>(row0) * D + col] = static_cast<double>(v[k]);
        }
    }
    const int row1 = 128 + 32 * warp + lane;
    for (int c = 0; c < 4; ++c) { // rows [128,256) × columns [128,256)
      tmem_ld_32(tmem + lane_base + 256 + c * 32, v);
      if (row1 < D)
        for (int k = 0; k < 32; ++k) {
          const int col = 128 + c * 32 + k;
          if (col < D) P[static_cast<size_t>(row1) * D + col] = static_cast<double>(v[k]);
        }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (failed && warp == 0 && lane == 0) {
    // let in-flight TMA copies land before the CTA's shared memory goes away
    for (int s = 0; s < kStages; ++s) mbar_wait(&full[s], 0);
  }
  __syncthreads();
  if (warp == 2)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Σ over CTAs in a fixed order; the lower triangle mirrors the upper one, so
// JᵀJ is exactly symmetric.
__global__ void gram_tc_reduce_kernel(const double *__restrict__ part, int nparts, int D, double *__restrict__ JtJ) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= D * D) return;
  const int a = idx / D, b = idx % D;
  const size_t src = (a > b) ? static_cast<size_t>(b) * D + a : static_cast<size_t>(idx);
  double s = 0.0;
  for (int k = 0; k < nparts; ++k) s += part[static_cast<size_t>(k) * D * D + src];
  JtJ[idx] = s;
}

} // namespace

namespace tc {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

} // namespace tc

int gram_tc(fs_gpu *h, int64_t M, double *JtJ) {
  const int D = h->D;
  const int64_t ld = h->ldj;
  (void)M;
  auto enc = encode_fn();
  if (!enc) return set_error(h, FS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  CUtensorMap map;
  const cuuint64_t gdim[2] = {static_cast<cuuint64_t>(ld), static_cast<cuuint64_t>(D)};
  const cuuint64_t gstride[1] = {static_cast<cuuint64_t>(ld) * sizeof(float)};
  const cuuint32_t box[2] = {kKChunk, kTileN};
  const cuuint32_t estr[2] = {1, 1};
  CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->d_J, gdim, gstride, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return set_error(h, FS_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  const int64_t chunks = ld / kKChunk;
  int ncta = static_cast<int>(std::min<int64_t>(148, chunks));
  const int64_t rows_per_cta = (chunks + ncta - 1) / ncta * kKChunk;
  ncta = static_cast<int>((ld + rows_per_cta - 1) / rows_per_cta);
  const size_t need = static_cast<size_t>(ncta) * D * D;
  if (h->gram_part_alloc < need || !h->d_gram_part) {
    if (h->d_gram_part) cudaFree(h->d_gram_part);
    h->d_gram_part = nullptr;
    FS_CUDA(cudaMalloc(&h->d_gram_part, need * sizeof(double)));
    h->gram_part_alloc = need;
  }
  if (!h->d_err) {
    FS_CUDA(cudaMalloc(&h->d_err, sizeof(int32_t)));
    FS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int32_t), h->stream));
  }
  const size_t smem = kStages * kStageBytes + 1024 + 256; // 3 × 64 KB + barriers
  FS_CUDA(cudaFuncSetAttribute(gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  gram_tc_kernel<<<ncta, kThreads, smem, h->stream>>>(map, D, rows_per_cta, ld, h->d_gram_part, h->d_err);
  FS_CUDA(cudaGetLastError());
  gram_tc_reduce_kernel<<<(D * D + 255) / 256, 256, 0, h->stream>>>(h->d_gram_part, ncta, D, JtJ);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

} // namespace fsg
