// JᵀJ on the 5th-generation tensor cores (tcgen05.mma, kind::tf32).
//
// The MMAs read both operands K-major (the residual rows are the contraction
// dimension K), 32 rows × 256 columns per stage with the 128-byte swizzle.
// Each CTA owns a contiguous slab of rows (split-K over 148 SMs):
//   - a TMA producer thread streams 32-row × 256-column tiles of J through
//     an mbarrier ring.  Column-major J (ld × D): the tile lands K-major and
//     swizzled (3 stages).  Row-major J (rows × ld, written that way so that
//     each atom's rows are contiguous for its producer): the tile lands
//     row-major, unswizzled, beside the K-major buffers (2 stages);
//   - eight warps split every landed tile into hi = TF32(x) (round to nearest)
//     and lo = x − hi (3×TF32: hi·hi + hi·lo + lo·hi keeps ≈ 2⁻²¹ relative
//     accuracy, where plain TF32 truncation biases JᵀJ by ≈ −1e-3): in place
//     for column-major J, transposed into the swizzled K-major layout for
//     row-major J;
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

constexpr int kKChunk = 32;                                  // rows of J per stage (128 B of FP32)
constexpr int kTileN = 256;                                  // columns of J per stage
constexpr uint32_t kTileBytes = kKChunk * kTileN * 4;        // 32 KB
constexpr int kConvWarps = 8;                                // warps 2..9 split the tiles
constexpr int kThreads = 64 + 32 * kConvWarps;
constexpr uint32_t kTmemCols = 512;
// Shared memory: NB buffers [hi | lo] of 64 KB that the MMAs read, and the NL
// slots TMA lands tiles in.  Column-major J lands in a buffer's hi half (NL =
// NB = 3: one ring).  Row-major J lands in NL = 3 slots of its own before
// the buffers (3 × 32 + 2 × 64 = 224 KB), freed as soon as the split has
// read them, so TMA runs ahead of the MMAs.
template <bool RM> struct GramLayout {
  static constexpr int NL = 3, NB = RM ? 2 : 3;
  static constexpr uint32_t land_bytes = RM ? NL * kTileBytes : 0;
  static constexpr uint32_t bytes = land_bytes + NB * 2 * kTileBytes;
  __device__ static unsigned char *land(unsigned char *b, int s) {
    return RM ? b + s * kTileBytes : b + s * 2 * kTileBytes;
  }
  __device__ static unsigned char *hi(unsigned char *b, int t) { return b + land_bytes + t * 2 * kTileBytes; }
};

template <bool RM>
__global__ void __launch_bounds__(kThreads, 1)
    gram_tc_kernel(const __grid_constant__ CUtensorMap tmap, int D, int64_t rows_per_cta, int64_t nrows,
                   double *__restrict__ part, int32_t *__restrict__ err) {
  using GL = GramLayout<RM>;
  constexpr int NL = GL::NL, NB = GL::NB;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base =
      reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  // full[s]: slot s landed; lfree[s]: slot s read (row-major only); conv[t]:
  // buffer t split; empty[t]: the MMAs on buffer t are done
  uint64_t *full = reinterpret_cast<uint64_t *>(base + GL::bytes);
  uint64_t *lfree = full + NL;
  uint64_t *conv = lfree + NL;
  uint64_t *empty = conv + NB;
  uint64_t *done = empty + NB;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
  __shared__ volatile int failed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * rows_per_cta;
  const int64_t r1 = min(nrows, r0 + rows_per_cta);
  const int nchunks = static_cast<int>((r1 - r0 + kKChunk - 1) / kKChunk);
  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < NL; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&lfree[s], kConvWarps);
    }
    for (int t = 0; t < NB; ++t) {
      mbar_init(&conv[t], kConvWarps);
      mbar_init(&empty[t], 1);
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
      const int s = kc % NL;
      // the slot is free once split (row-major) or once its MMAs are done (column-major: in place)
      if (kc >= NL && !mbar_wait(RM ? &lfree[s] : &empty[s], ((kc / NL) - 1) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      mbar_expect_tx(&full[s], kTileBytes);
      const int row = static_cast<int>(r0 + static_cast<int64_t>(kc) * kKChunk);
      if constexpr (RM)
        tma_load_2d(GL::land(base, s), &tmap, &full[s], 0, row);
      else
        tma_load_2d(GL::land(base, s), &tmap, &full[s], row, 0);
    }
  } else if (warp >= 2) {
    // hi/lo split of every landed tile (element-wise, so the swizzle is kept)
    for (int kc = 0; kc < nchunks && !failed; ++kc) {
      const int s = kc % NL, t = kc % NB;
      if (!mbar_wait(&full[s], (kc / NL) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      // row-major: buffer t must be free of the MMAs of two chunks back
      if (RM && kc >= NB && !mbar_wait(&empty[t], ((kc / NB) - 1) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      float4 *hi = reinterpret_cast<float4 *>(GL::hi(base, t));
      float4 *lo = reinterpret_cast<float4 *>(GL::hi(base, t) + kTileBytes);
      auto split = [](const float4 &x, float4 &a, float4 &b) {
        const float *xs = &x.x;
        float *as = &a.x, *bs = &b.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float h = __uint_as_float((__float_as_uint(xs[e]) + 0x1000u) & 0xFFFFE000u);
          as[e] = h;
          bs[e] = xs[e] - h;
        }
      };
      if constexpr (RM) {
        // landed: row k at k·256 floats.  Column n's 32 rows go to the 128-byte
        // line n of hi/lo, 16-byte chunk c (rows 4c..4c+3) at c XOR (n mod 8),
        // the 128-byte swizzle TMA would have applied.  A lane loads a 4 × 4
        // block (4 rows of columns n0..n0+3, 16-byte loads) and writes its 4
        // columns' chunk c; lanes split as column quad (lane mod 8) × row group
        // (lane / 8), so that loads and stores both take 4 wavefronts.
        const float *land = reinterpret_cast<const float *>(GL::land(base, s));
        const int cq = lane & 7, rg = lane >> 3;
        for (int blk = warp - 2; blk < kTileN / 32; blk += kConvWarps) {
          const int n0 = blk * 32 + 4 * cq;
#pragma unroll
          for (int pass = 0; pass < 2; ++pass) {
            const int c = rg + 4 * pass;
            float4 r[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) r[q] = *reinterpret_cast<const float4 *>(land + (4 * c + q) * kTileN + n0);
            const float4 col4[4] = {make_float4(r[0].x, r[1].x, r[2].x, r[3].x),
                                    make_float4(r[0].y, r[1].y, r[2].y, r[3].y),
                                    make_float4(r[0].z, r[1].z, r[2].z, r[3].z),
                                    make_float4(r[0].w, r[1].w, r[2].w, r[3].w)};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              float4 a, b;
              split(col4[e], a, b);
              const int n = n0 + e;
              const int q = n * 8 + (c ^ (n & 7));
              hi[q] = a;
              lo[q] = b;
            }
          }
        }
      } else {
        for (int k = threadIdx.x - 64; k < static_cast<int>(kTileBytes / 16); k += 32 * kConvWarps) {
          const float4 x = hi[k];
          float4 a, b;
          split(x, a, b);
          hi[k] = a;
          lo[k] = b;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&conv[t]);
        if (RM) mbar_arrive(&lfree[s]);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: per 8-element K step, hi·hi + hi·lo + lo·hi for both blocks
    constexpr uint32_t id_full = idesc_tf32(128, 256), id_half = idesc_tf32(128, 128);
    for (int kc = 0; kc < nchunks; ++kc) {
      const int t = kc % NB;
      if (!mbar_wait(&conv[t], (kc / NB) & 1)) {
        atomicExch(const_cast<int *>(&failed), 1);
        break;
      }
      tc_fence_after();
      const uint32_t sh = smem_u32(GL::hi(base, t));
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
      umma_commit(&empty[t]);
    }
    umma_commit(done);
  }
  __syncwarp();
  // epilogue: warps 0..3 drain their 32 TMEM lanes each
  const bool ok = mbar_wait(done, 0);
  if (!ok) atomicExch(const_cast<int *>(&failed), 1);
  tc_fence_after();
  __syncthreads();
  if (!failed && warp < 4) { // warp w may read TMEM lanes [32w, 32w + 32) only
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
    for (int s = 0; s < NL; ++s) mbar_wait(&full[s], 0);
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
  const bool rm = h->j_rowmajor;
  // rows of J (a multiple of 32; rows ≥ M are zero) and its stride
  const int64_t rows = rm ? (M + 31) / 32 * 32 : h->ldj;
  const int64_t ld = h->ldj;
  auto enc = encode_fn();
  if (!enc) return set_error(h, FS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  CUtensorMap map;
  CUresult cr;
  const cuuint32_t estr[2] = {1, 1};
  if (rm) { // rows × ld, row-major: a 256-column × 32-row box, columns ≥ D read as zero
    const cuuint64_t gdim[2] = {static_cast<cuuint64_t>(D), static_cast<cuuint64_t>(rows)};
    const cuuint64_t gstride[1] = {static_cast<cuuint64_t>(ld) * sizeof(float)};
    const cuuint32_t box[2] = {kTileN, kKChunk};
    cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->d_J, gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else { // ld × D, column-major
    const cuuint64_t gdim[2] = {static_cast<cuuint64_t>(ld), static_cast<cuuint64_t>(D)};
    const cuuint64_t gstride[1] = {static_cast<cuuint64_t>(ld) * sizeof(float)};
    const cuuint32_t box[2] = {kKChunk, kTileN};
    cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->d_J, gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  if (cr != CUDA_SUCCESS) return set_error(h, FS_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  const int64_t chunks = rows / kKChunk;
  int ncta = static_cast<int>(std::min<int64_t>(148, chunks));
  const int64_t rows_per_cta = (chunks + ncta - 1) / ncta * kKChunk;
  ncta = static_cast<int>((rows + rows_per_cta - 1) / rows_per_cta);
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
  // buffers + 1 KB alignment slack + barriers: 192 KB (column-major), 224 KB (row-major)
  if (rm) {
    const size_t smem = GramLayout<true>::bytes + 1024 + 256;
    FS_CUDA(cudaFuncSetAttribute(gram_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    gram_tc_kernel<true><<<ncta, kThreads, smem, h->stream>>>(map, D, rows_per_cta, rows, h->d_gram_part, h->d_err);
  } else {
    const size_t smem = GramLayout<false>::bytes + 1024 + 256;
    FS_CUDA(cudaFuncSetAttribute(gram_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    gram_tc_kernel<false><<<ncta, kThreads, smem, h->stream>>>(map, D, rows_per_cta, rows, h->d_gram_part, h->d_err);
  }
  FS_CUDA(cudaGetLastError());
  gram_tc_reduce_kernel<<<(D * D + 255) / 256, 256, 0, h->stream>>>(h->d_gram_part, ncta, D, JtJ);
  FS_CUDA(cudaGetLastError());
  h->launches += 2;
  return FS_OK;
}

} // namespace fsg
