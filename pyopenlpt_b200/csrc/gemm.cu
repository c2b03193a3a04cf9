// Tensor-core GEMM for the learned proposal's MLP (olpt_gemm.h): one CTA per
// 128 x BN output tile, TMA-fed 4-stage shared-memory ring, tcgen05 MMAs issued by
// one thread into a TMEM accumulator, and a fused epilogue by all eight warps (warp w
// owns TMEM lanes 32 (w % 4) .. + 31 = tile rows, and half of the tile's columns).
//
//   warp 0, lane 0: TMA producer (A tile 128 x 64, B tile BN x 64 per stage)
//   warp 1, lane 0: MMA issuer (4 x K=16 MMAs per stage, commit frees the stage)
//   all 8 warps:    epilogue after the final commit (vector stores for full chunks)
//
// Every mbarrier wait is bounded (umma::kWaitLimitNs); a timeout sets *err and the
// CTA still drains its MMAs and frees its TMEM before returning.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "olpt_ctx.cuh"
#include "olpt_gemm.h"
#include "olpt_umma.cuh"

namespace olpt {
namespace {

constexpr int kBM = 128, kBK = 64, kStages = 4;

struct EpiArgs {
  int M, N;
  GemmEpilogue e;
  int* err;
  int kt_per_split;
  int K;
  int splits;
};

template <int BN>
constexpr size_t smem_bytes() {
  return (size_t)kStages * (kBM + BN) * kBK * 2 + 1024 + 256;
}

template <int BN>
__global__ void __launch_bounds__(256, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     EpiArgs g) {
  using namespace umma;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t kABytes = kBM * kBK * 2, kBBytes = BN * kBK * 2;
  constexpr uint32_t kStageBytes = kABytes + kBBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* done = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int KT = (g.K + kBK - 1) / kBK;
  const int kt0 = blockIdx.z * g.kt_per_split;
  const int nk = max(0, min(KT, kt0 + g.kt_per_split) - kt0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(tmem_slot, BN);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    for (int i = 0; i < nk; ++i) {
      const int s = i % kStages;
      const uint32_t ph = (uint32_t)(i / kStages) & 1u;
      if (i >= kStages && !mbar_wait(&empty[s], ph ^ 1u)) {
        atomicOr(g.err, 1);
        break;
      }
      mbar_arrive_expect_tx(&full[s], kStageBytes);
      tma_load_2d(smem + s * kStageBytes, &tmA, &full[s], (kt0 + i) * kBK, m0);
      tma_load_2d(smem + s * kStageBytes + kABytes, &tmB, &full[s], (kt0 + i) * kBK, n0);
    }
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = idesc_bf16(kBM, BN);
    for (int i = 0; i < nk; ++i) {
      const int s = i % kStages;
      const uint32_t ph = (uint32_t)(i / kStages) & 1u;
      if (!mbar_wait(&full[s], ph)) {
        atomicOr(g.err, 2);
        break;
      }
      fence_after_sync();
      const uint64_t ad = sw128_desc(smem_u32(smem + s * kStageBytes));
      const uint64_t bd = sw128_desc(smem_u32(smem + s * kStageBytes + kABytes));
#pragma unroll
      for (int k = 0; k < kBK / 16; ++k)
        mma_bf16(tmem, ad + 2 * k, bd + 2 * k, idesc, (i > 0 || k > 0) ? 1u : 0u);
      mma_commit(&empty[s]);
    }
    mma_commit(done);  // also after an early exit: drains what was issued
  }
  __syncwarp();

  bool have = nk > 0;
  if (have && !mbar_wait(done, 0)) {
    atomicOr(g.err, 4);
    have = false;
  }
  fence_after_sync();

  // warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows); warps 0-3 take the first
  // half of the tile's columns, warps 4-7 the second
  const int quarter = warp & 3, half = warp >> 2;
  const int row = m0 + quarter * 32 + lane;
  const bool row_ok = row < g.M;
  const GemmEpilogue& e = g.e;
  const bool partial = g.splits > 1;
  for (int c = half * (BN / 2); c < (half + 1) * (BN / 2); c += 16) {
    float v[16];
    if (have) {
      tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c, v);
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = 0.0f;
    }
    if (!row_ok || n0 + c >= g.N) continue;
    const int nb = n0 + c;
    const int nv = min(16, g.N - nb);
    if (partial) {
      float* o = e.out_f32 + (size_t)blockIdx.z * g.M * e.ld_f32 + (size_t)row * e.ld_f32 + nb;
      if (nv == 16 && ((uintptr_t)o & 15) == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          reinterpret_cast<float4*>(o)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2],
                                                        v[4 * q + 3]);
      } else {
        for (int j = 0; j < nv; ++j) o[j] = v[j];
      }
      continue;
    }
    if (nv == 16) {
      // full chunk: vector loads and stores where the addresses allow
      if (e.bias) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] += e.bias[nb + j];
      }
      if (e.gelu_pre) {
        const float* pp = e.gelu_pre + (size_t)row * e.ld_pre + nb;
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] *= gelu_grad_f(pp[j]);
      }
      if (e.out_f32) {
        float* o = e.out_f32 + (size_t)row * e.ld_f32 + nb;
        if (((uintptr_t)o & 15) == 0) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            reinterpret_cast<float4*>(o)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2],
                                                          v[4 * q + 3]);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) o[j] = v[j];
        }
      }
      if (e.gelu) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = gelu_f(v[j]);
      }
      if (e.out_bf16) {
        __nv_bfloat16* o = e.out_bf16 + (size_t)row * e.ld_bf16 + nb;
        if (((uintptr_t)o & 15) == 0) {
          uint32_t w[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
            w[q] = *reinterpret_cast<const uint32_t*>(&b2);
          }
          reinterpret_cast<uint4*>(o)[0] = make_uint4(w[0], w[1], w[2], w[3]);
          reinterpret_cast<uint4*>(o)[1] = make_uint4(w[4], w[5], w[6], w[7]);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) o[j] = __float2bfloat16_rn(v[j]);
        }
      }
      if (e.out_bf16_t) {
#pragma unroll
        for (int j = 0; j < 16; ++j)
          e.out_bf16_t[(size_t)(nb + j) * e.ld_t + row] = __float2bfloat16_rn(v[j]);
      }
      continue;
    }
    for (int j = 0; j < nv; ++j) {
      const int n = nb + j;
      float x = v[j];
      if (e.bias) x += e.bias[n];
      if (e.gelu_pre) x *= gelu_grad_f(e.gelu_pre[(size_t)row * e.ld_pre + n]);
      if (e.out_f32) e.out_f32[(size_t)row * e.ld_f32 + n] = x;
      if (e.gelu) x = gelu_f(x);
      if (e.out_bf16) e.out_bf16[(size_t)row * e.ld_bf16 + n] = __float2bfloat16_rn(x);
      if (e.out_bf16_t) e.out_bf16_t[(size_t)n * e.ld_t + row] = __float2bfloat16_rn(x);
    }
  }

  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, BN);
}

// rows x cols bf16 (row stride ld elements), box box_rows x 64, 128-byte swizzle
CUtensorMap tile_map(const __nv_bfloat16* base, int rows, int cols, int ld, int box_rows) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides,
                                 box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  OLPT_REQUIRE(r == CUDA_SUCCESS, OLPT_ERR_CUDA,
               "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

template <int BN>
void launch(const CUtensorMap& ta, const CUtensorMap& tb, const EpiArgs& g, dim3 grid,
            cudaStream_t s) {
  OLPT_CUDA(cudaFuncSetAttribute(gemm_bf16_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes<BN>()));
  gemm_bf16_kernel<BN><<<OLPT_G(grid), 256, smem_bytes<BN>(), s>>>(ta, tb, g);
  OLPT_CUDA(cudaGetLastError());
}

}  // namespace

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  // thread-safe one-time lookup (contexts may run on several host threads)
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    OLPT_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    OLPT_REQUIRE(q == cudaDriverEntryPointSuccess && p, OLPT_ERR_CUDA,
                 "cuTensorMapEncodeTiled is not available");
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

void gemm_bf16(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N,
               int K, const GemmEpilogue& ep, int splits, int* err, cudaStream_t s) {
  OLPT_REQUIRE(M > 0 && N > 0 && K > 0, OLPT_ERR_INVALID_ARG, "gemm: empty shape");
  OLPT_REQUIRE(lda % 8 == 0 && ldb % 8 == 0 && lda >= K && ldb >= K, OLPT_ERR_INVALID_ARG,
               "gemm: leading dimensions must be multiples of 8 elements and >= K");
  OLPT_REQUIRE(((uintptr_t)A % 16) == 0 && ((uintptr_t)B % 16) == 0, OLPT_ERR_INVALID_ARG,
               "gemm: operands must be 16-byte aligned");
  const int KT = (K + kBK - 1) / kBK;
  splits = std::max(1, std::min(splits, KT));
  const int kps = (KT + splits - 1) / splits;
  splits = (KT + kps - 1) / kps;  // every split has at least one k tile
  OLPT_REQUIRE(splits == 1 || ep.out_f32, OLPT_ERR_INVALID_ARG, "gemm: split-K needs out_f32");
  EpiArgs g{M, N, ep, err, kps, K, splits};
  const int mt = (M + kBM - 1) / kBM;
  // the wide tile when it still gives a full wave of CTAs
  const bool wide = N > 128 && (int64_t)mt * ((N + 255) / 256) * splits >= 148;
  const CUtensorMap ta = tile_map(A, M, K, lda, kBM);
  if (wide) {
    const CUtensorMap tb = tile_map(B, N, K, ldb, 256);
    launch<256>(ta, tb, g, dim3(mt, (N + 255) / 256, splits), s);
  } else {
    const CUtensorMap tb = tile_map(B, N, K, ldb, 128);
    launch<128>(ta, tb, g, dim3(mt, (N + 127) / 128, splits), s);
  }
}

}  // namespace olpt
