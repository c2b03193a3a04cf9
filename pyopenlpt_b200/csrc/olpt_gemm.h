// Tensor-core GEMM of the learned proposal (gemm.cu):
//   D[M x N] = A[M x K] * B[N x K]^T,  A and B bf16 row-major (K contiguous), f32
// accumulation in TMEM, with a fused epilogue applied in this order:
//   v = acc (+ bias[n]) (* gelu'(pre[m][n]));  out_f32 = v;  v = gelu(v) if gelu;
//   out_bf16[m][n] = v;  out_bf16_t[n][m] = v.
// Split-K (splits > 1) writes one f32 partial per split (out_f32 + z * M * ld_f32,
// no bias / activation) for a later reduction.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace olpt {

struct GemmEpilogue {
  const float* bias = nullptr;      // N
  const float* gelu_pre = nullptr;  // M x ld_pre: multiply by gelu'(pre)
  int ld_pre = 0;
  bool gelu = false;
  float* out_f32 = nullptr;
  int ld_f32 = 0;
  __nv_bfloat16* out_bf16 = nullptr;
  int ld_bf16 = 0;
  __nv_bfloat16* out_bf16_t = nullptr;  // N x ld_t
  int ld_t = 0;
};

// A: M rows of K (leading dimension lda elements, a multiple of 8); B: N rows of K.
// err: device flag, nonzero after a wait timed out.
void gemm_bf16(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N,
               int K, const GemmEpilogue& ep, int splits, int* err, cudaStream_t s);

// Device-side GELU (erf form) and its derivative, shared by the MLP kernels.
__device__ __forceinline__ float gelu_f(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad_f(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
         x * 0.39894228040143268f * expf(-0.5f * x * x);
}

}  // namespace olpt
