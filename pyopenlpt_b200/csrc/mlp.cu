// Learned proposal (olpt_mlp.h): feature extraction from the residual images, the
// MLP forward and backward passes on the tensor-core GEMM (gemm.cu), the loss, and
// Adam.  Three hidden layers run as tcgen05 GEMMs with fused bias / GELU / transposed
// epilogues; the 4-wide head, the loss and the reductions are small CUDA-core
// kernels.  All reductions are deterministic (fixed order, no float atomics).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_gemm.h"
#include "olpt_mlp.h"
#include "olpt_otf.cuh"
#include "olpt_shake_dev.cuh"

namespace olpt {

namespace {

inline int nblk(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }
inline int64_t round8(int64_t n) { return (n + 7) / 8 * 8; }

// ---------------------------------------------------------------- weights
__global__ void pack_w1_kernel(const float* w1, int in, int in_pad, __nv_bfloat16* wb1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpHid * in_pad) return;
  const int r = i / in_pad, c = i % in_pad;
  wb1[i] = __float2bfloat16_rn(c < in ? w1[(int64_t)r * in + c] : 0.0f);
}

__global__ void pack_sq_kernel(const float* w, __nv_bfloat16* wb, __nv_bfloat16* wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpHid * kMlpHid) return;
  const int r = i / kMlpHid, c = i % kMlpHid;
  const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
  wb[i] = b;
  wt[(int64_t)c * kMlpHid + r] = b;
}

// ---------------------------------------------------------------- inputs
// f32 rows of `in` values -> bf16 rows of in_pad (zero padded)
__global__ void input_kernel(const float* xin, int64_t n, int in, int in_pad, __nv_bfloat16* x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * in_pad) return;
  const int64_t r = i / in_pad;
  const int c = (int)(i % in_pad);
  x[i] = __float2bfloat16_rn(c < in ? xin[r * in + c] : 0.0f);
}

// out[c][r] = in[r][c] for r < rows, c < cols (32 x 32 tiles through shared memory)
__global__ void transpose_kernel(const __nv_bfloat16* in, int64_t rows, int cols, int ld_in,
                                 __nv_bfloat16* out, int64_t ld_out) {
  __shared__ __nv_bfloat16 t[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t r = r0 + k;
    const int c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[k][threadIdx.x] = in[r * ld_in + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k;
    const int64_t r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(int64_t)c * ld_out + r] = t[threadIdx.x][k];
  }
}

// ---------------------------------------------------------------- head (256 -> 4)
// one warp per row: o = W4 h3 + b4
__global__ void head_fwd_kernel(const __nv_bfloat16* h3, int64_t n, const float* W4,
                                const float* b4, float* o) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  float acc[kMlpOut] = {0, 0, 0, 0};
  for (int k = lane; k < kMlpHid; k += 32) {
    const float h = __bfloat162float(h3[row * kMlpHid + k]);
#pragma unroll
    for (int j = 0; j < kMlpOut; ++j) acc[j] += h * W4[j * kMlpHid + k];
  }
#pragma unroll
  for (int j = 0; j < kMlpOut; ++j) {
    float v = acc[j];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    acc[j] = v;
  }
  if (lane < kMlpOut) o[row * kMlpOut + lane] = acc[lane] + b4[lane];
}

// loss per row: (1 - ghost) * mean_d (o_d - t_d)^2 + w * BCE(o_3, ghost); dout = dL/do / n.
// Per-block partial sums of the loss (double) for a fixed-order reduction.
__global__ void loss_kernel(const float* o, const float* tgt, int64_t n, float w_ghost, float* dout,
                            double* part) {
  __shared__ double red[256];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < n) {
    const float* oi = o + i * kMlpOut;
    const float* ti = tgt + i * kMlpOut;
    const float y = ti[3];
    const float pos = 1.0f - y;
    const float inv_n = 1.0f / (float)n;
    float mse = 0.0f;
    for (int d = 0; d < 3; ++d) {
      const float e = oi[d] - ti[d];
      mse += e * e;
      dout[i * kMlpOut + d] = pos * (2.0f / 3.0f) * e * inv_n;
    }
    const float z = oi[3];
    const float bce = fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)));
    const float p = 1.0f / (1.0f + expf(-z));
    dout[i * kMlpOut + 3] = w_ghost * (p - y) * inv_n;
    l = (double)(pos * mse / 3.0f + w_ghost * bce);
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void sum_double_kernel(const double* part, int n, double* out, double scale) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += part[i];
  *out = s * scale;
}

// dZ3 = (dout W4) * gelu'(z3): 32 rows per block, 256 threads (one per column);
// writes f32 and bf16 rows and the bf16 transpose (ld_t)
__global__ void head_bwd_kernel(const float* dout, const float* W4, const float* z3, int64_t n,
                                float* dzf, __nv_bfloat16* dzb, __nv_bfloat16* dzt, int64_t ld_t) {
  __shared__ __nv_bfloat16 tile[32][kMlpHid + 8];
  const int k = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const float w0 = W4[k], w1 = W4[kMlpHid + k], w2 = W4[2 * kMlpHid + k], w3 = W4[3 * kMlpHid + k];
  for (int rr = 0; rr < 32; ++rr) {
    const int64_t r = r0 + rr;
    if (r >= n) break;
    const float* d = dout + r * kMlpOut;
    const float dh = d[0] * w0 + d[1] * w1 + d[2] * w2 + d[3] * w3;
    const float dz = dh * gelu_grad_f(z3[r * kMlpHid + k]);
    dzf[r * kMlpHid + k] = dz;
    const __nv_bfloat16 b = __float2bfloat16_rn(dz);
    dzb[r * kMlpHid + k] = b;
    tile[rr][k] = b;
  }
  __syncthreads();
  // transpose: thread t writes rows k' = t/32 + 8j of the block, 32 consecutive r
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t r = r0 + lane;
  if (r < n)
    for (int kk = wid; kk < kMlpHid; kk += 8) dzt[(int64_t)kk * ld_t + r] = tile[lane][kk];
}

// partial dW4 (4 x 256) and db4 (4) per block of rows: partial[block][0..1027]
__global__ void head_wgrad_kernel(const float* dout, const __nv_bfloat16* h3, int64_t n,
                                  int64_t rows_per_blk, float* partial) {
  const int k = threadIdx.x;  // 256 threads
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk;
  const int64_t r1 = min(n, r0 + rows_per_blk);
  float a0 = 0, a1 = 0, a2 = 0, a3 = 0, b = 0;
  for (int64_t r = r0; r < r1; ++r) {
    const float h = __bfloat162float(h3[r * kMlpHid + k]);
    const float* d = dout + r * kMlpOut;
    a0 += d[0] * h;
    a1 += d[1] * h;
    a2 += d[2] * h;
    a3 += d[3] * h;
    if (k < kMlpOut) b += d[k];
  }
  float* p = partial + (int64_t)blockIdx.x * (kMlpOut * kMlpHid + kMlpOut);
  p[k] = a0;
  p[kMlpHid + k] = a1;
  p[2 * kMlpHid + k] = a2;
  p[3 * kMlpHid + k] = a3;
  if (k < kMlpOut) p[kMlpOut * kMlpHid + k] = b;
}

// out[i] = sum_p partial[p][i]  (i < len, partial row stride len)
__global__ void sum_partials_kernel(const float* partial, int n_part, int len, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  float s = 0.0f;
  for (int p = 0; p < n_part; ++p) s += partial[(int64_t)p * len + i];
  out[i] = s;
}

// split-K partials [S][M][ld] -> out[m * ld_out + c] for c < N
__global__ void splitk_reduce_kernel(const float* part, int S, int M, int N, int ld, float* out,
                                     int ld_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  const int m = i / N, c = i % N;
  float s = 0.0f;
  for (int z = 0; z < S; ++z) s += part[((int64_t)z * M + m) * ld + c];
  out[(int64_t)m * ld_out + c] = s;
}

// column sums of a [n x 256] f32 matrix (bias gradients): per block of kColRows rows
// a partial row, then sum_partials_kernel; fixed order throughout
constexpr int kColRows = 128;
__global__ void colsum_kernel(const float* a, int64_t n, float* partial) {
  const int k = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * kColRows;
  const int64_t r1 = min(n, r0 + kColRows);
  float s = 0.0f;
#pragma unroll 8
  for (int64_t r = r0; r < r1; ++r) s += a[r * kMlpHid + k];
  partial[(int64_t)blockIdx.x * kMlpHid + k] = s;
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int64_t n, float lr,
                            float b1, float b2, float eps, float bc1, float bc2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// ---------------------------------------------------------------- sampling
__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// mini-batch rows drawn uniformly with replacement from the resident dataset
__global__ void sample_kernel(const float* x, const float* t, int64_t n, int in, int batch,
                              uint64_t seed, int64_t step, float* xb, float* tb) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)batch * in) return;
  const int64_t r = i / in;
  const int c = (int)(i % in);
  const int64_t src = (int64_t)(mix64(seed ^ ((uint64_t)step << 32) ^ (uint64_t)r) % (uint64_t)n);
  xb[i] = x[src * in + c];
  if (c < kMlpOut) tb[r * kMlpOut + c] = t[src * kMlpOut + c];
}

// ---------------------------------------------------------------- features
// the residual planes of every camera, by value
struct PlaneSet {
  PlaneView p[kMlpMaxCams];
};

// one warp per object; lanes 0..C-1 project on their camera and evaluate the OTF there
template <typename Real>
__global__ void features_kernel(const CamDev* cams, OtfView otf, const double* xyz, int64_t n,
                                const PlaneSet planes, int n_cams, int in, int in_pad,
                                double r_px, __nv_bfloat16* x, float* f32) {
  const int64_t o = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (o >= n) return;
  const double X = xyz[3 * o], Y = xyz[3 * o + 1], Z = xyz[3 * o + 2];
  double u = 0, w = 0, q[5] = {0, 0, 0, 1, 0};
  if (lane < n_cams) {
    cam_project(cams[lane], X, Y, Z, u, w);
    otf_param(otf, lane, X, Y, Z, q);
  }
  constexpr int kArea = kMlpArea;
  __nv_bfloat16* xo = x + o * in_pad;
  float* fo = f32 ? f32 + o * in : nullptr;
  for (int c = 0; c < n_cams; ++c) {
    const double uc = __shfl_sync(0xffffffffu, u, c), wc = __shfl_sync(0xffffffffu, w, c);
    Real qc[5];
    for (int k = 0; k < 5; ++k) qc[k] = (Real)__shfl_sync(0xffffffffu, q[k], c);
    const CamDev& cm = cams[c];
    const double ru = round(uc), rw = round(wc);
    const bool finite = isfinite(uc) && isfinite(wc) && fabs(uc) < 1e6 && fabs(wc) < 1e6;
    const int cu = finite ? (int)ru : -100000, cw = finite ? (int)rw : -100000;
    const Rect pr = finite ? roi_bound(cm.n_row, cm.n_col, uc, wc, r_px, r_px) : Rect{1, 0, 1, 0};
    const PlaneView& P = planes.p[c];
    const Real* res = reinterpret_cast<const Real*>(P.p);
    const int64_t rp = P.pitch / (int64_t)sizeof(Real);
    const Real inv_a = (Real)1 / (qc[0] > (Real)1e-6 ? qc[0] : (Real)1e-6);
    for (int t = lane; t < kArea; t += 32) {
      const int row = cw + t / kMlpPatch - kMlpPatch / 2;
      const int col = cu + t % kMlpPatch - kMlpPatch / 2;
      Real val = 0;
      if (row >= 0 && row < cm.n_row && col >= 0 && col < cm.n_col) {
        val = res[(int64_t)row * rp + col];
        if (row >= pr.rmin && row < pr.rmax && col >= pr.cmin && col < pr.cmax)
          val += gauss<Real>(col, row, uc, wc, qc);
        val = val > (Real)0 ? val * inv_a : (Real)0;
      }
      xo[c * kArea + t] = __float2bfloat16_rn((float)val);
      if (fo) fo[c * kArea + t] = (float)val;
    }
    if (lane == 0) {
      const float du = finite ? (float)(uc - ru) : 0.0f, dw = finite ? (float)(wc - rw) : 0.0f;
      const int b = n_cams * kArea + 2 * c;
      xo[b] = __float2bfloat16_rn(du);
      xo[b + 1] = __float2bfloat16_rn(dw);
      if (fo) {
        fo[b] = du;
        fo[b + 1] = dw;
      }
    }
  }
  for (int k = in - 1 + lane; k < in_pad; k += 32) {
    const float val = k == in - 1 ? 1.0f : 0.0f;
    xo[k] = __float2bfloat16_rn(val);
    if (fo && k == in - 1) fo[k] = val;
  }
}

// ---------------------------------------------------------------- host helpers
void ensure_batch(olpt_ctx* ctx, int64_t n, bool training) {
  MlpWork& W = ctx->mlp;
  const MlpDims& D = W.dims;
  cudaStream_t s = ctx->stream;
  const int64_t m = std::max<int64_t>(n, 1);
  const int64_t lt = round8(m);
  const size_t hb = (size_t)m * kMlpHid;
  W.x.ensure((size_t)m * D.in_pad * 2, s);
  W.h1.ensure(hb * 2, s);
  W.h2.ensure(hb * 2, s);
  W.h3.ensure(hb * 2, s);
  W.o.ensure((size_t)m * kMlpOut * 4, s);
  W.err.ensure(16, s);
  if (!training) return;
  W.xin.ensure((size_t)m * D.in * 4, s);
  W.tgt.ensure((size_t)m * kMlpOut * 4, s);
  W.xt.ensure((size_t)D.in_pad * lt * 2, s);
  for (DevBuf* b : {&W.z1, &W.z2, &W.z3, &W.dz1f, &W.dz2f, &W.dz3f}) b->ensure(hb * 4, s);
  for (DevBuf* b : {&W.dz2b, &W.dz3b}) b->ensure(hb * 2, s);
  for (DevBuf* b : {&W.h1t, &W.h2t, &W.dz1t, &W.dz2t, &W.dz3t})
    b->ensure((size_t)kMlpHid * lt * 2, s);
  W.dout.ensure((size_t)m * kMlpOut * 4, s);
  W.loss.ensure((size_t)(nblk(m) + 2) * 8, s);
}

void pack_weights(olpt_ctx* ctx) {
  MlpWork& W = ctx->mlp;
  const MlpDims& D = W.dims;
  cudaStream_t s = ctx->stream;
  const float* M = W.master.as<float>();
  pack_w1_kernel<<<OLPT_G(nblk(kMlpHid * D.in_pad)), 256, 0, s>>>(M + D.off_w1, D.in, D.in_pad,
                                                                  W.wb1.as<__nv_bfloat16>());
  pack_sq_kernel<<<OLPT_G(nblk(kMlpHid * kMlpHid)), 256, 0, s>>>(
      M + D.off_w2, W.wb2.as<__nv_bfloat16>(), W.wt2.as<__nv_bfloat16>());
  pack_sq_kernel<<<OLPT_G(nblk(kMlpHid * kMlpHid)), 256, 0, s>>>(
      M + D.off_w3, W.wb3.as<__nv_bfloat16>(), W.wt3.as<__nv_bfloat16>());
  OLPT_CUDA(cudaGetLastError());
}

void alloc_params(olpt_ctx* ctx) {
  MlpWork& W = ctx->mlp;
  const MlpDims& D = W.dims;
  cudaStream_t s = ctx->stream;
  const size_t pb = (size_t)D.params * 4;
  for (DevBuf* b : {&W.master, &W.grad, &W.am, &W.av}) b->ensure(pb, s);
  W.wb1.ensure((size_t)kMlpHid * D.in_pad * 2, s);
  for (DevBuf* b : {&W.wb2, &W.wb3, &W.wt2, &W.wt3}) b->ensure((size_t)kMlpHid * kMlpHid * 2, s);
  OLPT_CUDA(cudaMemsetAsync(W.am.p, 0, pb, s));
  OLPT_CUDA(cudaMemsetAsync(W.av.p, 0, pb, s));
  OLPT_CUDA(cudaMemsetAsync(W.grad.p, 0, pb, s));
  W.adam_t = 0;
}

int check_err(olpt_ctx* ctx) {
  int e = 0;
  OLPT_CUDA(cudaMemcpyAsync(&e, ctx->mlp.err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  OLPT_REQUIRE(e == 0, OLPT_ERR_TIMEOUT,
               "tensor-core GEMM: a pipeline wait timed out (code " + std::to_string(e) + ")");
  return e;
}

// forward of the three hidden layers; with training, also the f32 pre-activations
// and the transposed activations for the weight gradients
void forward(olpt_ctx* ctx, int64_t n, bool training) {
  MlpWork& W = ctx->mlp;
  const MlpDims& D = W.dims;
  cudaStream_t s = ctx->stream;
  const int lt = (int)round8(n);
  const float* M = W.master.as<float>();
  int* err = W.err.as<int>();
  GemmEpilogue e1;
  e1.bias = M + D.off_b1;
  e1.gelu = true;
  e1.out_bf16 = W.h1.as<__nv_bfloat16>();
  e1.ld_bf16 = kMlpHid;
  if (training) {
    e1.out_f32 = W.z1.as<float>();
    e1.ld_f32 = kMlpHid;
    e1.out_bf16_t = W.h1t.as<__nv_bfloat16>();
    e1.ld_t = lt;
  }
  gemm_bf16(W.x.as<__nv_bfloat16>(), D.in_pad, W.wb1.as<__nv_bfloat16>(), D.in_pad, (int)n,
            kMlpHid, D.in_pad, e1, 1, err, s);
  GemmEpilogue e2 = e1;
  e2.bias = M + D.off_b2;
  e2.out_bf16 = W.h2.as<__nv_bfloat16>();
  if (training) {
    e2.out_f32 = W.z2.as<float>();
    e2.out_bf16_t = W.h2t.as<__nv_bfloat16>();
  }
  gemm_bf16(W.h1.as<__nv_bfloat16>(), kMlpHid, W.wb2.as<__nv_bfloat16>(), kMlpHid, (int)n, kMlpHid,
            kMlpHid, e2, 1, err, s);
  GemmEpilogue e3;
  e3.bias = M + D.off_b3;
  e3.gelu = true;
  e3.out_bf16 = W.h3.as<__nv_bfloat16>();
  e3.ld_bf16 = kMlpHid;
  if (training) {
    e3.out_f32 = W.z3.as<float>();
    e3.ld_f32 = kMlpHid;
  }
  gemm_bf16(W.h2.as<__nv_bfloat16>(), kMlpHid, W.wb3.as<__nv_bfloat16>(), kMlpHid, (int)n, kMlpHid,
            kMlpHid, e3, 1, err, s);
  head_fwd_kernel<<<OLPT_G(nblk(n * 32)), 256, 0, s>>>(W.h3.as<__nv_bfloat16>(), n, M + D.off_w4,
                                                      M + D.off_b4, W.o.as<float>());
  OLPT_CUDA(cudaGetLastError());
}

void bias_grad(olpt_ctx* ctx, const float* dz, int64_t n, float* out) {
  MlpWork& W = ctx->mlp;
  cudaStream_t s = ctx->stream;
  const int nb = (int)((n + kColRows - 1) / kColRows);
  W.hpart.ensure((size_t)nb * kMlpHid * 4 + 64, s);
  colsum_kernel<<<OLPT_G(nb), kMlpHid, 0, s>>>(dz, n, W.hpart.as<float>());
  sum_partials_kernel<<<OLPT_G(1), kMlpHid, 0, s>>>(W.hpart.as<float>(), nb, kMlpHid, out);
  OLPT_CUDA(cudaGetLastError());
}

// weight gradient dW[M x N] = A^T-layout GEMM over the batch (K = n), split-K partials
void wgrad(olpt_ctx* ctx, const __nv_bfloat16* at, const __nv_bfloat16* bt, int64_t n, int Mo,
           int No, int ld_part, float* out, int ld_out, int n_keep) {
  MlpWork& W = ctx->mlp;
  cudaStream_t s = ctx->stream;
  const int lt = (int)round8(n);
  const int tiles = ((Mo + 127) / 128) * ((No + 127) / 128);
  const int kt = (int)((n + 63) / 64);
  const int splits = std::max(1, std::min(kt, 148 / tiles));
  W.part.ensure((size_t)splits * Mo * ld_part * 4 + 64, s);
  GemmEpilogue e;
  e.out_f32 = W.part.as<float>();
  e.ld_f32 = ld_part;
  gemm_bf16(at, lt, bt, lt, Mo, No, (int)n, e, splits, W.err.as<int>(), s);
  // the launcher may merge splits so that none is empty; recompute as it does
  const int kps = (kt + splits - 1) / splits;
  const int S = (kt + kps - 1) / kps;
  splitk_reduce_kernel<<<OLPT_G(nblk((int64_t)Mo * n_keep)), 256, 0, s>>>(
      W.part.as<float>(), S, Mo, n_keep, ld_part, out, ld_out);
  OLPT_CUDA(cudaGetLastError());
}

}  // namespace

// The network's geometry follows the context's camera count (4 when no cameras are
// uploaded yet); buffers are grown when it changes.
void set_dims(olpt_ctx* ctx) {
  MlpWork& W = ctx->mlp;
  const int cams = ctx->n_cam >= 2 ? ctx->n_cam : 4;
  OLPT_REQUIRE(cams <= kMlpMaxCams, OLPT_ERR_UNSUPPORTED,
               "the learned proposal supports at most 8 cameras");
  if (W.dims.cams != cams) {
    W.dims = mlp_dims(cams);
    W.ready = false;
  }
}

void mlp_sync_dims(olpt_ctx* ctx) {
  if (!ctx->mlp.ready) set_dims(ctx);
}

void mlp_init(olpt_ctx* ctx, uint64_t seed) {
  set_dims(ctx);
  alloc_params(ctx);
  const MlpDims& D = ctx->mlp.dims;
  std::vector<float> p(D.params, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int64_t off, int fan_out, int fan_in) {
    const double lim = std::sqrt(6.0 / (double)fan_in);  // He-uniform for GELU layers
    std::uniform_real_distribution<double> U(-lim, lim);
    for (int64_t i = 0; i < (int64_t)fan_out * fan_in; ++i) p[off + i] = (float)U(rng);
  };
  fill(D.off_w1, kMlpHid, D.in);
  fill(D.off_w2, kMlpHid, kMlpHid);
  fill(D.off_w3, kMlpHid, kMlpHid);
  {
    const double lim = std::sqrt(1.0 / (double)kMlpHid);
    std::uniform_real_distribution<double> U(-lim, lim);
    for (int64_t i = 0; i < (int64_t)kMlpOut * kMlpHid; ++i) p[D.off_w4 + i] = (float)U(rng);
  }
  mlp_set_params(ctx, p.data());
}

void mlp_set_params(olpt_ctx* ctx, const float* host) {
  MlpWork& W = ctx->mlp;
  set_dims(ctx);
  if (!W.ready) alloc_params(ctx);
  OLPT_CUDA(cudaMemcpyAsync(W.master.p, host, (size_t)W.dims.params * 4, cudaMemcpyHostToDevice,
                            ctx->stream));
  pack_weights(ctx);
  OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  W.ready = true;
}

void mlp_get_params(olpt_ctx* ctx, float* host) {
  OLPT_REQUIRE(ctx->mlp.ready, OLPT_ERR_INVALID_ARG, "network not initialised");
  OLPT_CUDA(cudaMemcpyAsync(host, ctx->mlp.master.p, (size_t)ctx->mlp.dims.params * 4,
                            cudaMemcpyDeviceToHost, ctx->stream));
  OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
}

void mlp_features_device(olpt_ctx* ctx, const ShakeParams& sp, __nv_bfloat16* x, float* f32) {
  mlp_sync_dims(ctx);
  OLPT_REQUIRE(ctx->n_cam == ctx->mlp.dims.cams, OLPT_ERR_UNSUPPORTED,
               "learned proposal: the network was built for " +
                   std::to_string(ctx->mlp.dims.cams) + " cameras, the rig has " +
                   std::to_string(ctx->n_cam));
  const MlpDims& D = ctx->mlp.dims;
  const int64_t n = ctx->obj.n;
  if (n == 0) return;
  PlaneSet pv{};
  for (int c = 0; c < D.cams; ++c) {
    const ImagePlane& r = ctx->resid[c];
    pv.p[c] = PlaneView{r.buf.as<unsigned char>(), r.pitch, r.H, r.W, r.dtype};
  }
  const OtfView ov = otf_view(ctx);
  cudaStream_t s = ctx->stream;
  if (sp.precision == 1)
    features_kernel<double><<<OLPT_G(nblk(n * 32)), 256, 0, s>>>(
        ctx->cams_d.as<CamDev>(), ov, ctx->obj.xyz.as<double>(), n, pv, D.cams, D.in, D.in_pad,
        sp.radius_obj, x, f32);
  else
    features_kernel<float><<<OLPT_G(nblk(n * 32)), 256, 0, s>>>(
        ctx->cams_d.as<CamDev>(), ov, ctx->obj.xyz.as<double>(), n, pv, D.cams, D.in, D.in_pad,
        sp.radius_obj, x, f32);
  OLPT_CUDA(cudaGetLastError());
}

namespace {
__global__ void gelu_kernel(float* p, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = gelu_f(p[i]);
}
}  // namespace

void gelu_inplace_device(float* p, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  gelu_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(p, n);
  OLPT_CUDA(cudaGetLastError());
}

void mlp_input_device(olpt_ctx* ctx, const float* x_f32, int64_t n, __nv_bfloat16* x) {
  if (n == 0) return;
  const MlpDims& D = ctx->mlp.dims;
  input_kernel<<<OLPT_G(nblk(n * D.in_pad)), 256, 0, ctx->stream>>>(x_f32, n, D.in, D.in_pad, x);
  OLPT_CUDA(cudaGetLastError());
}

void mlp_infer_device(olpt_ctx* ctx, const __nv_bfloat16* x, int64_t n, float* o) {
  MlpWork& W = ctx->mlp;
  OLPT_REQUIRE(W.ready, OLPT_ERR_INVALID_ARG, "network not initialised");
  if (n == 0) return;
  cudaStream_t s = ctx->stream;
  ensure_batch(ctx, n, false);
  OLPT_CUDA(cudaMemsetAsync(W.err.p, 0, 16, s));
  if (x != W.x.as<__nv_bfloat16>())
    OLPT_CUDA(cudaMemcpyAsync(W.x.p, x, (size_t)n * W.dims.in_pad * 2, cudaMemcpyDeviceToDevice,
                              s));
  forward(ctx, n, false);
  if (o != W.o.as<float>())
    OLPT_CUDA(cudaMemcpyAsync(o, W.o.p, (size_t)n * kMlpOut * 4, cudaMemcpyDeviceToDevice, s));
  check_err(ctx);
}

namespace {
// One training step enqueued on the context's stream (no synchronisation); the mean
// loss is left on the device at the returned address.
const double* train_enqueue(olpt_ctx* ctx, const float* x_f32, const float* tgt, int64_t n,
                            double lr, double ghost_weight, bool update);
}  // namespace

double mlp_train_device(olpt_ctx* ctx, const float* x_f32, const float* tgt, int64_t n, double lr,
                        double ghost_weight, bool update) {
  OLPT_REQUIRE(ctx->mlp.ready, OLPT_ERR_INVALID_ARG, "network not initialised");
  OLPT_REQUIRE(n > 0, OLPT_ERR_INVALID_ARG, "empty batch");
  ensure_batch(ctx, n, true);
  OLPT_CUDA(cudaMemsetAsync(ctx->mlp.err.p, 0, 16, ctx->stream));
  const double* d_loss = train_enqueue(ctx, x_f32, tgt, n, lr, ghost_weight, update);
  double loss = 0.0;
  OLPT_CUDA(cudaMemcpyAsync(&loss, d_loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  check_err(ctx);
  return loss;
}

namespace {
const double* train_enqueue(olpt_ctx* ctx, const float* x_f32, const float* tgt, int64_t n,
                            double lr, double ghost_weight, bool update) {
  MlpWork& W = ctx->mlp;
  OLPT_REQUIRE(W.ready, OLPT_ERR_INVALID_ARG, "network not initialised");
  OLPT_REQUIRE(n > 0, OLPT_ERR_INVALID_ARG, "empty batch");
  cudaStream_t s = ctx->stream;
  const MlpDims& D = W.dims;
  ensure_batch(ctx, n, true);
  const int64_t lt = round8(n);
  input_kernel<<<OLPT_G(nblk(n * D.in_pad)), 256, 0, s>>>(x_f32, n, D.in, D.in_pad,
                                                          W.x.as<__nv_bfloat16>());
  {
    dim3 g((unsigned)((n + 31) / 32), D.in_pad / 32);
    transpose_kernel<<<OLPT_G(g), dim3(32, 8), 0, s>>>(W.x.as<__nv_bfloat16>(), n, D.in_pad,
                                                       D.in_pad, W.xt.as<__nv_bfloat16>(), lt);
  }
  forward(ctx, n, true);
  float* G = W.grad.as<float>();
  const float* M = W.master.as<float>();
  // loss and head
  const int lb = nblk(n);
  loss_kernel<<<OLPT_G(lb), 256, 0, s>>>(W.o.as<float>(), tgt, n, (float)ghost_weight,
                                         W.dout.as<float>(), W.loss.as<double>());
  sum_double_kernel<<<OLPT_G(1), 32, 0, s>>>(W.loss.as<double>(), lb, W.loss.as<double>() + lb,
                                             1.0 / (double)n);
  const int64_t rpb = 256;
  const int hb = (int)((n + rpb - 1) / rpb);
  const int hlen = kMlpOut * kMlpHid + kMlpOut;
  W.hpart.ensure((size_t)hb * hlen * 4 + 64, s);
  head_wgrad_kernel<<<OLPT_G(hb), 256, 0, s>>>(W.dout.as<float>(), W.h3.as<__nv_bfloat16>(), n, rpb,
                                               W.hpart.as<float>());
  sum_partials_kernel<<<OLPT_G(nblk(hlen)), 256, 0, s>>>(W.hpart.as<float>(), hb, hlen,
                                                         G + D.off_w4);
  // (hpart is reused by the bias gradients below, after these kernels in stream order)
  head_bwd_kernel<<<OLPT_G((unsigned)((n + 31) / 32)), 256, 0, s>>>(
      W.dout.as<float>(), M + D.off_w4, W.z3.as<float>(), n, W.dz3f.as<float>(), W.dz3b.as<__nv_bfloat16>(),
      W.dz3t.as<__nv_bfloat16>(), lt);
  OLPT_CUDA(cudaGetLastError());
  int* err = W.err.as<int>();
  // layer 3
  wgrad(ctx, W.dz3t.as<__nv_bfloat16>(), W.h2t.as<__nv_bfloat16>(), n, kMlpHid, kMlpHid, kMlpHid,
        G + D.off_w3, kMlpHid, kMlpHid);
  bias_grad(ctx, W.dz3f.as<float>(), n, G + D.off_b3);
  GemmEpilogue d2;
  d2.gelu_pre = W.z2.as<float>();
  d2.ld_pre = kMlpHid;
  d2.out_f32 = W.dz2f.as<float>();
  d2.ld_f32 = kMlpHid;
  d2.out_bf16 = W.dz2b.as<__nv_bfloat16>();
  d2.ld_bf16 = kMlpHid;
  d2.out_bf16_t = W.dz2t.as<__nv_bfloat16>();
  d2.ld_t = (int)lt;
  gemm_bf16(W.dz3b.as<__nv_bfloat16>(), kMlpHid, W.wt3.as<__nv_bfloat16>(), kMlpHid, (int)n,
            kMlpHid, kMlpHid, d2, 1, err, s);
  // layer 2
  wgrad(ctx, W.dz2t.as<__nv_bfloat16>(), W.h1t.as<__nv_bfloat16>(), n, kMlpHid, kMlpHid, kMlpHid,
        G + D.off_w2, kMlpHid, kMlpHid);
  bias_grad(ctx, W.dz2f.as<float>(), n, G + D.off_b2);
  GemmEpilogue d1;
  d1.gelu_pre = W.z1.as<float>();
  d1.ld_pre = kMlpHid;
  d1.out_f32 = W.dz1f.as<float>();
  d1.ld_f32 = kMlpHid;
  d1.out_bf16_t = W.dz1t.as<__nv_bfloat16>();
  d1.ld_t = (int)lt;
  gemm_bf16(W.dz2b.as<__nv_bfloat16>(), kMlpHid, W.wt2.as<__nv_bfloat16>(), kMlpHid, (int)n,
            kMlpHid, kMlpHid, d1, 1, err, s);
  // layer 1
  wgrad(ctx, W.dz1t.as<__nv_bfloat16>(), W.xt.as<__nv_bfloat16>(), n, kMlpHid, D.in_pad,
        D.in_pad, G + D.off_w1, D.in, D.in);
  bias_grad(ctx, W.dz1f.as<float>(), n, G + D.off_b1);
  OLPT_CUDA(cudaGetLastError());
  if (update) {
    ++W.adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - std::pow(b1, (float)W.adam_t);
    const float bc2 = 1.0f - std::pow(b2, (float)W.adam_t);
    adam_kernel<<<OLPT_G(nblk(D.params)), 256, 0, s>>>(W.master.as<float>(), G, W.am.as<float>(),
                                                       W.av.as<float>(), D.params, (float)lr, b1,
                                                       b2, 1e-8f, bc1, bc2);
    OLPT_CUDA(cudaGetLastError());
    pack_weights(ctx);
  }
  return W.loss.as<double>() + lb;
}
}  // namespace

void mlp_train_many(olpt_ctx* ctx, const float* x, const float* t, int64_t n, int batch, int steps,
                    double lr, double ghost_weight, uint64_t seed, float* losses) {
  MlpWork& W = ctx->mlp;
  OLPT_REQUIRE(W.ready, OLPT_ERR_INVALID_ARG, "network not initialised");
  OLPT_REQUIRE(n > 0 && batch > 0 && steps >= 0, OLPT_ERR_INVALID_ARG, "mlp_train: bad sizes");
  cudaStream_t s = ctx->stream;
  const int in = W.dims.in;
  W.xin.ensure((size_t)batch * in * 4, s);
  W.tgt.ensure((size_t)batch * kMlpOut * 4, s);
  // the steps are enqueued back to back; the losses stay on the device until the end
  W.loss_hist.ensure((size_t)(steps + 1) * sizeof(double), s);
  ensure_batch(ctx, batch, true);
  OLPT_CUDA(cudaMemsetAsync(W.err.p, 0, 16, s));
  for (int it = 0; it < steps; ++it) {
    const double a = lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * it / (double)steps)));
    sample_kernel<<<OLPT_G(nblk((int64_t)batch * in)), 256, 0, s>>>(
        x, t, n, in, batch, seed, it, W.xin.as<float>(), W.tgt.as<float>());
    OLPT_CUDA(cudaGetLastError());
    const double* d_loss = train_enqueue(ctx, W.xin.as<float>(), W.tgt.as<float>(), batch, a,
                                         ghost_weight, true);
    OLPT_CUDA(cudaMemcpyAsync(W.loss_hist.as<double>() + it, d_loss, sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
  }
  std::vector<double> h(steps);
  if (steps > 0)
    OLPT_CUDA(cudaMemcpyAsync(h.data(), W.loss_hist.p, (size_t)steps * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  check_err(ctx);
  if (losses)
    for (int it = 0; it < steps; ++it) losses[it] = (float)h[it];
}

}  // namespace olpt
