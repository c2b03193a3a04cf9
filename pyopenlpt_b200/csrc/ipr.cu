// IPR driver: IPR::runIPR + runSingleIPRIteration + limit2DObjectNumber +
// filterOutInvalid (src/srcSTB/IPR.cpp:19-305) over the device kernels.
//
// Everything numerical stays on the device: detection (peaks.cu), stereo matching
// (stereo.cu; only the order-dependent prune runs on the host), shake and
// residual (shake.cu).  Per loop the host reads back a few counts, the candidate
// list for the prune and the compacted object count.  The image of every camera is
// replaced by its residual after each loop, exactly as the reference's by-value
// `images` vector is.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <random>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_scan.cuh"
#include "olpt_shake.h"

namespace olpt {

void find_peaks_device(olpt_ctx* ctx, double min_int, bool sync_counts);

namespace {

inline int nblk(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

__global__ void gather_dets_kernel(const int* perm, int64_t n, const double* x, const double* y,
                                   const int2* rc, double* x2, double* y2, int2* rc2) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = perm[i];
  x2[i] = x[j];
  y2[i] = y[j];
  rc2[i] = rc[j];
}

__global__ void keep_flags_kernel(const uint8_t* flags, int64_t n, int* keep) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) keep[i] = flags[i] == 0 ? 1 : 0;
}

__global__ void append_kept_kernel(const uint8_t* flags, const int* pos, int64_t n, int n_cam,
                                   const double* xyz, const double* uv, int64_t base, double* oxyz,
                                   double* ouv) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || flags[i] != 0) return;
  const int64_t o = base + pos[i];
  for (int k = 0; k < 3; ++k) oxyz[3 * o + k] = xyz[3 * i + k];
  for (int k = 0; k < 2 * n_cam; ++k) ouv[o * 2 * n_cam + k] = uv[i * 2 * n_cam + k];
}

// myMATH::generateCombinations (myMATH.cpp:35-70): lexicographic K-subsets.
void combinations(int N, int K, std::vector<std::vector<int>>& out) {
  out.clear();
  if (K > N) return;
  std::vector<int> c(K);
  std::iota(c.begin(), c.end(), 0);
  while (true) {
    out.push_back(c);
    int i = K - 1;
    while (i >= 0 && c[i] == N - K + i) --i;
    if (i < 0) break;
    ++c[i];
    for (int j = i + 1; j < K; ++j) c[j] = c[j - 1] + 1;
  }
}

void set_active(olpt_ctx* ctx, const std::vector<int>& active) {
  for (int c = 0; c < ctx->n_cam; ++c) {
    ctx->cams_h[c].is_active = active[c];
    OLPT_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(ctx->cams_d.p) + sizeof(CamDev) * c +
                                  offsetof(CamDev, is_active),
                              &ctx->cams_h[c].is_active, sizeof(int), cudaMemcpyHostToDevice,
                              ctx->stream));
  }
}

// limit2DObjectNumber (IPR.cpp:19-38): the same libstdc++ std::shuffle with a fresh
// default_random_engine(1234) shared across the active cameras in order; the
// permutation is applied to the device lists.
void limit_detections(olpt_ctx* ctx, int64_t cap) {
  if (cap <= 0) return;
  bool any = false;
  for (int c = 0; c < ctx->n_cam; ++c)
    if (ctx->cams_h[c].is_active && ctx->det_counts_h[c] > cap) any = true;
  if (!any) return;
  std::default_random_engine rng(1234);
  for (int c = 0; c < ctx->n_cam; ++c) {
    if (!ctx->cams_h[c].is_active) continue;
    const int64_t n = ctx->det_counts_h[c];
    if (n <= cap) continue;
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    cudaStream_t s = ctx->stream;
    IprWork& W = ctx->ipr;
    W.perm.ensure(cap * sizeof(int), s);
    W.tx.ensure(cap * sizeof(double), s);
    W.ty.ensure(cap * sizeof(double), s);
    W.trc.ensure(cap * sizeof(int2), s);
    OLPT_CUDA(cudaMemcpyAsync(W.perm.p, perm.data(), cap * sizeof(int), cudaMemcpyHostToDevice, s));
    Dets& d = ctx->dets[c];
    gather_dets_kernel<<<OLPT_G(nblk(cap)), 256, 0, s>>>(W.perm.as<int>(), cap, d.x.as<double>(),
                                                 d.y.as<double>(), d.rc.as<int2>(), W.tx.as<double>(),
                                                 W.ty.as<double>(), W.trc.as<int2>());
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(d.x.p, W.tx.p, cap * sizeof(double), cudaMemcpyDeviceToDevice, s));
    OLPT_CUDA(cudaMemcpyAsync(d.y.p, W.ty.p, cap * sizeof(double), cudaMemcpyDeviceToDevice, s));
    OLPT_CUDA(cudaMemcpyAsync(d.rc.p, W.trc.p, cap * sizeof(int2), cudaMemcpyDeviceToDevice, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    ctx->det_counts_h[c] = cap;
  }
  OLPT_CUDA(cudaMemcpyAsync(ctx->det_counts.p, ctx->det_counts_h.data(),
                            ctx->n_cam * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
}

void append_result(olpt_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  IprWork& W = ctx->ipr;
  const int64_t n = ctx->obj.n;
  const int C = ctx->n_cam;
  if (n <= 0) return;
  W.keep.ensure((n + 1) * sizeof(int), s);
  W.pos.ensure((n + 1) * sizeof(int), s);
  keep_flags_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.flags.as<uint8_t>(), n, W.keep.as<int>());
  exclusive_scan(W.keep.as<int>(), (int)n, W.pos.as<int>(), W.scan_tmp, s);
  int kept = 0;
  OLPT_CUDA(cudaMemcpyAsync(&kept, W.pos.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  const int64_t need = W.n_out + kept;
  if (need > W.cap_out) {
    // grow, keeping what is there
    const int64_t cap = std::max<int64_t>(need * 2, 1024);
    DevBuf nx, nuv;
    nx.ensure(cap * 3 * sizeof(double), s);
    nuv.ensure(cap * C * 2 * sizeof(double), s);
    if (W.n_out > 0) {
      OLPT_CUDA(cudaMemcpyAsync(nx.p, W.out_xyz.p, W.n_out * 3 * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
      OLPT_CUDA(cudaMemcpyAsync(nuv.p, W.out_uv.p, W.n_out * C * 2 * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
    }
    W.out_xyz.release(s);
    W.out_uv.release(s);
    W.out_xyz = nx;
    W.out_uv = nuv;
    nx.p = nuv.p = nullptr;
    W.cap_out = cap;
  }
  append_kept_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.flags.as<uint8_t>(), W.pos.as<int>(), n, C,
                                             ctx->obj.xyz.as<double>(), ctx->obj.uv.as<double>(),
                                             W.n_out, W.out_xyz.as<double>(),
                                             W.out_uv.as<double>());
  OLPT_CUDA(cudaGetLastError());
  W.n_out = need;
}

// runSingleIPRIteration (IPR.cpp:69-192)
void single_iteration(olpt_ctx* ctx, const IprParams& p, const SmParams& sm) {
  {
    PhaseTimer pt(ctx->prof, PH_DETECT);
    find_peaks_device(ctx, p.min_obj_int, true);
    limit_detections(ctx, p.n_obj2d_process_max);
  }
  StereoResult& r = ctx->sm_result;
  {
    PhaseTimer pt(ctx->prof, PH_STEREO);
    stereo_match_device(ctx, sm, r);
  }
  if (stereo_objects(ctx, r) == 0) return;
  {
    PhaseTimer pt(ctx->prof, PH_SHAKE);
    if (ctx->mlp.lp.enable)
      learned_shake_device(ctx, p.shake);
    else
      shake_device(ctx, p.shake);
    if (ctx->prof.on) OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  PhaseTimer pt(ctx->prof, PH_OUTPUT);
  append_result(ctx);
  residual_device(ctx, p.shake, true, true);  // filtered objects only; becomes the image
  if (ctx->prof.on) OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace

void ipr_device(olpt_ctx* ctx, const IprParams& p) {
  IprWork& W = ctx->ipr;
  W.n_out = 0;
  const int n_cam = ctx->n_cam;
  if (n_cam < 2) return;
  std::vector<int> all(n_cam, 1);
  set_active(ctx, all);
  const int max_drop = std::min(p.n_cam_reduced, std::max(0, n_cam - 2));
  const int orig_mcc = p.sm.match_cam_count;
  for (int drop = 0; drop <= max_drop; ++drop) {
    const int K = n_cam - drop;
    std::vector<std::vector<int>> subsets;
    combinations(n_cam, K, subsets);
    const int loops = (drop == 0) ? p.n_loop_ipr : p.n_loop_ipr_reduced;
    SmParams sm = p.sm;
    sm.match_cam_count = std::min(orig_mcc, K);
    for (const auto& ids : subsets) {
      std::vector<int> act(n_cam, 0);
      for (int c : ids) act[c] = 1;
      set_active(ctx, act);
      const double tol_orig = sm.tol_2d_px;
      for (int loop = 0; loop < loops; ++loop) {
        single_iteration(ctx, p, sm);
        sm.tol_2d_px = sm.tol_2d_px * 1.5;
      }
      sm.tol_2d_px = tol_orig;
    }
  }
  set_active(ctx, all);
  OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace olpt
