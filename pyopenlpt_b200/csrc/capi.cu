// C ABI entry points: context, cameras, OTF, images, geometry helpers, detections.
// Declarations and reference citations: include/olpt.h.
#include <cuda_runtime.h>

#include <cstring>

#include <algorithm>

#include <cmath>
#include <new>
#include <string>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_gemm.h"
#include "olpt_otf.cuh"

namespace olpt {
std::atomic<long long> g_launches{0};
void find_peaks_device(olpt_ctx* ctx, double min_int, bool sync_counts);
void ensure_det_capacity(olpt_ctx* ctx, int cam, int64_t cap);

template <class F>
olpt_status_t guard(olpt_ctx* ctx, F&& f) {
  if (!ctx) return OLPT_ERR_INVALID_ARG;
  try {
    OLPT_CUDA(cudaSetDevice(ctx->device));
    f();
    ctx->err.clear();
    return OLPT_OK;
  } catch (ApiError const& e) {
    ctx->err = e.msg;
    return e.code;
  } catch (CudaError const& e) {
    ctx->err = std::string(cudaGetErrorString(e.code)) + " (" + e.where + ")";
    // a non-sticky error also stays recorded as the runtime's last error: clear it,
    // or the next call's launch check would report it again
    cudaGetLastError();
    return e.code == cudaErrorMemoryAllocation ? OLPT_ERR_OOM : OLPT_ERR_CUDA;
  } catch (std::bad_alloc const&) {
    ctx->err = "host allocation failed";
    return OLPT_ERR_OOM;
  } catch (std::exception const& e) {
    ctx->err = e.what();
    return OLPT_ERR_INTERNAL;
  }
}

namespace {

__global__ void project_kernel(const CamDev* cams, int cam, int64_t n, const double* xyz,
                               double* uv) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double u, v;
  cam_project(cams[cam], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], u, v);
  uv[2 * i] = u;
  uv[2 * i + 1] = v;
}

__global__ void los_kernel(const CamDev* cams, int cam, int64_t n, const double* uv,
                           double* line6) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  Line3 L;
  cam_los(cams[cam], uv[2 * i], uv[2 * i + 1], L);
  for (int k = 0; k < 3; ++k) {
    line6[6 * i + k] = L.p[k];
    line6[6 * i + 3 + k] = L.u[k];
  }
}

__global__ void triangulate_kernel(int64_t n, int k, const double* lines6, double* out4,
                                   int* ok) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  Line3 Ls[OLPT_MAX_CAM];
  const Line3* P[OLPT_MAX_CAM];
  for (int j = 0; j < k; ++j) {
    for (int q = 0; q < 3; ++q) {
      Ls[j].p[q] = lines6[(i * k + j) * 6 + q];
      Ls[j].u[q] = lines6[(i * k + j) * 6 + 3 + q];
    }
    P[j] = &Ls[j];
  }
  double X[3], err = 0;
  bool good = triangulate<OLPT_MAX_CAM>(P, k, X, err);
  out4[4 * i] = X[0];
  out4[4 * i + 1] = X[1];
  out4[4 * i + 2] = X[2];
  out4[4 * i + 3] = err;
  ok[i] = good ? 1 : 0;
}

template <typename T>
__global__ void convert_plane_kernel(const unsigned char* src, int64_t pitch, int H, int W,
                                     int src_dtype, T* dst) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)H * W) return;
  int r = (int)(i / W), c = (int)(i % W);
  const unsigned char* row = src + (int64_t)r * pitch;
  double v;
  switch (src_dtype) {
    case OLPT_U8: v = row[c]; break;
    case OLPT_U16: v = reinterpret_cast<const uint16_t*>(row)[c]; break;
    case OLPT_F32: v = reinterpret_cast<const float*>(row)[c]; break;
    default: v = reinterpret_cast<const double*>(row)[c]; break;
  }
  dst[i] = (T)v;
}

int esize(int dtype) {
  return dtype == OLPT_U8 ? 1 : dtype == OLPT_U16 ? 2 : dtype == OLPT_F32 ? 4 : 8;
}

inline int nblk(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

__global__ void otf_param_kernel(OtfView o, int cam, int64_t n, const double* xyz, double* out5) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double r[5];
  otf_param(o, cam, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], r);
  for (int k = 0; k < 5; ++k) out5[5 * i + k] = r[k];
}

}  // namespace

void ensure_plane(olpt_ctx* ctx, int c, int dtype, int H, int W) {
  ImagePlane& im = ctx->img[c];
  const int64_t pitch = ((int64_t)W * esize(dtype) + 15) / 16 * 16;
  im.buf.ensure((size_t)pitch * H + 64, ctx->stream);
  im.dtype = dtype;
  im.H = H;
  im.W = W;
  im.pitch = pitch;
}

OtfView otf_view(olpt_ctx* ctx) {
  OLPT_REQUIRE(ctx->otf_table.p, OLPT_ERR_INVALID_ARG, "no OTF uploaded");
  OtfView v;
  v.nx = ctx->otf.nx;
  v.ny = ctx->otf.ny;
  v.nz = ctx->otf.nz;
  v.n_grid = ctx->otf.n_grid;
  v.n_cam = ctx->n_cam;
  for (int k = 0; k < 3; ++k) {
    v.bmin[k] = ctx->otf.bmin[k];
    v.bmax[k] = ctx->otf.bmax[k];
    v.d[k] = ctx->otf.d[k];
  }
  v.table = ctx->otf_table.as<double>();
  v.alpha_zero = ctx->otf.alpha_zero;
  return v;
}

}  // namespace olpt

using namespace olpt;

extern "C" {

olpt_status_t olpt_ctx_create(olpt_ctx** out, int device) {
  if (!out) return OLPT_ERR_INVALID_ARG;
  *out = nullptr;
  olpt_ctx* ctx = new (std::nothrow) olpt_ctx();
  if (!ctx) return OLPT_ERR_OOM;
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return OLPT_ERR_CUDA;
  }
  ctx->own_stream = true;
  *out = ctx;
  return OLPT_OK;
}

void olpt_ctx_destroy(olpt_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->cams_d.release(ctx->stream);
  ctx->otf_table.release(ctx->stream);
  for (int c = 0; c < OLPT_MAX_CAM; ++c) {
    ctx->img[c].buf.release(ctx->stream);
    ctx->dets[c].x.release(ctx->stream);
    ctx->dets[c].y.release(ctx->stream);
    ctx->dets[c].rc.release(ctx->stream);
  }
  ctx->det_counts.release(ctx->stream);
  ctx->band_counts.release(ctx->stream);
  ctx->band_offsets.release(ctx->stream);
  ctx->lut_u8.release(ctx->stream);
  ctx->lut_u16.release(ctx->stream);
  ctx->scratch.release(ctx->stream);
  ctx->sm.release(ctx->stream);
  ctx->obj.release(ctx->stream);
  ctx->shk.release(ctx->stream);
  ctx->ipr.release(ctx->stream);
  for (int c = 0; c < OLPT_MAX_CAM; ++c) ctx->resid[c].buf.release(ctx->stream);
  ctx->stb.w.release(ctx->stream);
  for (int c = 0; c < OLPT_MAX_CAM; ++c) ctx->stb.frame_img[c].buf.release(ctx->stream);
  ctx->prune.release(ctx->stream);
  ctx->mlp.release(ctx->stream);
  ctx->tio.writer.stop();  // writes what is still queued
  ctx->tio.release(ctx->stream);
  ctx->prof.release();
  cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* olpt_last_error(const olpt_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

olpt_status_t olpt_sync(olpt_ctx* ctx) {
  return guard(ctx, [&] { OLPT_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

olpt_status_t olpt_stream(olpt_ctx* ctx, void** stream) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(stream, OLPT_ERR_INVALID_ARG, "null output");
    *stream = (void*)ctx->stream;
  });
}

int64_t olpt_launch_count(void) { return (int64_t)g_launches.load(); }

olpt_status_t olpt_profile(olpt_ctx* ctx, int enable) {
  return guard(ctx, [&] { ctx->prof.on = enable != 0; });
}

olpt_status_t olpt_profile_read(olpt_ctx* ctx, int kernel, double* total_ms, int64_t* launches,
                                double* bytes) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(kernel >= 0 && kernel < PROF_N + PH_N, OLPT_ERR_INVALID_ARG, "bad kernel id");
    double ms, b = 0;
    long long n;
    if (kernel < PROF_N)
      ctx->prof.read(kernel, ms, n, b);
    else
      ctx->prof.read_phase(kernel - PROF_N, ms, n);
    if (total_ms) *total_ms = ms;
    if (launches) *launches = n;
    if (bytes) *bytes = b;
  });
}

olpt_status_t olpt_cameras_upload(olpt_ctx* ctx, const olpt_camera_desc* cams, int n_cam) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cams && n_cam >= 1 && n_cam <= OLPT_MAX_CAM, OLPT_ERR_INVALID_ARG,
                 "n_cam must be in [1, 8]");
    std::vector<CamDev> h(n_cam);
    for (int i = 0; i < n_cam; ++i) {
      const olpt_camera_desc& d = cams[i];
      CamDev& c = h[i];
      std::memset(&c, 0, sizeof(CamDev));
      c.type = d.type;
      c.n_row = d.n_row;
      c.n_col = d.n_col;
      c.is_active = d.is_active;
      OLPT_REQUIRE(d.type == CAM_PINHOLE || d.type == CAM_POLYNOMIAL, OLPT_ERR_UNSUPPORTED,
                   "camera type must be PINHOLE (0) or POLYNOMIAL (1)");
      if (d.type == CAM_PINHOLE) {
        c.fx = d.cam_mtx[0];
        c.fy = d.cam_mtx[4];
        c.cx = d.cam_mtx[2];
        c.cy = d.cam_mtx[5];
        OLPT_REQUIRE(d.n_dist >= 0 && d.n_dist <= 12, OLPT_ERR_INVALID_ARG, "n_dist > 12");
        // Camera.cpp:55-80: distorted iff some coefficient > SMALLNUMBER
        bool dist = false;
        for (int k = 0; k < d.n_dist; ++k) {
          c.dist[k] = d.dist[k];
          if (d.dist[k] > 1e-8) dist = true;
        }
        c.is_distorted = dist ? 1 : 0;
        c.n_dist = dist ? d.n_dist : 0;
        OLPT_REQUIRE(!dist || d.n_dist == 4 || d.n_dist == 5 || d.n_dist == 8 || d.n_dist == 12,
                     OLPT_ERR_INVALID_ARG, "number of distortion coefficients must be 4/5/8/12");
        for (int k = 0; k < 9; ++k) {
          c.R[k] = d.r_mtx[k];
          c.Rinv[k] = d.r_inv[k];
        }
        for (int k = 0; k < 3; ++k) {
          c.T[k] = d.t_vec[k];
          c.Tinv[k] = d.t_inv[k];
        }
      } else {
        OLPT_REQUIRE(d.n_coeff >= 1 && d.n_coeff <= OLPT_MAX_POLY && d.u_coeffs && d.v_coeffs,
                     OLPT_ERR_INVALID_ARG, "polynomial camera needs 1..32 coefficients");
        OLPT_REQUIRE(d.ref_plane >= 1 && d.ref_plane <= 3, OLPT_ERR_INVALID_ARG,
                     "reference plane must be REF_X/REF_Y/REF_Z");
        c.ref_plane = d.ref_plane;
        c.plane[0] = d.plane[0];
        c.plane[1] = d.plane[1];
        const int n = c.n_coeff = d.n_coeff;
        for (int k = 0; k < 4 * n; ++k) {
          c.ucoef[k] = d.u_coeffs[k];
          c.vcoef[k] = d.v_coeffs[k];
        }
        // Camera::updatePolyDuDv (Camera.cpp:340-393)
        int d0 = 1, d1 = 2;
        if (c.ref_plane == 1) {
          d0 = 2;
          d1 = 3;
        } else if (c.ref_plane == 2) {
          d0 = 1;
          d1 = 3;
        }
        const int rp = c.ref_plane;
        for (int i2 = 0; i2 < n; ++i2) {
          const double* U = &c.ucoef[4 * i2];
          const double* V = &c.vcoef[4 * i2];
          double* DU = &c.ducoef[4 * i2];
          double* DV = &c.dvcoef[4 * i2];
          double* DU2 = &c.ducoef[4 * (i2 + n)];
          double* DV2 = &c.dvcoef[4 * (i2 + n)];
          DU[0] = U[0] * U[d0];
          DU[rp] = U[rp];
          DU[d0] = std::max(U[d0] - 1, 0.0);
          DU[d1] = U[d1];
          DU2[0] = U[0] * U[d1];
          DU2[rp] = U[rp];
          DU2[d0] = U[d0];
          DU2[d1] = std::max(U[d1] - 1, 0.0);
          DV[0] = V[0] * V[d0];
          DV[rp] = V[rp];
          DV[d0] = std::max(V[d0] - 1, 0.0);
          DV[d1] = V[d1];
          DV2[0] = V[0] * V[d1];
          DV2[rp] = V[rp];
          DV2[d0] = V[d0];
          DV2[d1] = std::max(V[d1] - 1, 0.0);
        }
        // exponents all in {0, 1, 2, 3}: the device evaluates the powers once per point
        auto small = [](double e) { return e == 0.0 || e == 1.0 || e == 2.0 || e == 3.0; };
        c.pow3 = 1;
        for (int i2 = 0; i2 < n; ++i2)
          for (int j = 1; j < 4; ++j)
            if (!small(c.ucoef[4 * i2 + j]) || !small(c.vcoef[4 * i2 + j]) ||
                !small(c.ducoef[4 * i2 + j]) || !small(c.dvcoef[4 * i2 + j]) ||
                !small(c.ducoef[4 * (i2 + n) + j]) || !small(c.dvcoef[4 * (i2 + n) + j]))
              c.pow3 = 0;
      }
    }
    ctx->cams_h = h;
    ctx->n_cam = n_cam;
    ctx->cams_d.ensure(sizeof(CamDev) * OLPT_MAX_CAM, ctx->stream);
    OLPT_CUDA(cudaMemcpyAsync(ctx->cams_d.p, h.data(), sizeof(CamDev) * n_cam,
                              cudaMemcpyHostToDevice, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_cameras_set_active(olpt_ctx* ctx, const int* active) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(active && ctx->n_cam > 0, OLPT_ERR_INVALID_ARG, "no cameras");
    for (int c = 0; c < ctx->n_cam; ++c) {
      ctx->cams_h[c].is_active = active[c] ? 1 : 0;
      OLPT_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(ctx->cams_d.p) + sizeof(CamDev) * c +
                                    offsetof(CamDev, is_active),
                                &ctx->cams_h[c].is_active, sizeof(int), cudaMemcpyHostToDevice,
                                ctx->stream));
    }
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_camera_project(olpt_ctx* ctx, int cam, int64_t n, const double* xyz,
                                  double* uv) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cam >= 0 && cam < ctx->n_cam && n >= 0 && (n == 0 || (xyz && uv)),
                 OLPT_ERR_INVALID_ARG, "bad camera index or buffers");
    if (n == 0) return;
    ctx->scratch.ensure(n * 5 * sizeof(double), ctx->stream);
    double* dx = ctx->scratch.as<double>();
    double* du = dx + 3 * n;
    OLPT_CUDA(cudaMemcpyAsync(dx, xyz, n * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    project_kernel<<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(ctx->cams_d.as<CamDev>(), cam, n, dx, du);
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(uv, du, n * 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_camera_los(olpt_ctx* ctx, int cam, int64_t n, const double* uv,
                              double* line6) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cam >= 0 && cam < ctx->n_cam && n >= 0 && (n == 0 || (uv && line6)),
                 OLPT_ERR_INVALID_ARG, "bad camera index or buffers");
    if (n == 0) return;
    ctx->scratch.ensure(n * 8 * sizeof(double), ctx->stream);
    double* du = ctx->scratch.as<double>();
    double* dl = du + 2 * n;
    OLPT_CUDA(cudaMemcpyAsync(du, uv, n * 2 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    los_kernel<<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(ctx->cams_d.as<CamDev>(), cam, n, du, dl);
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(line6, dl, n * 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_triangulate(olpt_ctx* ctx, int64_t n_sets, int k, const double* lines6,
                               double* out4, int* ok) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(k >= 2 && k <= OLPT_MAX_CAM && n_sets >= 0, OLPT_ERR_INVALID_ARG,
                 "k must be in [2, 8]");
    if (n_sets == 0) return;
    OLPT_REQUIRE(lines6 && out4 && ok, OLPT_ERR_INVALID_ARG, "null buffer");
    const size_t in_b = n_sets * k * 6 * sizeof(double), out_b = n_sets * 4 * sizeof(double);
    ctx->scratch.ensure(in_b + out_b + n_sets * sizeof(int) + 64, ctx->stream);
    double* dl = ctx->scratch.as<double>();
    double* dout = dl + n_sets * k * 6;
    int* dok = reinterpret_cast<int*>(dout + n_sets * 4);
    OLPT_CUDA(cudaMemcpyAsync(dl, lines6, in_b, cudaMemcpyHostToDevice, ctx->stream));
    triangulate_kernel<<<OLPT_G(nblk(n_sets, 128)), 128, 0, ctx->stream>>>(n_sets, k, dl, dout, dok);
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(out4, dout, out_b, cudaMemcpyDeviceToHost, ctx->stream));
    OLPT_CUDA(cudaMemcpyAsync(ok, dok, n_sets * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_otf_upload(olpt_ctx* ctx, int nx, int ny, int nz, const double* bound6,
                              const double* abca) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(ctx->n_cam > 0, OLPT_ERR_INVALID_ARG, "upload cameras before the OTF");
    OLPT_REQUIRE(bound6 && abca, OLPT_ERR_INVALID_ARG, "null OTF buffers");
    // OTF::loadParam clamps grid sizes below 2 up to 2 (OTF.cpp:159-171)
    nx = nx < 2 ? 2 : nx;
    ny = ny < 2 ? 2 : ny;
    nz = nz < 2 ? 2 : nz;
    OtfDev& o = ctx->otf;
    o.nx = nx;
    o.ny = ny;
    o.nz = nz;
    o.n_grid = nx * ny * nz;
    const int n[3] = {nx, ny, nz};
    for (int k = 0; k < 3; ++k) {
      o.bmin[k] = bound6[2 * k];
      o.bmax[k] = bound6[2 * k + 1];
      o.d[k] = (o.bmax[k] - o.bmin[k]) / (n[k] - 1);  // OTF::setGrid (OTF.cpp:146-157)
    }
    const size_t bytes = (size_t)4 * ctx->n_cam * o.n_grid * sizeof(double);
    o.alpha_zero = 1;
    const double* alpha = abca + (size_t)3 * ctx->n_cam * o.n_grid;
    for (size_t i = 0; i < (size_t)ctx->n_cam * o.n_grid; ++i) {
      uint64_t bits;
      std::memcpy(&bits, alpha + i, sizeof(bits));
      if (bits != 0) o.alpha_zero = 0;
    }
    ctx->otf_table.ensure(bytes, ctx->stream);
    OLPT_CUDA(cudaMemcpyAsync(ctx->otf_table.p, abca, bytes, cudaMemcpyHostToDevice, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_otf_param(olpt_ctx* ctx, int cam, int64_t n, const double* xyz, double* out5) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cam >= 0 && cam < ctx->n_cam && n >= 0 && (n == 0 || (xyz && out5)),
                 OLPT_ERR_INVALID_ARG, "bad camera index or buffers");
    if (n == 0) return;
    OtfView v = otf_view(ctx);
    ctx->scratch.ensure(n * 8 * sizeof(double), ctx->stream);
    double* dx = ctx->scratch.as<double>();
    double* dout = dx + 3 * n;
    OLPT_CUDA(cudaMemcpyAsync(dx, xyz, n * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    otf_param_kernel<<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(v, cam, n, dx, dout);
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(out5, dout, n * 5 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_images_upload(olpt_ctx* ctx, int n_cam, olpt_dtype_t dtype,
                                 const void* const* imgs, const int* H, const int* W,
                                 const int64_t* pitch_bytes, int on_device) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n_cam == ctx->n_cam && imgs && H && W, OLPT_ERR_INVALID_ARG,
                 "image count must equal camera count");
    OLPT_REQUIRE(dtype >= OLPT_U8 && dtype <= OLPT_F64, OLPT_ERR_INVALID_ARG, "bad dtype");
    for (int c = 0; c < n_cam; ++c) {
      OLPT_REQUIRE(imgs[c] && H[c] > 0 && W[c] > 0, OLPT_ERR_INVALID_ARG, "empty image");
      ensure_plane(ctx, c, dtype, H[c], W[c]);
      const int64_t row_b = (int64_t)W[c] * esize(dtype);
      const int64_t sp = (pitch_bytes && pitch_bytes[c]) ? pitch_bytes[c] : row_b;
      OLPT_CUDA(cudaMemcpy2DAsync(ctx->img[c].buf.p, ctx->img[c].pitch, imgs[c], sp, row_b, H[c],
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  ctx->stream));
    }
  });
}

olpt_status_t olpt_image_download(olpt_ctx* ctx, int cam, olpt_dtype_t dtype, void* out) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cam >= 0 && cam < ctx->n_cam && out, OLPT_ERR_INVALID_ARG, "bad camera/buffer");
    OLPT_REQUIRE(dtype == OLPT_F32 || dtype == OLPT_F64, OLPT_ERR_INVALID_ARG,
                 "download dtype must be F32 or F64");
    ImagePlane& im = ctx->img[cam];
    OLPT_REQUIRE(im.buf.p, OLPT_ERR_INVALID_ARG, "no image");
    const int64_t n = (int64_t)im.H * im.W;
    ctx->scratch.ensure(n * 8, ctx->stream);
    if (dtype == OLPT_F32)
      convert_plane_kernel<float><<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(
          im.buf.as<unsigned char>(), im.pitch, im.H, im.W, im.dtype, ctx->scratch.as<float>());
    else
      convert_plane_kernel<double><<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(
          im.buf.as<unsigned char>(), im.pitch, im.H, im.W, im.dtype, ctx->scratch.as<double>());
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(out, ctx->scratch.p, n * esize(dtype), cudaMemcpyDeviceToHost,
                              ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_find_peaks(olpt_ctx* ctx, double min_obj_int, int64_t* counts) {
  return guard(ctx, [&] {
    find_peaks_device(ctx, min_obj_int, true);
    if (counts)
      for (int c = 0; c < ctx->n_cam; ++c) counts[c] = ctx->det_counts_h[c];
  });
}

olpt_status_t olpt_get_peaks(olpt_ctx* ctx, int cam, double* xy, int32_t* rc, int64_t cap) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cam >= 0 && cam < ctx->n_cam, OLPT_ERR_INVALID_ARG, "bad camera index");
    OLPT_REQUIRE((int64_t)ctx->det_counts_h.size() > cam, OLPT_ERR_INVALID_ARG, "no detections");
    const int64_t n = std::min<int64_t>(cap, ctx->det_counts_h[cam]);
    if (n <= 0) return;
    Dets& d = ctx->dets[cam];
    if (xy) {
      std::vector<double> hx(n), hy(n);
      OLPT_CUDA(cudaMemcpyAsync(hx.data(), d.x.p, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
      OLPT_CUDA(cudaMemcpyAsync(hy.data(), d.y.p, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
      OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
      for (int64_t i = 0; i < n; ++i) {
        xy[2 * i] = hx[i];
        xy[2 * i + 1] = hy[i];
      }
    }
    if (rc) {
      OLPT_CUDA(cudaMemcpyAsync(rc, d.rc.p, n * sizeof(int2), cudaMemcpyDeviceToHost, ctx->stream));
      OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
    }
  });
}

olpt_status_t olpt_detections_upload(olpt_ctx* ctx, int n_cam, const int64_t* counts,
                                     const double* const* xy) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n_cam == ctx->n_cam && counts && xy, OLPT_ERR_INVALID_ARG,
                 "detection lists must cover every camera");
    ctx->det_counts_h.assign(n_cam, 0);
    ctx->det_counts.ensure(OLPT_MAX_CAM * sizeof(int64_t), ctx->stream);
    for (int c = 0; c < n_cam; ++c) {
      const int64_t n = counts[c];
      OLPT_REQUIRE(n >= 0 && (n == 0 || xy[c]), OLPT_ERR_INVALID_ARG, "bad detection list");
      ensure_det_capacity(ctx, c, std::max<int64_t>(n, 1));
      std::vector<double> hx(n), hy(n);
      std::vector<int2> hrc(n);
      for (int64_t i = 0; i < n; ++i) {
        hx[i] = xy[c][2 * i];
        hy[i] = xy[c][2 * i + 1];
        hrc[i] = make_int2((int)std::floor(hy[i] + 0.5), (int)std::floor(hx[i] + 0.5));
      }
      if (n) {
        OLPT_CUDA(cudaMemcpyAsync(ctx->dets[c].x.p, hx.data(), n * 8, cudaMemcpyHostToDevice, ctx->stream));
        OLPT_CUDA(cudaMemcpyAsync(ctx->dets[c].y.p, hy.data(), n * 8, cudaMemcpyHostToDevice, ctx->stream));
        OLPT_CUDA(cudaMemcpyAsync(ctx->dets[c].rc.p, hrc.data(), n * sizeof(int2),
                                  cudaMemcpyHostToDevice, ctx->stream));
      }
      ctx->det_counts_h[c] = n;
    }
    OLPT_CUDA(cudaMemcpyAsync(ctx->det_counts.p, ctx->det_counts_h.data(), n_cam * sizeof(int64_t),
                              cudaMemcpyHostToDevice, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

}  // extern "C"

extern "C" {

olpt_status_t olpt_stereo_match(olpt_ctx* ctx, const olpt_sm_params* p, int64_t* n_candidates,
                                int64_t* n_matches) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    OLPT_REQUIRE((int)ctx->det_counts_h.size() == ctx->n_cam, OLPT_ERR_INVALID_ARG,
                 "no detections: run olpt_find_peaks or olpt_detections_upload first");
    SmParams prm;
    prm.match_cam_count = p->match_cam_count;
    prm.idmap_cell_px = p->idmap_cell_px;
    prm.tol_2d_px = p->tol_2d_px;
    prm.tol_3d_mm = p->tol_3d_mm;
    for (int q = 0; q < 6; ++q) prm.limit[q] = p->limit[q];
    StereoResult& r = ctx->sm_result;
    stereo_match_device(ctx, prm, r);
    // selected matches become the current 3D objects (triangulateMatch order)
    const int64_t n = stereo_objects(ctx, r);
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
    if (n_candidates) *n_candidates = r.M;
    if (n_matches) *n_matches = n;
  });
}

olpt_status_t olpt_test_hold_detection_band(olpt_ctx* ctx, int ticket, int64_t wait_limit_ns) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(ticket >= 0 && wait_limit_ns > 0 && wait_limit_ns <= 2000000000ll,
                 OLPT_ERR_INVALID_ARG, "ticket >= 0 and 0 < wait_limit_ns <= 2 s");
    ctx->test_hold_ticket = ticket;
    ctx->test_wait_limit_ns = (unsigned long long)wait_limit_ns;
  });
}

olpt_status_t olpt_stereo_near_log_enable(olpt_ctx* ctx, double band_px, int64_t capacity) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(band_px >= 0.0 && capacity >= 0, OLPT_ERR_INVALID_ARG,
                 "band_px and capacity must be non-negative");
    StereoWork& W = ctx->sm;
    W.near_band = band_px;
    W.near_cap = band_px > 0.0 ? capacity : 0;
    if (band_px > 0.0) {
      W.near_rec.ensure(sizeof(olpt_near_record) * (size_t)(capacity + 1), ctx->stream);
      W.near_count.ensure(sizeof(unsigned long long), ctx->stream);
      OLPT_CUDA(cudaMemsetAsync(W.near_count.p, 0, sizeof(unsigned long long), ctx->stream));
      OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
    }
  });
}

olpt_status_t olpt_stereo_near_log_reset(olpt_ctx* ctx) {
  return guard(ctx, [&] {
    if (ctx->sm.near_band > 0.0) {
      OLPT_CUDA(cudaMemsetAsync(ctx->sm.near_count.p, 0, sizeof(unsigned long long), ctx->stream));
      OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
    }
  });
}

olpt_status_t olpt_stereo_near_log_read(olpt_ctx* ctx, olpt_near_record* out, int64_t cap,
                                        int64_t* n_total) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cap >= 0 && (cap == 0 || out), OLPT_ERR_INVALID_ARG, "null output");
    StereoWork& W = ctx->sm;
    unsigned long long n = 0;
    if (W.near_band > 0.0) {
      OLPT_CUDA(cudaMemcpyAsync(&n, W.near_count.p, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream));
      OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
      const int64_t k = std::min<int64_t>({(int64_t)n, W.near_cap, cap});
      if (k > 0) {
        OLPT_CUDA(cudaMemcpyAsync(out, W.near_rec.p, sizeof(olpt_near_record) * (size_t)k,
                                  cudaMemcpyDeviceToHost, ctx->stream));
        OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
      }
    }
    if (n_total) *n_total = (int64_t)n;
  });
}

olpt_status_t olpt_get_candidates(olpt_ctx* ctx, int32_t* ids, double* e_check, double* xyz) {
  return guard(ctx, [&] {
    StereoResult& r = ctx->sm_result;
    stereo_result_to_host(ctx, r);
    const size_t M = r.e.size();
    if (ids) std::copy(r.ids.begin(), r.ids.end(), ids);
    if (e_check) std::copy(r.e.begin(), r.e.end(), e_check);
    if (xyz) std::copy(r.X.begin(), r.X.end(), xyz);
    (void)M;
  });
}

olpt_status_t olpt_prune_matches(int n_cam, int64_t M, const int32_t* ids, const double* e_check,
                                 const int64_t* det_counts, const int* active, uint8_t* selected) {
  if (n_cam < 1 || n_cam > OLPT_MAX_CAM || M < 0 || (M > 0 && (!ids || !e_check || !selected)) ||
      !det_counts || !active)
    return OLPT_ERR_INVALID_ARG;
  try {
    StereoResult r;
    r.n_cam = n_cam;
    r.ids.assign(ids, ids + M * n_cam);
    r.e.assign(e_check, e_check + M);
    r.X.assign(3 * M, 0.0);
    std::vector<int> counts(n_cam), act(n_cam);
    for (int c = 0; c < n_cam; ++c) {
      counts[c] = (int)det_counts[c];
      act[c] = active[c];
    }
    prune_candidates(r, counts, act);
    for (int64_t j = 0; j < M; ++j) selected[j] = (uint8_t)r.selected[j];
    return OLPT_OK;
  } catch (...) {
    return OLPT_ERR_INTERNAL;
  }
}

olpt_status_t olpt_prune_matches_device(olpt_ctx* ctx, int n_cam, int64_t M, const int32_t* ids,
                                        const double* e_check, const int64_t* det_counts,
                                        const int* active, uint8_t* selected) {
  if (!ctx) return OLPT_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    OLPT_REQUIRE(n_cam >= 1 && n_cam <= OLPT_MAX_CAM && M >= 0 && M < (int64_t)INT32_MAX / n_cam &&
                     (M == 0 || (ids && e_check && selected)) && det_counts && active,
                 OLPT_ERR_INVALID_ARG, "prune_matches_device: bad arguments");
    cudaStream_t s = ctx->stream;
    PruneView pv{};
    int64_t total = 0;
    for (int c = 0; c < n_cam; ++c) {
      OLPT_REQUIRE(det_counts[c] >= 0 && det_counts[c] < INT32_MAX, OLPT_ERR_INVALID_ARG,
                   "prune_matches_device: bad det_counts");
      pv.active[c] = active[c];
      pv.count[c] = (int)det_counts[c];
      pv.offset[c] = (int)total;
      total += det_counts[c];
    }
    OLPT_REQUIRE(total < INT32_MAX, OLPT_ERR_UNSUPPORTED, "prune_matches_device: too many points");
    for (int64_t j = 0; j < M * n_cam; ++j) {
      const int c = (int)(j % n_cam);
      OLPT_REQUIRE(ids[j] >= -1 && (!active[c] || ids[j] < det_counts[c]), OLPT_ERR_INVALID_ARG,
                   "prune_matches_device: id out of range");
    }
    stereo_result_to_host(ctx, ctx->sm_result);  // its arrays live in the same workspace
    PruneWork& P = ctx->prune;
    P.ids_s.ensure((size_t)(M + 1) * n_cam * sizeof(int), s);
    P.e_s.ensure((size_t)(M + 1) * sizeof(double), s);
    if (M > 0) {
      OLPT_CUDA(cudaMemcpyAsync(P.ids_s.p, ids, (size_t)M * n_cam * sizeof(int),
                                cudaMemcpyHostToDevice, s));
      OLPT_CUDA(cudaMemcpyAsync(P.e_s.p, e_check, (size_t)M * sizeof(double),
                                cudaMemcpyHostToDevice, s));
    }
    std::vector<char> sel(M, 0);
    if (!prune_select_device(ctx, pv, (int)M, n_cam, total, sel.data())) {
      OLPT_CUDA(cudaStreamSynchronize(s));
      StereoResult r;
      r.n_cam = n_cam;
      r.ids.assign(ids, ids + M * n_cam);
      r.e.assign(e_check, e_check + M);
      r.X.assign(3 * M, 0.0);
      std::vector<int> counts(n_cam), act(n_cam);
      for (int c = 0; c < n_cam; ++c) {
        counts[c] = pv.count[c];
        act[c] = active[c];
      }
      prune_candidates(r, counts, act);
      sel.assign(r.selected.begin(), r.selected.end());
    }
    for (int64_t j = 0; j < M; ++j) selected[j] = (uint8_t)sel[j];
  });
}

olpt_status_t olpt_get_matches(olpt_ctx* ctx, int32_t* ids, double* xyz) {
  return guard(ctx, [&] {
    StereoResult& r = ctx->sm_result;
    stereo_result_to_host(ctx, r);
    const int n = r.n_cam;
    int64_t k = 0;
    for (size_t j = 0; j < r.e.size(); ++j) {
      if (!r.selected[j]) continue;
      if (ids) std::copy(&r.ids[j * n], &r.ids[j * n] + n, ids + k * n);
      if (xyz) std::copy(&r.X[3 * j], &r.X[3 * j] + 3, xyz + 3 * k);
      ++k;
    }
  });
}

}  // extern "C"

// ---------------------------------------------------------------- objects / shake
#include "olpt_shake.h"

namespace olpt {
namespace {
olpt::ShakeParams to_shake_params(const olpt_shake_params* p) {
  olpt::ShakeParams s;
  s.shake_width = p->shake_width;
  s.shakewidth_min = p->shakewidth_min;
  s.n_shake_loop = p->n_shake_loop;
  s.thred_ghost = p->thred_ghost;
  s.ratio_augimg = p->ratio_augimg;
  s.radius_obj = p->radius_obj;
  s.tol_3d_mm = p->tol_3d_mm;
  s.precision = p->precision;
  return s;
}

__global__ void init_objects_kernel(uint8_t* flags, double* score, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  flags[i] = 0;
  score[i] = 1.0;
}
}  // namespace
}  // namespace olpt

extern "C" {

olpt_status_t olpt_objects_upload(olpt_ctx* ctx, int64_t n, const double* xyz) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(ctx->n_cam > 0, OLPT_ERR_INVALID_ARG, "upload cameras first");
    OLPT_REQUIRE(n >= 0 && (n == 0 || xyz), OLPT_ERR_INVALID_ARG, "bad object buffer");
    ctx->obj.ensure(std::max<int64_t>(n, 1), ctx->n_cam, ctx->stream);
    ctx->obj.n = n;
    if (n > 0) {
      OLPT_CUDA(cudaMemcpyAsync(ctx->obj.xyz.p, xyz, n * 3 * sizeof(double), cudaMemcpyHostToDevice,
                                ctx->stream));
      init_objects_kernel<<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(ctx->obj.flags.as<uint8_t>(),
                                                             ctx->obj.score.as<double>(), n);
      OLPT_CUDA(cudaGetLastError());
    }
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_objects_count(olpt_ctx* ctx, int64_t* n) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n, OLPT_ERR_INVALID_ARG, "null output");
    *n = ctx->obj.n;
  });
}

olpt_status_t olpt_objects_download(olpt_ctx* ctx, double* xyz, double* uv, uint8_t* flags,
                                    double* score) {
  return guard(ctx, [&] {
    const int64_t n = ctx->obj.n;
    if (n <= 0) return;
    cudaStream_t s = ctx->stream;
    if (xyz) OLPT_CUDA(cudaMemcpyAsync(xyz, ctx->obj.xyz.p, n * 3 * 8, cudaMemcpyDeviceToHost, s));
    if (uv)
      OLPT_CUDA(cudaMemcpyAsync(uv, ctx->obj.uv.p, n * ctx->n_cam * 2 * 8, cudaMemcpyDeviceToHost, s));
    if (flags) OLPT_CUDA(cudaMemcpyAsync(flags, ctx->obj.flags.p, n, cudaMemcpyDeviceToHost, s));
    if (score) OLPT_CUDA(cudaMemcpyAsync(score, ctx->obj.score.p, n * 8, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
  });
}

olpt_status_t olpt_shake(olpt_ctx* ctx, const olpt_shake_params* p) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    OLPT_REQUIRE(p->precision == 0 || p->precision == 1, OLPT_ERR_INVALID_ARG,
                 "precision must be 0 (FP32) or 1 (FP64)");
    shake_device(ctx, to_shake_params(p));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_residual(olpt_ctx* ctx, const olpt_shake_params* p, int use_flags,
                            int make_current) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    residual_device(ctx, to_shake_params(p), use_flags != 0, make_current != 0);
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

}  // extern "C"

namespace olpt {
namespace {
IprParams to_ipr_params(const olpt_ipr_params* p) {
  OLPT_REQUIRE(p->shake.precision == 0 || p->shake.precision == 1, OLPT_ERR_INVALID_ARG,
               "precision must be 0 (FP32) or 1 (FP64)");
  IprParams ip;
  ip.min_obj_int = p->min_obj_int;
  ip.sm.match_cam_count = p->sm.match_cam_count;
  ip.sm.idmap_cell_px = p->sm.idmap_cell_px;
  ip.sm.tol_2d_px = p->sm.tol_2d_px;
  ip.sm.tol_3d_mm = p->sm.tol_3d_mm;
  for (int q = 0; q < 6; ++q) ip.sm.limit[q] = p->sm.limit[q];
  ip.shake = to_shake_params(&p->shake);
  ip.n_cam_reduced = p->n_cam_reduced;
  ip.n_loop_ipr = p->n_loop_ipr;
  ip.n_loop_ipr_reduced = p->n_loop_ipr_reduced;
  ip.n_obj2d_process_max = p->n_obj2d_process_max;
  return ip;
}
}  // namespace
}  // namespace olpt

extern "C" {

olpt_status_t olpt_ipr_run(olpt_ctx* ctx, const olpt_ipr_params* p, int64_t* n_objects) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    OLPT_REQUIRE(p->shake.precision == 0 || p->shake.precision == 1, OLPT_ERR_INVALID_ARG,
                 "precision must be 0 (FP32) or 1 (FP64)");
    ipr_device(ctx, to_ipr_params(p));
    if (n_objects) *n_objects = ctx->ipr.n_out;
  });
}

// Persistent host workers for the batch entry points: job i of a batch runs on worker
// i, which keeps its thread across batches (no thread start-up per frame).
class BatchPool {
 public:
  ~BatchPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      quit_ = true;
      gen_++;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  // runs fn(0 .. n-1) on n workers and waits for all of them; one batch at a time
  void run(int n, const std::function<void(int)>& fn) {
    std::lock_guard<std::mutex> one(batch_mu_);
    std::unique_lock<std::mutex> lk(mu_);
    while ((int)th_.size() < n) {
      // a new worker starts from the generation before this batch, so that it takes
      // this batch however late it first acquires the lock
      const int id = (int)th_.size();
      th_.emplace_back([this, id, g = gen_] { loop(id, g); });
    }
    fn_ = &fn;
    n_ = n;
    left_ = n;
    gen_++;
    cv_.notify_all();
    done_cv_.wait(lk, [this] { return left_ == 0; });
    fn_ = nullptr;
  }

 private:
  void loop(int id, uint64_t seen) {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return gen_ != seen; });
      seen = gen_;
      if (quit_) return;
      if (id >= n_) continue;
      const std::function<void(int)>* f = fn_;
      lk.unlock();
      (*f)(id);
      lk.lock();
      if (--left_ == 0) done_cv_.notify_all();
    }
  }
  std::mutex mu_, batch_mu_;
  std::condition_variable cv_, done_cv_;
  std::vector<std::thread> th_;
  const std::function<void(int)>* fn_ = nullptr;
  int n_ = 0, left_ = 0;
  uint64_t gen_ = 0;
  bool quit_ = false;
};

static BatchPool& batch_pool() {
  static BatchPool pool;
  return pool;
}

static bool distinct_contexts(olpt_ctx* const* ctxs, int n_ctx) {
  for (int i = 0; i < n_ctx; ++i)
    for (int j = 0; j < i; ++j)
      if (!ctxs[i] || ctxs[i] == ctxs[j]) return false;
  return n_ctx > 0 && ctxs[0];
}

olpt_status_t olpt_ipr_run_batch(olpt_ctx* const* ctxs, int n_ctx, const olpt_ipr_params* p,
                                 int64_t* n_objects) {
  if (!ctxs || n_ctx <= 0 || !p || !distinct_contexts(ctxs, n_ctx)) return OLPT_ERR_INVALID_ARG;
  std::vector<olpt_status_t> st(n_ctx, OLPT_OK);
  std::vector<int64_t> cnt(n_ctx, 0);
  batch_pool().run(n_ctx, [&](int i) {
    cudaSetDevice(ctxs[i]->device);
    st[i] = olpt_ipr_run(ctxs[i], p, &cnt[i]);
  });
  for (int i = 0; i < n_ctx; ++i)
    if (n_objects) n_objects[i] = cnt[i];
  for (int i = 0; i < n_ctx; ++i)
    if (st[i] != OLPT_OK) return st[i];
  return OLPT_OK;
}

olpt_status_t olpt_tuning_get(olpt_ctx* ctx, olpt_tuning* out) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(out, OLPT_ERR_INVALID_ARG, "null output");
    *out = ctx->tune;
  });
}

olpt_status_t olpt_tuning_set(olpt_ctx* ctx, const olpt_tuning* t) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(t, OLPT_ERR_INVALID_ARG, "null tuning");
    const int w = t->shake_warps_per_block, r = t->residual_threads, g = t->shake_regs;
    OLPT_REQUIRE(w == 1 || w == 2 || w == 4, OLPT_ERR_INVALID_ARG,
                 "shake warps per block must be 1, 2 or 4");
    OLPT_REQUIRE(r == 128 || r == 256, OLPT_ERR_INVALID_ARG,
                 "residual threads per block must be 128 or 256");
    OLPT_REQUIRE(g == 64 || g == 128, OLPT_ERR_INVALID_ARG,
                 "shake registers per thread must be 64 or 128");
    ctx->tune = *t;
  });
}

static const olpt_tuning kTuneCand[OLPT_TUNING_CANDIDATES] = {
    {4, 256, 64},  {2, 256, 64},  {1, 256, 64},  {4, 256, 128},
    {2, 256, 128}, {4, 128, 64},  {2, 128, 64},  {4, 128, 128}};

olpt_status_t olpt_tuning_candidates(olpt_tuning* out, int* n) {
  if (!n) return OLPT_ERR_INVALID_ARG;
  *n = OLPT_TUNING_CANDIDATES;
  if (out)
    for (int i = 0; i < OLPT_TUNING_CANDIDATES; ++i) out[i] = kTuneCand[i];
  return OLPT_OK;
}

olpt_status_t olpt_autotune_ipr(olpt_ctx* ctx, const olpt_ipr_params* p, int reps,
                                olpt_tuning* best, double* best_ms, double* cand_ms) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p && reps > 0, OLPT_ERR_INVALID_ARG, "bad arguments");
    OLPT_REQUIRE(ctx->n_cam > 0 && ctx->img[0].buf.p, OLPT_ERR_INVALID_ARG, "no images uploaded");
    cudaStream_t s = ctx->stream;
    // the images as uploaded: every trial starts from them, and they are put back
    // (the IPR leaves its residual in the planes, as F32 or F64: the planes' type and
    // geometry are put back with their contents)
    std::vector<DevBuf> keep(ctx->n_cam);
    std::vector<ImagePlane> meta(ctx->n_cam);
    for (int c = 0; c < ctx->n_cam; ++c) {
      const ImagePlane& im = ctx->img[c];
      meta[c].dtype = im.dtype;
      meta[c].H = im.H;
      meta[c].W = im.W;
      meta[c].pitch = im.pitch;
      const size_t bytes = (size_t)im.pitch * im.H;
      keep[c].ensure(bytes + 16, s);
      OLPT_CUDA(cudaMemcpyAsync(keep[c].p, im.buf.p, bytes, cudaMemcpyDeviceToDevice, s));
    }
    auto restore = [&] {
      for (int c = 0; c < ctx->n_cam; ++c) {
        const ImagePlane& m = meta[c];
        ensure_plane(ctx, c, m.dtype, m.H, m.W);
        OLPT_CUDA(cudaMemcpy2DAsync(ctx->img[c].buf.p, ctx->img[c].pitch, keep[c].p, m.pitch,
                                    (size_t)m.W * esize(m.dtype), m.H,
                                    cudaMemcpyDeviceToDevice, s));
      }
    };
    auto run = [&](std::vector<double>* xyz) {
      int64_t n = 0;
      const olpt_status_t st = olpt_ipr_run(ctx, p, &n);
      if (st != OLPT_OK) throw ApiError{st, ctx->err};
      if (xyz) {
        xyz->resize((size_t)n * 3);
        if (n > 0)
          OLPT_CUDA(cudaMemcpyAsync(xyz->data(), ctx->ipr.out_xyz.p, n * 3 * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
        OLPT_CUDA(cudaStreamSynchronize(s));
      }
    };
    const olpt_tuning start = ctx->tune;
    const olpt_tuning* cand = kTuneCand;
    std::vector<double> first, got;
    double best_t = 0;
    olpt_tuning pick = start;
    try {
      for (int k = 0; k < OLPT_TUNING_CANDIDATES; ++k) {
        ctx->tune = cand[k];
        restore();
        run(&got);  // untimed: warms the launch shape, and its objects are checked
        if (k == 0)
          first = got;
        else
          OLPT_REQUIRE(got == first, OLPT_ERR_INTERNAL,
                       "autotune: a launch shape changed the reconstructed objects");
        double total = 0;
        for (int r = 0; r < reps; ++r) {
          restore();
          OLPT_CUDA(cudaStreamSynchronize(s));
          const auto a = std::chrono::steady_clock::now();
          run(nullptr);
          OLPT_CUDA(cudaStreamSynchronize(s));
          total += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a)
                       .count();
        }
        const double t = total / reps;
        if (cand_ms) cand_ms[k] = t;
        if (k == 0 || t < best_t) {
          best_t = t;
          pick = cand[k];
        }
      }
    } catch (...) {
      ctx->tune = start;
      restore();
      for (auto& b : keep) b.release(s);
      throw;
    }
    ctx->tune = pick;
    restore();
    OLPT_CUDA(cudaStreamSynchronize(s));
    for (auto& b : keep) b.release(s);
    if (best) *best = pick;
    if (best_ms) *best_ms = best_t;
  });
}

olpt_status_t olpt_stb_process_frame_batch(olpt_ctx* const* ctxs, int n_ctx, const int* frames) {
  if (!ctxs || n_ctx <= 0 || !frames || !distinct_contexts(ctxs, n_ctx)) return OLPT_ERR_INVALID_ARG;
  std::vector<olpt_status_t> st(n_ctx, OLPT_OK);
  batch_pool().run(n_ctx, [&](int i) {
    cudaSetDevice(ctxs[i]->device);
    st[i] = olpt_stb_process_frame(ctxs[i], frames[i]);
  });
  for (int i = 0; i < n_ctx; ++i)
    if (st[i] != OLPT_OK) return st[i];
  return OLPT_OK;
}

olpt_status_t olpt_ipr_result(olpt_ctx* ctx, double* xyz, double* uv) {
  return guard(ctx, [&] {
    const int64_t n = ctx->ipr.n_out;
    if (n <= 0) return;
    if (xyz)
      OLPT_CUDA(cudaMemcpyAsync(xyz, ctx->ipr.out_xyz.p, n * 3 * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
    if (uv)
      OLPT_CUDA(cudaMemcpyAsync(uv, ctx->ipr.out_uv.p, n * ctx->n_cam * 2 * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_residual_download(olpt_ctx* ctx, int cam, olpt_dtype_t dtype, void* out) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cam >= 0 && cam < ctx->n_cam && out, OLPT_ERR_INVALID_ARG, "bad camera/buffer");
    OLPT_REQUIRE(dtype == OLPT_F32 || dtype == OLPT_F64, OLPT_ERR_INVALID_ARG,
                 "download dtype must be F32 or F64");
    ImagePlane& im = ctx->resid[cam];
    OLPT_REQUIRE(im.buf.p, OLPT_ERR_INVALID_ARG, "no residual computed");
    const int64_t n = (int64_t)im.H * im.W;
    ctx->scratch.ensure(n * 8, ctx->stream);
    if (dtype == OLPT_F32)
      convert_plane_kernel<float><<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(
          im.buf.as<unsigned char>(), im.pitch, im.H, im.W, im.dtype, ctx->scratch.as<float>());
    else
      convert_plane_kernel<double><<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(
          im.buf.as<unsigned char>(), im.pitch, im.H, im.W, im.dtype, ctx->scratch.as<double>());
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(out, ctx->scratch.p, n * esize(dtype), cudaMemcpyDeviceToHost,
                              ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_stb_configure(olpt_ctx* ctx, const olpt_stb_params* p) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    OLPT_REQUIRE(ctx->n_cam >= 2, OLPT_ERR_INVALID_ARG, "upload at least 2 cameras first");
    StbParams sp;
    sp.frame_start = p->frame_start;
    sp.frame_end = p->frame_end;
    sp.n_initial_frames = p->n_initial_frames;
    sp.radius_search_obj = p->radius_search_obj_mm;
    sp.radius_search_track = p->radius_search_track_mm;
    for (int q = 0; q < 6; ++q) sp.limit[q] = p->limit[q];
    for (int k = 0; k < 3; ++k) {
      sp.pf_n[k] = p->pf_n[k];
      sp.pf_nbin[k] = p->pf_nbin[k];
      sp.pf_sigma[k] = p->pf_sigma[k];
    }
    sp.pf_r = p->pf_r_mm;
    sp.pf_smooth = p->pf_smooth;
    sp.output_path = p->output_path ? p->output_path : "";
    stb_configure(ctx, sp, to_ipr_params(&p->ipr));
  });
}

olpt_status_t olpt_stb_process_frame(olpt_ctx* ctx, int frame) {
  return guard(ctx, [&] { stb_process_frame(ctx, frame); });
}

olpt_status_t olpt_stb_counts(olpt_ctx* ctx, int64_t counts[4], int64_t* n_extended,
                              int64_t* n_new) {
  return guard(ctx, [&] {
    if (counts)
      for (int w = 0; w < 4; ++w) counts[w] = (int64_t)stb_list(ctx, w).size();
    if (n_extended) *n_extended = ctx->stb.last_extended;
    if (n_new) *n_new = ctx->stb.last_new;
  });
}

olpt_status_t olpt_stb_frame_objects(olpt_ctx* ctx, int64_t* n, double* xyz) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n, OLPT_ERR_INVALID_ARG, "null count");
    const std::vector<double>& v = ctx->stb.last_xyz;
    const int64_t m = (int64_t)(v.size() / 3);
    if (xyz) {
      OLPT_REQUIRE(*n >= m, OLPT_ERR_INVALID_ARG, "output capacity too small");
      std::copy(v.begin(), v.end(), xyz);
    }
    *n = m;
  });
}

olpt_status_t olpt_stb_frame_image(olpt_ctx* ctx, int cam, olpt_dtype_t dtype, void* out) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(cam >= 0 && cam < ctx->n_cam && out, OLPT_ERR_INVALID_ARG, "bad camera/buffer");
    OLPT_REQUIRE(dtype == OLPT_F32 || dtype == OLPT_F64, OLPT_ERR_INVALID_ARG,
                 "download dtype must be F32 or F64");
    const ImagePlane& im = ctx->stb.frame_img[cam];
    OLPT_REQUIRE(im.buf.p, OLPT_ERR_INVALID_ARG, "no frame processed");
    const int64_t n = (int64_t)im.H * im.W;
    ctx->scratch.ensure(n * 8, ctx->stream);
    if (dtype == OLPT_F32)
      convert_plane_kernel<float><<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(
          im.buf.as<unsigned char>(), im.pitch, im.H, im.W, im.dtype, ctx->scratch.as<float>());
    else
      convert_plane_kernel<double><<<OLPT_G(nblk(n)), 256, 0, ctx->stream>>>(
          im.buf.as<unsigned char>(), im.pitch, im.H, im.W, im.dtype, ctx->scratch.as<double>());
    OLPT_CUDA(cudaGetLastError());
    OLPT_CUDA(cudaMemcpyAsync(out, ctx->scratch.p, n * esize(dtype), cudaMemcpyDeviceToHost,
                              ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_stb_frame_points(olpt_ctx* ctx, int frame, int64_t* n) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n, OLPT_ERR_INVALID_ARG, "null count");
    int64_t m = 0;
    for (int w = 0; w < 4; ++w)
      for (const auto& tr : stb_list(ctx, w))
        m += (int64_t)std::count(tr.t.begin(), tr.t.end(), frame);
    *n = m;
  });
}

olpt_status_t olpt_stb_track_rows(olpt_ctx* ctx, int which, int64_t* n_tracks, int64_t* n_rows) {
  return guard(ctx, [&] {
    const auto& L = stb_list(ctx, which);
    int64_t r = 0;
    for (const auto& t : L) r += (int64_t)t.size();
    if (n_tracks) *n_tracks = (int64_t)L.size();
    if (n_rows) *n_rows = r;
  });
}

olpt_status_t olpt_stb_get_tracks(olpt_ctx* ctx, int which, int32_t* track_id, int32_t* frame,
                                  double* xyz, int64_t capacity_rows) {
  return guard(ctx, [&] {
    const auto& L = stb_list(ctx, which);
    int64_t r = 0;
    for (size_t i = 0; i < L.size(); ++i)
      for (size_t k = 0; k < L[i].size(); ++k, ++r) {
        OLPT_REQUIRE(r < capacity_rows, OLPT_ERR_INVALID_ARG, "output capacity too small");
        if (track_id) track_id[r] = (int32_t)i;
        if (frame) frame[r] = L[i].t[k];
        if (xyz)
          for (int d = 0; d < 3; ++d) xyz[3 * r + d] = L[i].xyz[3 * k + d];
      }
  });
}

olpt_status_t olpt_stb_set_tracks(olpt_ctx* ctx, int which, const int32_t* track_id,
                                  const int32_t* frame, const double* xyz, int64_t n_rows) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n_rows >= 0 && (n_rows == 0 || (track_id && frame && xyz)), OLPT_ERR_INVALID_ARG,
                 "bad track rows");
    auto& L = stb_list(ctx, which);
    L.clear();
    for (int64_t r = 0; r < n_rows; ++r) {
      OLPT_REQUIRE(track_id[r] >= 0, OLPT_ERR_INVALID_ARG, "negative track id");
      while ((int64_t)L.size() <= track_id[r]) L.emplace_back();
      TrackH& t = L[track_id[r]];
      t.xyz.insert(t.xyz.end(), xyz + 3 * r, xyz + 3 * r + 3);
      t.t.push_back(frame[r]);
    }
  });
}

olpt_status_t olpt_stb_save_tracks(olpt_ctx* ctx, int which, const char* path) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(path, OLPT_ERR_INVALID_ARG, "null path");
    stb_save_tracks(ctx, which, path);
  });
}

olpt_status_t olpt_stb_load_tracks(olpt_ctx* ctx, int which, const char* path) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(path, OLPT_ERR_INVALID_ARG, "null path");
    flush_files(ctx);  // the file may still be queued for writing
    stb_load_tracks(ctx, which, path);
  });
}

olpt_status_t olpt_otf_estimate(olpt_ctx* ctx, double min_obj_int, double radius_obj_px,
                                int max_per_image, double abc[3], int64_t* n_samples) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(abc && n_samples && max_per_image > 0 && radius_obj_px >= 0,
                 OLPT_ERR_INVALID_ARG, "bad arguments");
    *n_samples = 0;
    otf_estimate_device(ctx, min_obj_int, radius_obj_px, max_per_image, abc, n_samples);
  });
}

olpt_status_t olpt_track_files_async(olpt_ctx* ctx, int enable) {
  return guard(ctx, [&] {
    if (!enable) flush_files(ctx);
    ctx->tio.async = enable != 0;
  });
}

olpt_status_t olpt_track_files_flush(olpt_ctx* ctx) {
  return guard(ctx, [&] { flush_files(ctx); });
}

olpt_status_t olpt_format_fixed6(olpt_ctx* ctx, const double* values, int64_t n, char* out,
                                 int64_t capacity, int64_t* length) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n >= 0 && (n == 0 || values) && length, OLPT_ERR_INVALID_ARG, "bad arguments");
    std::string o;
    TrackIoWork& W = ctx->tio;
    for (int64_t at = 0; at < n; at += kMaxRowsPerPass) {
      const int64_t m = std::min<int64_t>(kMaxRowsPerPass, n - at);
      W.xyz.ensure((size_t)m * sizeof(double) + 16, ctx->stream);
      OLPT_CUDA(cudaMemcpyAsync(W.xyz.p, values + at, (size_t)m * sizeof(double),
                                cudaMemcpyHostToDevice, ctx->stream));
      format_rows_device(ctx, nullptr, 0, W.xyz.as<double>(), 1, nullptr, 0, m, o);
    }
    *length = (int64_t)o.size();
    OLPT_REQUIRE(!out || capacity >= (int64_t)o.size(), OLPT_ERR_INVALID_ARG,
                 "output capacity too small");
    if (out) std::memcpy(out, o.data(), o.size());
  });
}


// ---------------------------------------------------------------- learned proposal
olpt_status_t olpt_mlp_dims(int n_cam, int* n_in, int64_t* n_params) {
  if (n_cam < 2 || n_cam > kMlpMaxCams) return OLPT_ERR_INVALID_ARG;
  const MlpDims d = mlp_dims(n_cam);
  if (n_in) *n_in = d.in;
  if (n_params) *n_params = d.params;
  return OLPT_OK;
}

olpt_status_t olpt_mlp_init(olpt_ctx* ctx, uint64_t seed) {
  return guard(ctx, [&] { mlp_init(ctx, seed); });
}

olpt_status_t olpt_mlp_set_params(olpt_ctx* ctx, const float* params) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(params, OLPT_ERR_INVALID_ARG, "null params");
    mlp_set_params(ctx, params);
  });
}

olpt_status_t olpt_mlp_get_params(olpt_ctx* ctx, float* params) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(params, OLPT_ERR_INVALID_ARG, "null params");
    mlp_get_params(ctx, params);
  });
}

olpt_status_t olpt_mlp_forward(olpt_ctx* ctx, int64_t n, const float* x, float* out,
                               int on_device) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n >= 0 && n < (int64_t)INT32_MAX && (n == 0 || (x && out)),
                 OLPT_ERR_INVALID_ARG, "mlp_forward: bad arguments");
    if (n == 0) return;
    MlpWork& W = ctx->mlp;
    cudaStream_t s = ctx->stream;
    const float* dx = x;
    if (!on_device) {
      W.xin.ensure((size_t)n * ctx->mlp.dims.in * 4, s);
      OLPT_CUDA(cudaMemcpyAsync(W.xin.p, x, (size_t)n * ctx->mlp.dims.in * 4, cudaMemcpyHostToDevice, s));
      dx = W.xin.as<float>();
    }
    W.x.ensure((size_t)n * ctx->mlp.dims.in_pad * 2, s);
    W.o.ensure((size_t)n * kMlpOut * 4, s);
    mlp_input_device(ctx, dx, n, W.x.as<__nv_bfloat16>());
    mlp_infer_device(ctx, W.x.as<__nv_bfloat16>(), n, W.o.as<float>());
    OLPT_CUDA(cudaMemcpyAsync(out, W.o.p, (size_t)n * kMlpOut * 4,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
  });
}

olpt_status_t olpt_mlp_train_step(olpt_ctx* ctx, int64_t n, const float* x, const float* targets,
                                  int on_device, double lr, double ghost_weight, int update,
                                  double* loss, float* grad) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n > 0 && n < (int64_t)INT32_MAX && x && targets, OLPT_ERR_INVALID_ARG,
                 "mlp_train_step: bad arguments");
    MlpWork& W = ctx->mlp;
    cudaStream_t s = ctx->stream;
    const float* dx = x;
    const float* dt = targets;
    if (!on_device) {
      W.xin.ensure((size_t)n * ctx->mlp.dims.in * 4, s);
      W.tgt.ensure((size_t)n * kMlpOut * 4, s);
      OLPT_CUDA(cudaMemcpyAsync(W.xin.p, x, (size_t)n * ctx->mlp.dims.in * 4, cudaMemcpyHostToDevice, s));
      OLPT_CUDA(cudaMemcpyAsync(W.tgt.p, targets, (size_t)n * kMlpOut * 4, cudaMemcpyHostToDevice,
                                s));
      dx = W.xin.as<float>();
      dt = W.tgt.as<float>();
    }
    const double l = mlp_train_device(ctx, dx, dt, n, lr, ghost_weight, update != 0);
    if (loss) *loss = l;
    if (grad) {
      OLPT_CUDA(cudaMemcpyAsync(grad, W.grad.p, (size_t)ctx->mlp.dims.params * 4, cudaMemcpyDeviceToHost, s));
      OLPT_CUDA(cudaStreamSynchronize(s));
    }
  });
}

olpt_status_t olpt_mlp_train(olpt_ctx* ctx, int64_t n, const float* x, const float* targets,
                             int on_device, int batch, int steps, double lr, double ghost_weight,
                             uint64_t seed, float* losses) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(n > 0 && x && targets && batch > 0 && steps >= 0, OLPT_ERR_INVALID_ARG,
                 "mlp_train: bad arguments");
    MlpWork& W = ctx->mlp;
    cudaStream_t s = ctx->stream;
    const float* dx = x;
    const float* dt = targets;
    if (!on_device) {
      W.ds_x.ensure((size_t)n * ctx->mlp.dims.in * 4, s);
      W.ds_t.ensure((size_t)n * kMlpOut * 4, s);
      OLPT_CUDA(cudaMemcpyAsync(W.ds_x.p, x, (size_t)n * ctx->mlp.dims.in * 4, cudaMemcpyHostToDevice, s));
      OLPT_CUDA(cudaMemcpyAsync(W.ds_t.p, targets, (size_t)n * kMlpOut * 4, cudaMemcpyHostToDevice,
                                s));
      dx = W.ds_x.as<float>();
      dt = W.ds_t.as<float>();
    }
    mlp_train_many(ctx, dx, dt, n, batch, steps, lr, ghost_weight, seed, losses);
    OLPT_CUDA(cudaStreamSynchronize(s));
  });
}

olpt_status_t olpt_mlp_features(olpt_ctx* ctx, const olpt_shake_params* p, float* x,
                                int on_device) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    const ShakeParams sp = to_shake_params(p);
    const int64_t n = ctx->obj.n;
    if (n == 0) return;
    OLPT_REQUIRE(x, OLPT_ERR_INVALID_ARG, "null output");
    mlp_sync_dims(ctx);
    residual_all_device(ctx, sp);
    MlpWork& W = ctx->mlp;
    cudaStream_t s = ctx->stream;
    W.x.ensure((size_t)n * ctx->mlp.dims.in_pad * 2, s);
    float* f = x;
    if (!on_device) {
      W.xin.ensure((size_t)n * ctx->mlp.dims.in * 4, s);
      f = W.xin.as<float>();
    }
    mlp_features_device(ctx, sp, W.x.as<__nv_bfloat16>(), f);
    if (!on_device)
      OLPT_CUDA(cudaMemcpyAsync(x, f, (size_t)n * ctx->mlp.dims.in * 4, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
  });
}

olpt_status_t olpt_learned_configure(olpt_ctx* ctx, const olpt_learned_params* p) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    OLPT_REQUIRE(p->out_scale_mm > 0 && p->refine_loops >= 0 && p->refine_width_mm >= 0,
                 OLPT_ERR_INVALID_ARG, "learned params out of range");
    OLPT_REQUIRE(!p->enable || ctx->mlp.ready, OLPT_ERR_INVALID_ARG,
                 "learned shake enabled before the network was initialised");
    LearnedParams& lp = ctx->mlp.lp;
    lp.enable = p->enable;
    lp.out_scale_mm = p->out_scale_mm;
    lp.ghost_logit = p->ghost_logit;
    lp.refine_loops = p->refine_loops;
    lp.refine_width_mm = p->refine_width_mm;
    lp.fallback_residual = p->fallback_residual;
  });
}

olpt_status_t olpt_shake_learned(olpt_ctx* ctx, const olpt_shake_params* p) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(p, OLPT_ERR_INVALID_ARG, "null params");
    learned_shake_device(ctx, to_shake_params(p));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

olpt_status_t olpt_learned_stats(olpt_ctx* ctx, int64_t* n_learned, int64_t* n_fallback) {
  return guard(ctx, [&] {
    if (n_learned) *n_learned = ctx->mlp.n_learned;
    if (n_fallback) *n_fallback = ctx->mlp.n_fallback;
  });
}

olpt_status_t olpt_bf16_gemm(olpt_ctx* ctx, int M, int N, int K, const uint16_t* A,
                             const uint16_t* B, const float* bias, int gelu, float* out) {
  return guard(ctx, [&] {
    OLPT_REQUIRE(M > 0 && N > 0 && K > 0 && A && B && out, OLPT_ERR_INVALID_ARG,
                 "bf16_gemm: bad arguments");
    cudaStream_t s = ctx->stream;
    const int ld = (K + 7) / 8 * 8;
    DevBuf dA, dB, dBias, dO, dErr;
    dA.ensure((size_t)M * ld * 2, s);
    dB.ensure((size_t)N * ld * 2, s);
    dO.ensure((size_t)M * N * 4, s);
    dErr.ensure(16, s);
    OLPT_CUDA(cudaMemsetAsync(dErr.p, 0, 16, s));
    OLPT_CUDA(cudaMemcpy2DAsync(dA.p, (size_t)ld * 2, A, (size_t)K * 2, (size_t)K * 2, M,
                                cudaMemcpyHostToDevice, s));
    OLPT_CUDA(cudaMemcpy2DAsync(dB.p, (size_t)ld * 2, B, (size_t)K * 2, (size_t)K * 2, N,
                                cudaMemcpyHostToDevice, s));
    GemmEpilogue e;
    if (bias) {
      dBias.ensure((size_t)N * 4, s);
      OLPT_CUDA(cudaMemcpyAsync(dBias.p, bias, (size_t)N * 4, cudaMemcpyHostToDevice, s));
      e.bias = dBias.as<float>();
    }
    e.out_f32 = dO.as<float>();
    e.ld_f32 = N;
    e.gelu = false;
    gemm_bf16(dA.as<__nv_bfloat16>(), ld, dB.as<__nv_bfloat16>(), ld, M, N, K, e, 1,
              dErr.as<int>(), s);
    if (gelu) gelu_inplace_device(dO.as<float>(), (int64_t)M * N, s);
    int err = 0;
    OLPT_CUDA(cudaMemcpyAsync(&err, dErr.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(out, dO.p, (size_t)M * N * 4, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    for (DevBuf* b : {&dA, &dB, &dBias, &dO, &dErr}) b->release(s);
    OLPT_REQUIRE(err == 0, OLPT_ERR_TIMEOUT, "tensor-core GEMM: a pipeline wait timed out");
  });
}

}  // extern "C"
