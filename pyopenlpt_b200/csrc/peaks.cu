// Kernel family (a): 2D tracer detection with sub-pixel Gaussian fit.
//
// Reference: ObjectFinder2D::findTracer2D (src/srcObject/ObjectFinder.cpp:37-111) and
// myMATH::isLocalMax (inc/libMath/myMATH.h:399-435).
//
// Layout: each camera image is one HBM plane with a 16-byte aligned row pitch.  A CTA
// owns a band of whole rows; its threads walk the band in raster order, one 16-byte
// chunk (16 u8 / 8 u16 / 4 f32 / 2 f64 pixels) per thread per round, with the rows
// above and below read as 16-byte vectors too.  Detection is two passes over the
// same bands: COUNT writes one count per band, a per-camera scan turns counts into
// offsets, EMIT re-evaluates the band and writes each detection at
// offset + block-scan rank, which reproduces the reference's raster order exactly
// without atomics.  The second read of a band hits L2 (a 6 x 2048^2 u16 frame is 48 MB).
//
// Exactness: integer-level images use a host-built table of ln(max(v, 1e-4)) (the
// same libm log the reference calls); the fit then evaluates the reference's
// expressions in the same order with no FMA contraction, so sub-pixel centres are
// bit-identical.  Floating-point images (residuals) call CUDA's log.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "olpt_ctx.cuh"

namespace olpt {
namespace {

constexpr int kPeakThreads = 256;

struct PeakCam {
  const unsigned char* img;
  int64_t pitch;  // bytes
  int H, W;
  int band_rows;
  int n_bands;
  int band_base;
  int active;
  double* x;
  double* y;
  int2* rc;
};

struct PeakArgs {
  int n_cam;
  PeakCam cam[OLPT_MAX_CAM];
  double min_int;
  const double* lut;  // integer images only
  int* band_counts;
  const int64_t* band_offsets;
};

template <typename T>
struct Ln;
template <>
struct Ln<uint8_t> {
  static __device__ __forceinline__ double f(uint8_t v, const double* lut) { return lut[v]; }
};
template <>
struct Ln<uint16_t> {
  static __device__ __forceinline__ double f(uint16_t v, const double* lut) { return lut[v]; }
};
template <>
struct Ln<float> {
  static __device__ __forceinline__ double f(float v, const double*) {
    double d = (double)v;
    return log(d < 1e-4 ? 1e-4 : d);
  }
};
template <>
struct Ln<double> {
  static __device__ __forceinline__ double f(double v, const double*) {
    return log(v < 1e-4 ? 1e-4 : v);
  }
};

// Load N consecutive pixels starting at column c0 of row r (c0 .. c0+N-1 may run past W).
template <typename T, int N>
__device__ __forceinline__ void load_chunk(const PeakCam& c, int r, int c0, T (&v)[N]) {
  const T* row = reinterpret_cast<const T*>(c.img + (int64_t)r * c.pitch);
  if (c0 + N <= c.W) {
    uint4 q = __ldg(reinterpret_cast<const uint4*>(row + c0));
    const T* qt = reinterpret_cast<const T*>(&q);
#pragma unroll
    for (int j = 0; j < N; ++j) v[j] = qt[j];
  } else {
#pragma unroll
    for (int j = 0; j < N; ++j) v[j] = (c0 + j < c.W) ? __ldg(row + c0 + j) : T(0);
  }
}

// Sub-pixel centre along one axis: the reference's 3-point log-parabola
// (ObjectFinder.cpp:70-97) in absolute pixel coordinates.
__device__ __forceinline__ bool fit3(double l1, double l2, double l3, int p, double& out) {
  const int p1 = p - 1, p2 = p, p3 = p + 1;
  const double num = l1 * (double)((p2 * p2) - (p3 * p3)) - l2 * (double)((p1 * p1) - (p3 * p3)) +
                     l3 * (double)((p1 * p1) - (p2 * p2));
  const double den = l1 * (double)(p3 - p2) - l3 * (double)(p1 - p2) + l2 * (double)(p1 - p3);
  if (den == 0.0) return false;
  const double c = -0.5 * (num / den);
  if (!isfinite(c)) return false;
  out = c;
  return true;
}

// Evaluate one chunk; returns a bitmask of detections (bit j = pixel c0 + j) and
// fills xs/ys for them when EMIT.
template <typename T, int N, bool EMIT>
__device__ __forceinline__ unsigned eval_chunk(const PeakCam& c, const PeakArgs& a, int r, int c0,
                                               double (&xs)[N], double (&ys)[N]) {
  if (r < 1 || r > c.H - 2) return 0u;
  T cen[N];
  load_chunk<T, N>(c, r, c0, cen);
  // quick reject: nothing in the chunk reaches the threshold
  bool any = false;
#pragma unroll
  for (int j = 0; j < N; ++j) any |= !((double)cen[j] < a.min_int);
  if (!any) return 0u;
  T up[N], dn[N];
  load_chunk<T, N>(c, r - 1, c0, up);
  load_chunk<T, N>(c, r + 1, c0, dn);
  const T* row = reinterpret_cast<const T*>(c.img + (int64_t)r * c.pitch);
  const T left = (c0 > 0) ? __ldg(row + c0 - 1) : T(0);
  const T right = (c0 + N < c.W) ? __ldg(row + c0 + N) : T(0);
  unsigned mask = 0u;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const int col = c0 + j;
    if (col < 1 || col > c.W - 2) continue;
    const T v = cen[j];
    if ((double)v < a.min_int) continue;
    const T l = (j > 0) ? cen[j - 1] : left;
    const T rr = (j < N - 1) ? cen[j + 1] : right;
    // isLocalMax tie rule: up/left reject if strictly greater, down/right if >=.
    if (up[j] > v || l > v || dn[j] >= v || rr >= v) continue;
    const double lc = Ln<T>::f(v, a.lut);
    double xc, yc;
    if (!fit3(Ln<T>::f(l, a.lut), lc, Ln<T>::f(rr, a.lut), col, xc)) continue;
    if (!fit3(Ln<T>::f(up[j], a.lut), lc, Ln<T>::f(dn[j], a.lut), r, yc)) continue;
    if (EMIT) {
      xs[j] = xc;
      ys[j] = yc;
    }
    mask |= 1u << j;
  }
  return mask;
}

__device__ __forceinline__ int find_cam(const PeakArgs& a, int blk) {
  int cam = 0;
  for (int i = 1; i < a.n_cam; ++i)
    if (blk >= a.cam[i].band_base) cam = i;
  return cam;
}

template <typename T, bool EMIT>
__global__ void __launch_bounds__(kPeakThreads) peaks_kernel(const PeakArgs a) {
  constexpr int N = 16 / sizeof(T);
  const int cam = find_cam(a, blockIdx.x);
  const PeakCam& c = a.cam[cam];
  const int band = blockIdx.x - c.band_base;
  if (!c.active || band >= c.n_bands) return;
  const int cpr = (c.W + N - 1) / N;  // chunks per row
  const int r0 = band * c.band_rows;
  const int rows = min(c.band_rows, c.H - r0);
  const int total = rows * cpr;

  __shared__ int warp_sums[kPeakThreads / 32];
  __shared__ int s_base;
  int64_t base = 0;
  if (EMIT) base = a.band_offsets[blockIdx.x];
  int running = 0;
  int count = 0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int start = 0; start < total; start += kPeakThreads) {
    const int i = start + threadIdx.x;
    double xs[N], ys[N];
    unsigned mask = 0u;
    int r = 0, c0 = 0;
    if (i < total) {
      r = r0 + i / cpr;
      c0 = (i % cpr) * N;
      mask = eval_chunk<T, N, EMIT>(c, a, r, c0, xs, ys);
    }
    const int n = __popc(mask);
    if (!EMIT) {
      count += n;
      continue;
    }
    // block-wide exclusive scan of n in thread (= raster) order
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int w = 0; w < kPeakThreads / 32; ++w) {
        int t = warp_sums[w];
        warp_sums[w] = acc;
        acc += t;
      }
      s_base = acc;
    }
    __syncthreads();
    int pos = running + warp_sums[wid] + incl - n;
    if (mask) {
      for (int j = 0; j < N; ++j) {
        if (mask & (1u << j)) {
          const int64_t o = base + pos;
          c.x[o] = xs[j];
          c.y[o] = ys[j];
          c.rc[o] = make_int2(r, c0 + j);
          ++pos;
        }
      }
    }
    running += s_base;
    __syncthreads();
  }
  if (!EMIT) {
    // block reduction of count
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) count += __shfl_down_sync(0xffffffffu, count, o);
    if (lane == 0) warp_sums[wid] = count;
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int w = 0; w < kPeakThreads / 32; ++w) acc += warp_sums[w];
      a.band_counts[blockIdx.x] = acc;
    }
  }
}

// Per-camera exclusive scan of band counts -> band offsets, and totals.
__global__ void band_scan_kernel(const PeakArgs a, int64_t* band_offsets, int64_t* totals) {
  const int cam = blockIdx.x;
  if (cam >= a.n_cam) return;
  const PeakCam& c = a.cam[cam];
  __shared__ int64_t s_run, s_total;
  __shared__ int64_t warp_sums[32];
  if (threadIdx.x == 0) s_run = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int s = 0; s < c.n_bands; s += blockDim.x) {
    const int b = s + threadIdx.x;
    int64_t v = (b < c.n_bands && c.active) ? a.band_counts[c.band_base + b] : 0;
    int64_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t acc = 0;
      for (int w = 0; w < nw; ++w) {
        int64_t t = warp_sums[w];
        warp_sums[w] = acc;
        acc += t;
      }
      s_total = acc;
    }
    __syncthreads();
    if (b < c.n_bands) band_offsets[c.band_base + b] = s_run + warp_sums[wid] + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) s_run += s_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) totals[cam] = s_run;
}

template <typename T>
void launch_peaks(const PeakArgs& a, int n_blocks, int64_t* band_offsets, int64_t* totals,
                  cudaStream_t s) {
  peaks_kernel<T, false><<<OLPT_G(n_blocks), kPeakThreads, 0, s>>>(a);
  OLPT_CUDA(cudaGetLastError());
  band_scan_kernel<<<OLPT_G(a.n_cam), 256, 0, s>>>(a, band_offsets, totals);
  OLPT_CUDA(cudaGetLastError());
  PeakArgs b = a;
  b.band_offsets = band_offsets;
  peaks_kernel<T, true><<<OLPT_G(n_blocks), kPeakThreads, 0, s>>>(b);
  OLPT_CUDA(cudaGetLastError());
}

}  // namespace

void ensure_log_luts(olpt_ctx* ctx) {
  if (ctx->lut_u8.p) return;
  std::vector<double> t(65536);
  for (int v = 0; v < 65536; ++v) {
    const double d = (double)v;
    t[v] = std::log(d < 1e-4 ? 1e-4 : d);  // ObjectFinder.cpp:54-57 safe_ln
  }
  ctx->lut_u8.ensure(256 * sizeof(double), ctx->stream);
  ctx->lut_u16.ensure(65536 * sizeof(double), ctx->stream);
  OLPT_CUDA(cudaMemcpyAsync(ctx->lut_u8.p, t.data(), 256 * sizeof(double), cudaMemcpyHostToDevice,
                            ctx->stream));
  OLPT_CUDA(cudaMemcpyAsync(ctx->lut_u16.p, t.data(), 65536 * sizeof(double),
                            cudaMemcpyHostToDevice, ctx->stream));
  OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
}

void ensure_det_capacity(olpt_ctx* ctx, int cam, int64_t cap) {
  Dets& d = ctx->dets[cam];
  if (d.cap >= cap) return;
  d.x.ensure(cap * sizeof(double), ctx->stream);
  d.y.ensure(cap * sizeof(double), ctx->stream);
  d.rc.ensure(cap * sizeof(int2), ctx->stream);
  d.cap = cap;
}

// Detect on the current images; counts stay on the device in ctx->det_counts and are
// mirrored to det_counts_h when `sync_counts`.
void find_peaks_device(olpt_ctx* ctx, double min_int, bool sync_counts) {
  OLPT_REQUIRE(ctx->n_cam > 0, OLPT_ERR_INVALID_ARG, "no cameras uploaded");
  ensure_log_luts(ctx);
  PeakArgs a{};
  a.n_cam = ctx->n_cam;
  a.min_int = min_int;
  int dtype = -1;
  int blocks = 0;
  for (int c = 0; c < ctx->n_cam; ++c) {
    ImagePlane& im = ctx->img[c];
    OLPT_REQUIRE(im.buf.p != nullptr, OLPT_ERR_INVALID_ARG, "no image uploaded for camera");
    if (dtype < 0) dtype = im.dtype;
    OLPT_REQUIRE(im.dtype == dtype, OLPT_ERR_INVALID_ARG, "all cameras must share one dtype");
    const int esz = dtype == OLPT_U8 ? 1 : dtype == OLPT_U16 ? 2 : dtype == OLPT_F32 ? 4 : 8;
    const int N = 16 / esz;
    const int cpr = (im.W + N - 1) / N;
    int band_rows = (2048 + cpr - 1) / cpr;
    if (band_rows < 1) band_rows = 1;
    PeakCam& pc = a.cam[c];
    pc.img = im.buf.as<unsigned char>();
    pc.pitch = im.pitch;
    pc.H = im.H;
    pc.W = im.W;
    pc.band_rows = band_rows;
    pc.n_bands = (im.H + band_rows - 1) / band_rows;
    pc.band_base = blocks;
    pc.active = ctx->cams_h[c].is_active;
    blocks += pc.n_bands;
    ensure_det_capacity(ctx, c, ((int64_t)im.H * im.W + 1) / 2 + 1);
    pc.x = ctx->dets[c].x.as<double>();
    pc.y = ctx->dets[c].y.as<double>();
    pc.rc = ctx->dets[c].rc.as<int2>();
  }
  ctx->band_counts.ensure(blocks * sizeof(int), ctx->stream);
  ctx->band_offsets.ensure(blocks * sizeof(int64_t), ctx->stream);
  ctx->det_counts.ensure(OLPT_MAX_CAM * sizeof(int64_t), ctx->stream);
  a.band_counts = ctx->band_counts.as<int>();
  int64_t* offs = ctx->band_offsets.as<int64_t>();
  int64_t* tot = ctx->det_counts.as<int64_t>();
  double img_bytes = 0;
  for (int c = 0; c < ctx->n_cam; ++c)
    if (a.cam[c].active)
      img_bytes += (double)a.cam[c].H * a.cam[c].W *
                   (dtype == OLPT_U8 ? 1 : dtype == OLPT_U16 ? 2 : dtype == OLPT_F32 ? 4 : 8);
  const int pid = ctx->prof.begin(PROF_PEAKS, ctx->stream);
  switch (dtype) {
    case OLPT_U8:
      a.lut = ctx->lut_u8.as<double>();
      launch_peaks<uint8_t>(a, blocks, offs, tot, ctx->stream);
      break;
    case OLPT_U16:
      a.lut = ctx->lut_u16.as<double>();
      launch_peaks<uint16_t>(a, blocks, offs, tot, ctx->stream);
      break;
    case OLPT_F32:
      launch_peaks<float>(a, blocks, offs, tot, ctx->stream);
      break;
    default:
      launch_peaks<double>(a, blocks, offs, tot, ctx->stream);
      break;
  }
  ctx->prof.end(PROF_PEAKS, pid, ctx->stream, img_bytes);
  ctx->det_counts_h.assign(ctx->n_cam, 0);
  if (sync_counts) {
    OLPT_CUDA(cudaMemcpyAsync(ctx->det_counts_h.data(), tot, ctx->n_cam * sizeof(int64_t),
                              cudaMemcpyDeviceToHost, ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
  }
}

// ---------------------------------------------------------------------------
// Allocation-free detection for callers that cannot allocate device memory:
// code running inside a host-side memory arena or pool that forbids outside
// allocations, code that must not perturb another framework's caching allocator,
// or plug-in hosts whose device memory is budgeted by someone else.  Their scratch
// (the per-band counts and offsets of the two-pass raster compaction) and the
// log table for integer images live in these file-scope device arrays, which every
// GPU that loads this library holds until the process exits.
constexpr int kNoAllocMaxBands = 16384;  // one band per row at most: images up to 16384 rows
constexpr int kNoAllocMaxCols = 16384;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocMaxBands * (4 + 8) + 256];
static __device__ __align__(256) double g_noalloc_log_lut[65536];

namespace {
struct NoAllocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  double* lut = nullptr;             // device address of g_noalloc_log_lut
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[64];
}  // namespace

// Once per device, with that device current: resolve the arrays' device addresses
// (in host code their names are host-side stand-ins, not device addresses) and fill
// the log table.  Synchronous; must run before any stream capture.
static olpt_status_t noalloc_setup(int dev, NoAllocDevice*& out, std::string& err) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= 64) {
    err = "device ordinal out of range";
    return OLPT_ERR_INVALID_ARG;
  }
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (!d.ready) {
    cudaError_t e = cudaGetSymbolAddress((void**)&d.scratch, g_noalloc_scratch);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.lut, g_noalloc_log_lut);
    if (e != cudaSuccess) {
      err = std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
      return OLPT_ERR_CUDA;
    }
    std::vector<double> t(65536);
    for (int v = 0; v < 65536; ++v) {
      const double x = (double)v;
      t[v] = std::log(x < 1e-4 ? 1e-4 : x);
    }
    e = cudaMemcpy(d.lut, t.data(), sizeof(double) * 65536, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      err = std::string("log table upload failed: ") + cudaGetErrorString(e);
      return OLPT_ERR_CUDA;
    }
    d.ready = true;
  }
  out = &d;
  return OLPT_OK;
}

thread_local std::string g_noalloc_err;

}  // namespace olpt

extern "C" {

const char* olpt_find_peaks_noalloc_error(void) { return olpt::g_noalloc_err.c_str(); }

olpt_status_t olpt_find_peaks_noalloc(const void* d_img, olpt_dtype_t dtype, int H, int W,
                                      int64_t pitch_bytes, double min_obj_int, double* d_x,
                                      double* d_y, int32_t* d_rc, int64_t capacity,
                                      int64_t* d_count, void* stream) {
  using namespace olpt;
  std::string& err = g_noalloc_err;
  err.clear();
  if (!d_img || !d_x || !d_y || !d_rc || !d_count) {
    err = "null buffer";
    return OLPT_ERR_INVALID_ARG;
  }
  if (dtype < OLPT_U8 || dtype > OLPT_F64) {
    err = "bad dtype";
    return OLPT_ERR_INVALID_ARG;
  }
  const int esz = dtype == OLPT_U8 ? 1 : dtype == OLPT_U16 ? 2 : dtype == OLPT_F32 ? 4 : 8;
  if (H < 1 || W < 1 || H > kNoAllocMaxBands || W > kNoAllocMaxCols) {
    err = "image must be 1..16384 rows and 1..16384 columns for the allocation-free detector";
    return OLPT_ERR_INVALID_ARG;
  }
  if (pitch_bytes < (int64_t)W * esz || pitch_bytes % 16 != 0 ||
      reinterpret_cast<uintptr_t>(d_img) % 16 != 0) {
    err = "image rows must start on 16-byte boundaries (pitch a multiple of 16, >= W * elem)";
    return OLPT_ERR_INVALID_ARG;
  }
  if (capacity < ((int64_t)H * W + 1) / 2) {
    err = "capacity must be at least (H * W + 1) / 2 (the most 4-neighbour maxima an image can hold)";
    return OLPT_ERR_INVALID_ARG;
  }
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) {
    err = cudaGetErrorString(ce);
    return OLPT_ERR_CUDA;
  }
  NoAllocDevice* nd = nullptr;
  olpt_status_t st = noalloc_setup(dev, nd, err);
  if (st != OLPT_OK) return st;
  try {
    const int N = 16 / esz;
    const int cpr = (W + N - 1) / N;
    int band_rows = (2048 + cpr - 1) / cpr;
    if (band_rows < 1) band_rows = 1;
    PeakArgs a{};
    a.n_cam = 1;
    a.min_int = min_obj_int;
    PeakCam& pc = a.cam[0];
    pc.img = static_cast<const unsigned char*>(d_img);
    pc.pitch = pitch_bytes;
    pc.H = H;
    pc.W = W;
    pc.band_rows = band_rows;
    pc.n_bands = (H + band_rows - 1) / band_rows;
    pc.band_base = 0;
    pc.active = 1;
    pc.x = d_x;
    pc.y = d_y;
    pc.rc = reinterpret_cast<int2*>(d_rc);
    // scratch layout: band offsets (int64) then band counts (int); every band count
    // that the scan reads is written by this call's count pass first.
    int64_t* offs = reinterpret_cast<int64_t*>(nd->scratch);
    a.band_counts = reinterpret_cast<int*>(nd->scratch + sizeof(int64_t) * kNoAllocMaxBands);
    a.lut = nd->lut;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (dtype) {
      case OLPT_U8: launch_peaks<uint8_t>(a, pc.n_bands, offs, d_count, s); break;
      case OLPT_U16: launch_peaks<uint16_t>(a, pc.n_bands, offs, d_count, s); break;
      case OLPT_F32: launch_peaks<float>(a, pc.n_bands, offs, d_count, s); break;
      default: launch_peaks<double>(a, pc.n_bands, offs, d_count, s); break;
    }
  } catch (CudaError const& e) {
    err = std::string(cudaGetErrorString(e.code)) + " (" + e.where + ")";
    return OLPT_ERR_CUDA;
  }
  return OLPT_OK;
}

}  // extern "C"
