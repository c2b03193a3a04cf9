// Kernel family (a): 2D tracer detection with sub-pixel Gaussian fit.
//
// Reference: ObjectFinder2D::findTracer2D (src/srcObject/ObjectFinder.cpp:37-111) and
// myMATH::isLocalMax (inc/libMath/myMATH.h:399-435).
//
// Layout: each camera image is one HBM plane with a 16-byte aligned row pitch.  A CTA
// owns a band of whole rows.
//
// Staged detector (detect_kernel, the production path): one read of the image.  The
// CTA takes a band ticket, TMA-loads its band plus one halo row above and below into
// shared memory (boxes of 256 columns, zero fill outside the image), evaluates every
// 16-byte chunk (16 u8 / 8 u16 / 4 f32 / 2 f64 pixels) from shared memory, ranks its
// detections in raster order with a block scan, learns the detections of the bands
// before it by a decoupled look-back over per-band states (aggregate / inclusive
// prefix, published with release stores), and writes each detection at prefix +
// rank: the reference's raster order without a second pass over the image.  Tickets
// are handed out in band order, so a band only waits on bands whose CTAs are already
// running; every wait is bounded and a timeout is reported through an error word.
//
// Two-pass detector (peaks_kernel; allocation-free entry point and images too wide to
// stage three rows of in shared memory): COUNT writes one count per band, a
// per-camera scan turns counts into offsets, EMIT re-evaluates the band from global
// memory and writes each detection at offset + block-scan rank.
//
// Exactness: integer-level images use a host-built table of ln(max(v, 1e-4)) (the
// same libm log the reference calls); the fit then evaluates the reference's
// expressions in the same order with no FMA contraction, so sub-pixel centres are
// bit-identical.  Floating-point images (residuals) call CUDA's log.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_umma.cuh"

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
  static __device__ __forceinline__ double f(uint8_t v, const double* lut) { return __ldg(lut + v); }
};
template <>
struct Ln<uint16_t> {
  static __device__ __forceinline__ double f(uint16_t v, const double* lut) {
    return __ldg(lut + v);
  }
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


// ---------------------------------------------------------------------------
// Staged single-read detector.

constexpr int kDetThreads = 256;
constexpr int kBoxW = 256;  // TMA box width in elements (the hardware maximum)
constexpr int kDetList = 2048;  // detections listed per emission round
// det_counts words after the per-camera totals
constexpr int kDcErr = OLPT_MAX_CAM, kDcTicket = OLPT_MAX_CAM + 1, kDcState = OLPT_MAX_CAM + 2;
// look-back state of a band: flag in the top two bits, detection count below
constexpr unsigned long long kStAggregate = 1ull << 62, kStPrefix = 2ull << 62;
constexpr unsigned long long kStValue = (1ull << 62) - 1;

struct DetCam {
  int H, W;
  int band_rows;  // R: rows per band; the staged tile holds R + 2 rows
  int box_w;      // columns per box: 256, or the row's chunk-padded width if one box covers it
  int n_box;      // boxes per row
  int cpr;        // 16-byte chunks per row
  int n_bands, band_base;
  double* x;
  double* y;
  int2* rc;
};

struct DetArgs {
  CUtensorMap map[OLPT_MAX_CAM];
  DetCam cam[OLPT_MAX_CAM];
  int n_cam;
  double min_int;
  int min_level;            // integer images: v < min_level  <=>  (double)v < min_int
  const double* lut;        // integer images only
  unsigned long long* dc;   // det_counts words
  // failure-detection tests only (olpt_test_hold_detection_band): the band with this
  // ticket never publishes its count, and the look-back waits give up after
  // wait_limit_ns; -1 / the default limit otherwise
  int hold_ticket;
  unsigned long long wait_limit_ns;
};

// A band state is read as one word (flag and count together), so a relaxed load is
// enough: nothing else that the publishing CTA wrote is read through it.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Element (tile row lr, image column col) of a staged band: boxes of box_w columns,
// each box_h rows of box_w elements, box after box.
template <typename T>
__device__ __forceinline__ int tile_index(const DetCam& c, int box_h, int lr, int col) {
  return ((col >> 8) * box_h + lr) * c.box_w + (col & (kBoxW - 1));
}

// One chunk of image row r (tile row lr) from shared memory: bit j set if pixel c0 + j
// passes eval_chunk's tests and fit.  Pixels at or past W are the TMA's zero fill, as
// eval_chunk's loads.
// Threshold test of one pixel: (double)v < min_int, for integer levels as the integer
// compare v < min_level (the same outcome for every level and every min_int).
template <typename T>
__device__ __forceinline__ bool below(T v, double min_int, int min_level) {
  if constexpr (std::is_integral<T>::value) {
    return (int)v < min_level;
  } else {
    return (double)v < min_int;
  }
}

template <typename T, int N>
__device__ __forceinline__ unsigned mask_staged(const T* tile, const DetCam& c, int box_h,
                                                double min_int, int min_level, const double* lut,
                                                int r, int lr, int c0) {
  if (r < 1 || r > c.H - 2) return 0u;
  T cen[N], up[N], dn[N];
  const int ic = tile_index<T>(c, box_h, lr, c0);
  {
    const uint4 q = *reinterpret_cast<const uint4*>(tile + ic);
    const T* qt = reinterpret_cast<const T*>(&q);
#pragma unroll
    for (int j = 0; j < N; ++j) cen[j] = qt[j];
  }
  bool any = false;
#pragma unroll
  for (int j = 0; j < N; ++j) any |= !below<T>(cen[j], min_int, min_level);
  if (!any) return 0u;
  {
    const uint4 qu = *reinterpret_cast<const uint4*>(tile + ic - c.box_w);
    const uint4 qd = *reinterpret_cast<const uint4*>(tile + ic + c.box_w);
    const T* tu = reinterpret_cast<const T*>(&qu);
    const T* td = reinterpret_cast<const T*>(&qd);
#pragma unroll
    for (int j = 0; j < N; ++j) {
      up[j] = tu[j];
      dn[j] = td[j];
    }
  }
  const int wpad = c.n_box * c.box_w;
  const T left = (c0 > 0) ? tile[tile_index<T>(c, box_h, lr, c0 - 1)] : T(0);
  const T right = (c0 + N < wpad) ? tile[tile_index<T>(c, box_h, lr, c0 + N)] : T(0);
  unsigned cand = 0u;  // threshold and local-maximum tests
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const int col = c0 + j;
    if (col < 1 || col > c.W - 2) continue;
    const T v = cen[j];
    if (below<T>(v, min_int, min_level)) continue;
    const T l = (j > 0) ? cen[j - 1] : left;
    const T rr = (j < N - 1) ? cen[j + 1] : right;
    if (up[j] > v || l > v || dn[j] >= v || rr >= v) continue;
    cand |= 1u << j;
  }
  // Integer levels: a local maximum has v >= 1 and ln(left), ln(up) <= ln(v) >
  // ln(right), ln(down) (ln(max(x, 1e-4)) increases strictly over the integers), so
  // both fits have a negative denominator and a finite centre: every candidate is a
  // detection.  Floating-point levels can tie in the clamped log or be non-finite.
  if constexpr (std::is_integral<T>::value) return cand;
  unsigned mask = 0u;  // the fit of each candidate (one loop iteration per candidate)
  while (cand) {
    const int j = __ffs(cand) - 1;
    cand &= cand - 1;
    const int col = c0 + j;
    const T v = tile[ic + j];
    const T l = tile[tile_index<T>(c, box_h, lr, col - 1)];
    const T rr = tile[tile_index<T>(c, box_h, lr, col + 1)];
    const double lc = Ln<T>::f(v, lut);
    double xc, yc;
    if (!fit3(Ln<T>::f(l, lut), lc, Ln<T>::f(rr, lut), col, xc)) continue;
    if (!fit3(Ln<T>::f(tile[ic + j - c.box_w], lut), lc, Ln<T>::f(tile[ic + j + c.box_w], lut), r,
              yc))
      continue;
    mask |= 1u << j;
  }
  return mask;
}


// One chunk of integer levels: bit j set if pixel c0 + j passes the threshold and the
// isLocalMax tie rule (up / left reject if strictly greater, down / right if >=).
// qc: the chunk (the chunks above and below are read only if a pixel passes the
// threshold); left / right: the pixels beside it (0 outside the image, as the zero
// fill); cols: the interior-column bits.
template <typename T>
__device__ __forceinline__ unsigned mask_int(const uint4& qc, const T* tile, int ic, int box_w,
                                             uint32_t left, uint32_t right, int min_level,
                                             unsigned cols) {
  constexpr int N = 16 / sizeof(T);  // pixels per chunk
  const T* cen = reinterpret_cast<const T*>(&qc);
  unsigned cand = 0u;
#pragma unroll
  for (int j = 0; j < N; ++j) cand |= (unsigned)((int)cen[j] >= min_level) << j;
  cand &= cols;
  if (!cand) return 0u;
  const uint4 qu = *reinterpret_cast<const uint4*>(tile + ic - box_w);
  const uint4 qd = *reinterpret_cast<const uint4*>(tile + ic + box_w);
  const T* up = reinterpret_cast<const T*>(&qu);
  const T* dn = reinterpret_cast<const T*>(&qd);
  unsigned mask = 0u;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const uint32_t v = cen[j];
    const uint32_t l = j > 0 ? (uint32_t)cen[j - 1] : left;
    const uint32_t rr = j < N - 1 ? (uint32_t)cen[j + 1] : right;
    mask |= (unsigned)((uint32_t)up[j] <= v && l <= v && (uint32_t)dn[j] < v && rr < v) << j;
  }
  return mask & cand;
}

template <typename T>
__global__ void __launch_bounds__(kDetThreads, 3) detect_kernel(const __grid_constant__ DetArgs a) {
  constexpr int N = 16 / sizeof(T);
  // declared with the alignment the runtime guarantees (dynamic shared memory follows
  // the static variables), so the rounding below is computed, not assumed away
  extern __shared__ __align__(16) unsigned char det_smem[];
  __shared__ uint64_t bar;
  __shared__ int s_ticket, s_ok;
  __shared__ int s_warp[kDetThreads / 32];
  __shared__ long long s_prefix;
  __shared__ int s_total;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  unsigned long long* dc = a.dc;

  if (tid == 0) {
    umma::mbar_init(&bar, 1);
    umma::fence_barrier_init();
    s_ticket = (int)atomicAdd(dc + kDcTicket, 1ull);
  }
  __syncthreads();
  const int tk = s_ticket;
  int cam = 0;
  for (int i = 0; i < a.n_cam; ++i)
    if (tk >= a.cam[i].band_base && tk < a.cam[i].band_base + a.cam[i].n_bands) cam = i;
  const DetCam& c = a.cam[cam];
  const int band = tk - c.band_base;
  const int box_h = c.band_rows + 2;
  const int r0 = band * c.band_rows;
  const int rows = min(c.band_rows, c.H - r0);
  // TMA destinations are 128-byte aligned (every box is a multiple of 128 bytes)
  unsigned char* base = det_smem + ((128u - (umma::smem_u32(det_smem) & 127u)) & 127u);
  T* tile = reinterpret_cast<T*>(base);
  const int tile_elems = c.n_box * box_h * c.box_w;
  uint16_t* masks = reinterpret_cast<uint16_t*>(base + (size_t)tile_elems * sizeof(T));

  // stage the band with its halo rows (row r0 - 1 may be -1: zero fill)
  if (tid == 0) {
    const uint32_t box_bytes = (uint32_t)(box_h * c.box_w * (int)sizeof(T));
    umma::mbar_arrive_expect_tx(&bar, box_bytes * (uint32_t)c.n_box);
    for (int b = 0; b < c.n_box; ++b)
      umma::tma_load_2d(tile + (size_t)b * box_h * c.box_w, &a.map[cam], &bar, b * kBoxW, r0 - 1);
  }
  const bool staged = __syncthreads_and(umma::mbar_wait(&bar, 0)) != 0;
  unsigned long long* state = dc + kDcState + tk;
  if (!staged) {
    if (tid == 0) {
      atomicOr(dc + kDcErr, 1ull);
      umma::mbar_wait(&bar, 0);              // the copies must land before the CTA exits
      st_release_u64(state, kStPrefix);      // successors go on (results are void)
    }
    return;
  }

  // 1. evaluate every chunk of the band (coalesced over threads), keep the masks
  const int cpr = c.cpr;
  const int n_chunks = rows * cpr;
  if constexpr (std::is_integral<T>::value) {
    // chunk i = (lr - 1) * cpr + ci, stepped without divisions; a warp's lanes hold
    // consecutive chunks, so the pixels beside a chunk come from the neighbour lanes
    constexpr int kShift = 32 - 8 * (int)sizeof(T);
    constexpr uint32_t kLow = sizeof(T) == 1 ? 0xffu : 0xffffu;
    const int kMaxLevel = sizeof(T) == 1 ? 255 : 65535;
    int lr = 1 + tid / cpr, ci = tid % cpr;
    const int step_r = kDetThreads / cpr, step_c = kDetThreads % cpr;
    for (int i = tid; i - lane < n_chunks; i += kDetThreads) {  // warp-uniform condition
      const bool act = i < n_chunks;
      const int c0 = ci * N;
      const int ic = act ? tile_index<T>(c, box_h, lr, c0) : 0;
      const uint4 qc = act ? *reinterpret_cast<const uint4*>(tile + ic) : make_uint4(0, 0, 0, 0);
      const uint32_t prev = __shfl_up_sync(0xffffffffu, qc.w, 1);
      const uint32_t next = __shfl_down_sync(0xffffffffu, qc.x, 1);
      if (act) {
        const int r = r0 + lr - 1;
        unsigned m = 0u;
        if (r >= 1 && r <= c.H - 2 && a.min_level <= kMaxLevel) {
          uint32_t left = 0u, right = 0u;
          if (ci > 0)
            left = lane > 0 ? prev >> kShift : (uint32_t)tile[tile_index<T>(c, box_h, lr, c0 - 1)];
          if (ci + 1 < cpr)
            right = lane < 31 ? next & kLow : (uint32_t)tile[tile_index<T>(c, box_h, lr, c0 + N)];
          const int lo = max(0, 1 - c0), hi = min(N - 1, c.W - 2 - c0);
          const unsigned cols = hi < lo ? 0u : (((1u << (hi + 1)) - 1u) & ~((1u << lo) - 1u));
          m = cols ? mask_int<T>(qc, tile, ic, c.box_w, left, right, a.min_level, cols) : 0u;
        }
        masks[i] = (uint16_t)m;
      }
      lr += step_r;
      ci += step_c;
      if (ci >= cpr) {
        ci -= cpr;
        ++lr;
      }
    }
  } else {
    int lr = 1 + tid / cpr, ci = tid % cpr;
    const int step_r = kDetThreads / cpr, step_c = kDetThreads % cpr;
    for (int i = tid; i < n_chunks; i += kDetThreads) {
      masks[i] = (uint16_t)mask_staged<T, N>(tile, c, box_h, a.min_int, a.min_level, a.lut,
                                             r0 + lr - 1, lr, ci * N);
      lr += step_r;
      ci += step_c;
      if (ci >= cpr) {
        ci -= cpr;
        ++lr;
      }
    }
  }
  __syncthreads();

  // 2. raster-order ranks: thread t owns chunks [t K, t K + K)
  const int K = (n_chunks + kDetThreads - 1) / kDetThreads;
  const int i0 = min(tid * K, n_chunks), i1 = min(i0 + K, n_chunks);
  int n = 0;
  for (int i = i0; i < i1; ++i) n += __popc((unsigned)masks[i]);
  int incl = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int acc = 0;
    if (lane == 0) {
      for (int w = 0; w < kDetThreads / 32; ++w) {
        const int t = s_warp[w];
        s_warp[w] = acc;
        acc += t;
      }
    }
    const unsigned long long total = (unsigned long long)__shfl_sync(0xffffffffu, acc, 0);
    if (lane == 0) s_total = acc;
    const bool held = tk == a.hold_ticket;
    if (lane == 0 && !held) st_release_u64(state, (band == 0 ? kStPrefix : kStAggregate) | total);
    // 3. look-back over windows of 32 earlier bands: sum the aggregates down to the
    //    nearest published prefix (bands before the camera's first count as an empty
    //    prefix); wait while a band above that prefix has published nothing yet
    unsigned long long prefix = 0;
    int ok = 1;
    if (band > 0) {
      int top = tk - 1;
      uint64_t t0 = 0;
      while (true) {
        const int idx = top - 31 + lane;
        const unsigned long long w =
            idx >= c.band_base ? ld_relaxed_u64(dc + kDcState + idx) : kStPrefix;
        const unsigned long long flag = w & ~kStValue;
        const unsigned pmask = __ballot_sync(0xffffffffu, flag == kStPrefix);
        const int nearest = pmask ? 31 - __clz(pmask) : 0;  // highest lane with a prefix
        if (__any_sync(0xffffffffu, flag == 0 && lane > nearest - (pmask ? 0 : 1))) {
          int expired = 0;
          if (lane == 0) {
            const uint64_t now = umma::global_timer();
            if (t0 == 0) t0 = now;
            else if (now - t0 > a.wait_limit_ns) expired = 1;
          }
          if (__shfl_sync(0xffffffffu, expired, 0)) {
            if (lane == 0) atomicOr(dc + kDcErr, 2ull);
            ok = 0;
            break;
          }
          __nanosleep(64);
          continue;
        }
        unsigned long long v = lane >= nearest ? (w & kStValue) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        prefix += v;
        if (pmask) break;
        top -= 32;
      }
      if (lane == 0 && !held) st_release_u64(state, kStPrefix | (prefix + total));
    }
    if (held) ok = 0;
    if (lane == 0) {
      if (band == c.n_bands - 1) dc[cam] = prefix + total;
      s_prefix = (long long)prefix;
      s_ok = ok;
    }
  }
  __syncthreads();
  if (!s_ok) return;

  // 4. write the detections at prefix + rank, kDetList at a time: the block's
  //    detections are listed in rank order in shared memory, then fitted and written
  //    one per thread (coalesced stores, the fits spread over all threads)
  uint32_t* dlist = reinterpret_cast<uint32_t*>(
      base + (((size_t)tile_elems * sizeof(T) + (size_t)c.band_rows * cpr * sizeof(uint16_t) + 3) &
              ~(size_t)3));
  const int my0 = s_warp[wid] + incl - n;  // this thread's first rank in the block
  const int block_total = s_total;
  for (int lo = 0; lo < block_total; lo += kDetList) {
    if (my0 < lo + kDetList && my0 + n > lo) {
      int rank = my0;
      int lr = 1 + i0 / cpr, ci = i0 % cpr;
      for (int i = i0; i < i1 && rank < lo + kDetList; ++i) {
        unsigned m = masks[i];
        while (m) {
          const int j = __ffs(m) - 1;
          m &= m - 1;
          if (rank >= lo && rank < lo + kDetList)
            dlist[rank - lo] = ((uint32_t)lr << 16) | (uint32_t)(ci * N + j);  // tile row, column
          ++rank;
        }
        if (++ci == cpr) {
          ci = 0;
          ++lr;
        }
      }
    }
    __syncthreads();
    const int cnt = min(kDetList, block_total - lo);
    const int64_t base = s_prefix + lo;
    // three detections per thread at a time: their log lookups are in flight together
    constexpr int U = 3;
    for (int k0 = tid; k0 < cnt; k0 += U * kDetThreads) {
      int rr[U], cc[U];
      double ln[U][5];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = min(k0 + u * kDetThreads, cnt - 1);  // past the end: a repeat, not stored
        const uint32_t code = dlist[k];
        const int lr = (int)(code >> 16);
        rr[u] = r0 + lr - 1;
        cc[u] = (int)(code & 0xffffu);
        const int ic = tile_index<T>(c, box_h, lr, cc[u]);
        ln[u][0] = Ln<T>::f(tile[tile_index<T>(c, box_h, lr, cc[u] - 1)], a.lut);
        ln[u][1] = Ln<T>::f(tile[ic], a.lut);
        ln[u][2] = Ln<T>::f(tile[tile_index<T>(c, box_h, lr, cc[u] + 1)], a.lut);
        ln[u][3] = Ln<T>::f(tile[ic - c.box_w], a.lut);
        ln[u][4] = Ln<T>::f(tile[ic + c.box_w], a.lut);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * kDetThreads;
        if (k >= cnt) break;
        // the two fits of eval_chunk / mask_staged: same operands, same operations
        double xc, yc;
        fit3(ln[u][0], ln[u][1], ln[u][2], cc[u], xc);
        fit3(ln[u][3], ln[u][1], ln[u][4], rr[u], yc);
        c.x[base + k] = xc;
        c.y[base + k] = yc;
        c.rc[base + k] = make_int2(rr[u], cc[u]);
      }
    }
    __syncthreads();
  }
}

// Dynamic shared memory of detect_kernel<T> on the current device raised to at least
// `bytes` (the attribute is per device; set once per device and size).
template <typename T>
void detect_smem_attr(size_t bytes) {
  static std::mutex mu;
  static size_t set[64] = {};
  int dev = 0;
  OLPT_CUDA(cudaGetDevice(&dev));
  OLPT_REQUIRE(dev >= 0 && dev < 64, OLPT_ERR_INVALID_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (bytes <= 48 * 1024 || bytes <= set[dev]) return;
  OLPT_CUDA(cudaFuncSetAttribute(detect_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
  set[dev] = bytes;
}

template <typename T>
void launch_detect(const DetArgs& a, int n_blocks, size_t smem, cudaStream_t s) {
  detect_smem_attr<T>(smem);
  detect_kernel<T><<<OLPT_G(n_blocks), kDetThreads, smem, s>>>(a);
  OLPT_CUDA(cudaGetLastError());
}

CUtensorMapDataType tma_dtype(int dtype) {
  switch (dtype) {
    case OLPT_U8: return CU_TENSOR_MAP_DATA_TYPE_UINT8;
    case OLPT_U16: return CU_TENSOR_MAP_DATA_TYPE_UINT16;
    case OLPT_F32: return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    default: return CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  }
}

// Shared memory of one staged band: 64 KB (three CTAs per SM), up to 200 KB when a
// row is so wide that fewer than four rows would fit.
constexpr size_t kDetTileBudget = 64 * 1024, kDetTileBudgetMax = 200 * 1024;

struct DetGeom {
  int cpr, n_box, box_w;
  size_t row_img, row_mask;
};

DetGeom det_geom(int W, int esz) {
  DetGeom g;
  const int N = 16 / esz;
  g.cpr = (W + N - 1) / N;
  g.n_box = (W + kBoxW - 1) / kBoxW;
  g.box_w = g.n_box > 1 ? kBoxW : g.cpr * N;  // a multiple of N, at most 256
  g.row_img = (size_t)g.n_box * g.box_w * esz;
  g.row_mask = (size_t)g.cpr * sizeof(uint16_t);
  return g;
}

// Rows per band that fit `budget` bytes: (R + 2) image rows, R mask rows, the
// detection list, alignment.
int det_rows_fitting(const DetGeom& g, size_t budget) {
  const size_t fixed = 128 + 2 * g.row_img + 8 + kDetList * sizeof(uint32_t);
  if (budget <= fixed) return 0;
  return (int)std::min<size_t>((budget - fixed) / (g.row_img + g.row_mask), 254);
}

size_t det_smem_bytes(const DetGeom& g, int R) {
  return 128 + (size_t)(R + 2) * g.row_img + (size_t)R * g.row_mask + 8 +
         kDetList * sizeof(uint32_t);
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

// The two-pass detector on the context's images (images too wide to stage).
template <typename T>
void two_pass(olpt_ctx* ctx, PeakArgs& a, int blocks, int64_t* tot) {
  ctx->band_counts.ensure(blocks * sizeof(int), ctx->stream);
  ctx->band_offsets.ensure(blocks * sizeof(int64_t), ctx->stream);
  a.band_counts = ctx->band_counts.as<int>();
  launch_peaks<T>(a, blocks, ctx->band_offsets.as<int64_t>(), tot, ctx->stream);
}

// Detect on the current images; counts stay on the device in ctx->det_counts and are
// mirrored to det_counts_h when `sync_counts`.
void find_peaks_device(olpt_ctx* ctx, double min_int, bool sync_counts) {
  OLPT_REQUIRE(ctx->n_cam > 0, OLPT_ERR_INVALID_ARG, "no cameras uploaded");
  ensure_log_luts(ctx);
  int dtype = -1;
  int64_t active_rows = 0;
  for (int c = 0; c < ctx->n_cam; ++c) {
    ImagePlane& im = ctx->img[c];
    OLPT_REQUIRE(im.buf.p != nullptr, OLPT_ERR_INVALID_ARG, "no image uploaded for camera");
    if (dtype < 0) dtype = im.dtype;
    OLPT_REQUIRE(im.dtype == dtype, OLPT_ERR_INVALID_ARG, "all cameras must share one dtype");
    if (ctx->cams_h[c].is_active) active_rows += im.H;
    ensure_det_capacity(ctx, c, ((int64_t)im.H * im.W + 1) / 2 + 1);
  }
  const int esz = dtype == OLPT_U8 ? 1 : dtype == OLPT_U16 ? 2 : dtype == OLPT_F32 ? 4 : 8;
  const double* lut = dtype == OLPT_U8    ? ctx->lut_u8.as<double>()
                      : dtype == OLPT_U16 ? ctx->lut_u16.as<double>()
                                          : nullptr;
  double img_bytes = 0;
  for (int c = 0; c < ctx->n_cam; ++c)
    if (ctx->cams_h[c].is_active) img_bytes += (double)ctx->img[c].H * ctx->img[c].W * esz;

  // staged geometry: bands of R rows, R small enough for about three CTAs per SM over
  // all cameras' rows and for the shared-memory budget
  const int rows_fill = (int)std::max<int64_t>(4, active_rows / (3 * 148));
  bool staged = true;
  DetGeom geo[OLPT_MAX_CAM];
  int band_rows[OLPT_MAX_CAM];
  size_t smem = 0;
  for (int c = 0; c < ctx->n_cam; ++c) {
    geo[c] = det_geom(ctx->img[c].W, esz);
    int R = det_rows_fitting(geo[c], kDetTileBudget);
    if (R < 4) R = det_rows_fitting(geo[c], kDetTileBudgetMax);
    if (R < 1 || ctx->img[c].W > 65535) staged = false;  // detection codes hold 16-bit columns
    band_rows[c] = std::max(1, std::min(R, rows_fill));
    if (ctx->cams_h[c].is_active) smem = std::max(smem, det_smem_bytes(geo[c], band_rows[c]));
  }

  const int pid = ctx->prof.begin(PROF_PEAKS, ctx->stream);
  if (staged) {
    DetArgs a{};
    a.n_cam = ctx->n_cam;
    a.min_int = min_int;
    // levels are 0 .. 65535: NaN or <= 0 rejects none, above 65535 rejects all
    a.min_level = !(min_int > 0.0) ? 0 : min_int > 65535.0 ? 65536 : (int)std::ceil(min_int);
    a.lut = lut;
    int blocks = 0;
    for (int c = 0; c < ctx->n_cam; ++c) {
      ImagePlane& im = ctx->img[c];
      DetCam& dc = a.cam[c];
      dc.H = im.H;
      dc.W = im.W;
      dc.band_rows = band_rows[c];
      dc.box_w = geo[c].box_w;
      dc.n_box = geo[c].n_box;
      dc.cpr = geo[c].cpr;
      dc.n_bands = ctx->cams_h[c].is_active ? (im.H + dc.band_rows - 1) / dc.band_rows : 0;
      dc.band_base = blocks;
      dc.x = ctx->dets[c].x.as<double>();
      dc.y = ctx->dets[c].y.as<double>();
      dc.rc = ctx->dets[c].rc.as<int2>();
      blocks += dc.n_bands;
      olpt_ctx::DetMap& m = ctx->det_map[c];
      if (m.p != im.buf.p || m.dtype != dtype || m.H != im.H || m.W != im.W ||
          m.pitch != im.pitch || m.box_w != dc.box_w || m.box_h != dc.band_rows + 2) {
        const cuuint64_t dims[2] = {(cuuint64_t)im.W, (cuuint64_t)im.H};
        const cuuint64_t strides[1] = {(cuuint64_t)im.pitch};
        const cuuint32_t box[2] = {(cuuint32_t)dc.box_w, (cuuint32_t)(dc.band_rows + 2)};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = tensor_map_encoder()(
            &m.map, tma_dtype(dtype), 2, im.buf.p, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        OLPT_REQUIRE(r == CUDA_SUCCESS, OLPT_ERR_CUDA,
                     "cuTensorMapEncodeTiled failed for a camera image (" +
                         std::to_string((int)r) + ")");
        m.p = im.buf.p;
        m.dtype = dtype;
        m.H = im.H;
        m.W = im.W;
        m.pitch = im.pitch;
        m.box_w = dc.box_w;
        m.box_h = dc.band_rows + 2;
      }
      a.map[c] = m.map;
    }
    const size_t words = (size_t)kDcState + blocks;
    ctx->det_counts.ensure(words * sizeof(int64_t), ctx->stream);
    a.dc = ctx->det_counts.as<unsigned long long>();
    a.hold_ticket = ctx->test_hold_ticket;
    a.wait_limit_ns = ctx->test_hold_ticket >= 0 ? ctx->test_wait_limit_ns : umma::kWaitLimitNs;
    ctx->test_hold_ticket = -1;
    // totals, error word, ticket and band states start at zero
    OLPT_CUDA(cudaMemsetAsync(ctx->det_counts.p, 0, words * sizeof(int64_t), ctx->stream));
    if (blocks > 0) {
      switch (dtype) {
        case OLPT_U8: launch_detect<uint8_t>(a, blocks, smem, ctx->stream); break;
        case OLPT_U16: launch_detect<uint16_t>(a, blocks, smem, ctx->stream); break;
        case OLPT_F32: launch_detect<float>(a, blocks, smem, ctx->stream); break;
        default: launch_detect<double>(a, blocks, smem, ctx->stream); break;
      }
    }
  } else {
    PeakArgs a{};
    a.n_cam = ctx->n_cam;
    a.min_int = min_int;
    a.lut = lut;
    int blocks = 0;
    for (int c = 0; c < ctx->n_cam; ++c) {
      ImagePlane& im = ctx->img[c];
      const int N = 16 / esz;
      const int cpr = (im.W + N - 1) / N;
      PeakCam& pc = a.cam[c];
      pc.img = im.buf.as<unsigned char>();
      pc.pitch = im.pitch;
      pc.H = im.H;
      pc.W = im.W;
      pc.band_rows = std::max(1, (2048 + cpr - 1) / cpr);
      pc.n_bands = (im.H + pc.band_rows - 1) / pc.band_rows;
      pc.band_base = blocks;
      pc.active = ctx->cams_h[c].is_active;
      blocks += pc.n_bands;
      pc.x = ctx->dets[c].x.as<double>();
      pc.y = ctx->dets[c].y.as<double>();
      pc.rc = ctx->dets[c].rc.as<int2>();
    }
    ctx->det_counts.ensure((size_t)(kDcErr + 1) * sizeof(int64_t), ctx->stream);
    int64_t* tot = ctx->det_counts.as<int64_t>();
    OLPT_CUDA(cudaMemsetAsync(tot, 0, (size_t)(kDcErr + 1) * sizeof(int64_t), ctx->stream));
    switch (dtype) {
      case OLPT_U8: two_pass<uint8_t>(ctx, a, blocks, tot); break;
      case OLPT_U16: two_pass<uint16_t>(ctx, a, blocks, tot); break;
      case OLPT_F32: two_pass<float>(ctx, a, blocks, tot); break;
      default: two_pass<double>(ctx, a, blocks, tot); break;
    }
  }
  ctx->prof.end(PROF_PEAKS, pid, ctx->stream, img_bytes);
  ctx->det_counts_h.assign(ctx->n_cam, 0);
  if (sync_counts) {
    int64_t h[kDcErr + 1];
    OLPT_CUDA(cudaMemcpyAsync(h, ctx->det_counts.p, sizeof(h), cudaMemcpyDeviceToHost,
                              ctx->stream));
    OLPT_CUDA(cudaStreamSynchronize(ctx->stream));
    OLPT_REQUIRE(h[kDcErr] == 0, OLPT_ERR_TIMEOUT,
                 "peak detection: a staging or look-back wait timed out");
    for (int c = 0; c < ctx->n_cam; ++c) ctx->det_counts_h[c] = h[c];
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
  unsigned long long ctx_id = 0;     // CUDA context the table was filled in (0 = never)
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  double* lut = nullptr;             // device address of g_noalloc_log_lut
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[64];

// Unique id of the calling thread's current CUDA context (cuCtxGetId, driver API
// looked up through the runtime); a device reset gives the device a new context and
// hence a new id, so the log table is filled again in it.
cudaError_t current_context_id(unsigned long long* id) {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) return cudaErrorNotSupported;
    get_current = reinterpret_cast<GetCurrent>(p);
    e = cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) return cudaErrorNotSupported;
    get_id = reinterpret_cast<GetId>(p);
  }
  void* ctx = nullptr;
  if (get_current(&ctx) != 0 || !ctx) return cudaErrorDeviceUninitialized;
  return get_id(ctx, id) == 0 ? cudaSuccess : cudaErrorDeviceUninitialized;
}
}  // namespace

// Every call, with the device current: resolve the arrays' device addresses (in host
// code their names are host-side stand-ins, not device addresses) and, the first time
// in each CUDA context of the device (after a cudaDeviceReset too), fill the log
// table.  The fill is a synchronous copy, so the first call in a context must come
// before any stream capture.
static olpt_status_t noalloc_setup(int dev, NoAllocDevice*& out, std::string& err) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= 64) {
    err = "device ordinal out of range";
    return OLPT_ERR_INVALID_ARG;
  }
  NoAllocDevice& d = g_noalloc_dev[dev];
  cudaError_t e = cudaGetSymbolAddress((void**)&d.scratch, g_noalloc_scratch);
  if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.lut, g_noalloc_log_lut);
  if (e != cudaSuccess) {
    err = std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
    return OLPT_ERR_CUDA;
  }
  unsigned long long ctx_id = 0;
  e = current_context_id(&ctx_id);
  if (e != cudaSuccess) {
    err = std::string("no current CUDA context: ") + cudaGetErrorString(e);
    return OLPT_ERR_CUDA;
  }
  if (d.ctx_id != ctx_id) {
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
    d.ctx_id = ctx_id;
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
