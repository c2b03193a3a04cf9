// Kernel family (c): Shake -- residual image, per-particle line search, score,
// repeated and ghost flags.
//
// Reference: Shake::runShake (src/srcSTB/Shake.cpp:36-163), calResidueImage (:165-244),
// calROIBound (:246-277), buildROIInfo (:279-328), shakeOneObject (:409-665),
// calObjectScore (:668-782), markRepeatedObj (:785-823), TracerShakeStrategy
// gaussIntensity / project2DInt / calShakeResidue (:901-1045).
//
// B200 mapping, per shake iteration:
//  1. prep: one thread per object projects it on every camera (FP64), evaluates the
//     OTF at its centre and keys each (object, camera) pair by the 32x32 image tile
//     of its projection; a counting sort turns the keys into per-tile bins.
//  2. residual: one CTA owns one image tile, gathers the objects binned in the 3x3
//     neighbouring tiles, max-fuses their Gaussian footprints in shared memory and
//     writes residual = image - max projection for the whole tile.  No global
//     atomics, and the result does not depend on object order (min-fusion in the
//     reference is a max over projections).
//  3. shake: one warp per particle stages its 8x8 augmented ROI of every camera in
//     shared memory, then runs the reference's axis-wise line search.  Each residue
//     evaluation spreads (camera, pixel) pairs over the lanes; the scalar control
//     flow is executed identically by all lanes.
// Precision: Real = float is the production path (residual, OTF Gaussian and MSE in
// FP32); Real = double is the parity path, which also sums every camera's squared
// error in the reference's row-major order so that only exp() rounding differs.
// Projections, polyfit and all decisions stay in FP64 in both.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_shake_dev.cuh"
#include "olpt_otf.cuh"
#include "olpt_scan.cuh"
#include "olpt_shake.h"

namespace olpt {

constexpr int kTile = 32;

namespace {

inline int nblk(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------- 1. prep
template <typename Real>
__global__ void prep_kernel(const __grid_constant__ ShakeView v, const double* xyz, int64_t n, double* uv, Real* otfp,
                            int* pair_key, const uint8_t* flags, int all_cams) {
  int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= n) return;
  const double X = xyz[3 * o], Y = xyz[3 * o + 1], Z = xyz[3 * o + 2];
  const bool masked = flags && flags[o] != 0;
  for (int c = 0; c < v.n_cam; ++c) {
    double u, w;
    cam_project(v.cams[c], X, Y, Z, u, w);
    uv[(o * v.n_cam + c) * 2] = u;
    uv[(o * v.n_cam + c) * 2 + 1] = w;
    double q[5];
    otf_param(v.otf, c, X, Y, Z, q);
    for (int k = 0; k < 5; ++k) otfp[(o * v.n_cam + c) * 5 + k] = (Real)q[k];
    int key = -1;
    if (!masked && (all_cams || v.cams[c].is_active)) {
      const Rect r = roi_bound(v.cams[c].n_row, v.cams[c].n_col, u, w, v.r_px, v.r_px);
      if (!rect_empty(r)) {
        const int ntx = (v.cams[c].n_col + kTile - 1) / kTile;
        key = v.tile_base[c] + (r.rmin / kTile) * ntx + (r.cmin / kTile);
      }
    }
    pair_key[o * v.n_cam + c] = key;
  }
}

// ---------------------------------------------------------------- 2. residual
__device__ __forceinline__ void smem_max(float* p, float v) {
  atomicMax(reinterpret_cast<unsigned int*>(p), __float_as_uint(v));
}
__device__ __forceinline__ void smem_max(double* p, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

// Window tiles are keyed by the tile of the window's top-left pixel, so a CTA
// gathers bins of its own tile and the tiles up/left of it (windows < 32 px).
template <typename Real>
__global__ void __launch_bounds__(256) residual_kernel(const __grid_constant__ ShakeView v, const double* uv,
                                                       const Real* otfp, const int* bin_start,
                                                       const int* bin_items, int clamp,
                                                       int all_cams) {
  __shared__ Real pmax[kTile * kTile];
  // locate camera and tile
  int cam = 0;
  for (int c = 1; c < v.n_cam; ++c)
    if ((int)blockIdx.x >= v.tile_base[c]) cam = c;
  const CamDev& cm = v.cams[cam];
  if (!(all_cams || cm.is_active)) return;
  const int ntx = (cm.n_col + kTile - 1) / kTile;
  const int t = blockIdx.x - v.tile_base[cam];
  const int ty = t / ntx, tx = t % ntx;
  const int r0 = ty * kTile, c0 = tx * kTile;
  for (int i = threadIdx.x; i < kTile * kTile; i += blockDim.x) pmax[i] = (Real)0;
  __syncthreads();
  const int nty = (cm.n_row + kTile - 1) / kTile;
  const int win = v.win_w * v.win_h;
  for (int dy = -1; dy <= 0; ++dy) {
    const int by = ty + dy;
    if (by < 0 || by >= nty) continue;
    for (int dx = -1; dx <= 0; ++dx) {
      const int bx = tx + dx;
      if (bx < 0 || bx >= ntx) continue;
      const int b = v.tile_base[cam] + by * ntx + bx;
      const int s0 = bin_start[b], s1 = bin_start[b + 1];
      const int total = (s1 - s0) * win;
      for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int pair = bin_items[s0 + k / win];
        const int pix = k % win;
        const int64_t o = pair / v.n_cam;
        const double u = uv[2 * (int64_t)pair], w = uv[2 * (int64_t)pair + 1];
        const Rect r = roi_bound(cm.n_row, cm.n_col, u, w, v.r_px, v.r_px);
        const int rr = r.rmin + pix / v.win_w, cc = r.cmin + pix % v.win_w;
        if (rr >= r.rmax || cc >= r.cmax) continue;
        if (rr < r0 || rr >= r0 + kTile || cc < c0 || cc >= c0 + kTile) continue;
        const Real p = gauss<Real>(cc, rr, u, w, otfp + (int64_t)pair * 5);
        (void)o;
        if (p == (Real)0) continue;
        smem_max(&pmax[(rr - r0) * kTile + (cc - c0)], p);
      }
    }
  }
  __syncthreads();
  const PlaneView& src = v.orig[cam];
  Real* dst = reinterpret_cast<Real*>(v.res[cam].p);
  const int64_t dpitch = v.res[cam].pitch / (int64_t)sizeof(Real);
  for (int i = threadIdx.x; i < kTile * kTile; i += blockDim.x) {
    const int rr = r0 + i / kTile, cc = c0 + i % kTile;
    if (rr >= cm.n_row || cc >= cm.n_col) continue;
    const Real o = (Real)load_any(src, rr, cc);
    const Real pm = pmax[i];
    Real val = o;
    if (pm > (Real)0) {
      val = o - pm;
      if (val > o) val = o;  // keep min(o, o - p)
      if (clamp && val < (Real)0) val = (Real)0;
    }
    dst[(int64_t)rr * dpitch + cc] = val;
  }
}

// ---------------------------------------------------------------- 3. shake
struct WarpCtx {
  int n_cam, lane;
};

template <typename Real>
struct Smem {
  Real* aug;      // n_cam x roi_area
  double* dd;     // n_cam x roi_area (FP64 ordered sums)
  Real* otf;      // n_cam x 5 at the current trial point
  double* uvc;    // n_cam x 2 at the current trial point
};

// All lanes: project point P on every camera and evaluate the OTF there.
template <typename Real, int NC>
__device__ void eval_geom(const ShakeView& v, const double P[3], Smem<Real>& S) {
  const int lane = threadIdx.x & 31;
  if (lane < NC) {
    double u, w;
    cam_project(v.cams[lane], P[0], P[1], P[2], u, w);
    S.uvc[2 * lane] = u;
    S.uvc[2 * lane + 1] = w;
    double q[5];
    otf_param(v.otf, lane, P[0], P[1], P[2], q);
    for (int k = 0; k < 5; ++k) S.otf[5 * lane + k] = (Real)q[k];
  }
  __syncwarp();
}

template <typename Real, int NC, int K>
__device__ void residueK(const ShakeView& v, const Rect* roi, Smem<Real>& S, double f[K]);

// TracerShakeStrategy::calShakeResidue (Shake.cpp:951-1045) for the point whose
// geometry is in S (eval_geom), against the staged augmented ROIs.  The production
// path is residueK with one point; the FP64 parity path stages the squared
// differences and sums them per camera in row-major order.
template <typename Real, int NC>
__device__ double residue(const ShakeView& v, const Rect* roi, Smem<Real>& S) {
  if (!(sizeof(Real) == 8 && v.exact_sums)) {
    double f1[1];
    residueK<Real, NC, 1>(v, roi, S, f1);
    return f1[0];
  }
  const int lane = threadIdx.x & 31;
  const int area = v.roi_area;
  double mse[NC];
  Real part[NC];
  for (int c = 0; c < NC; ++c) part[c] = (Real)0;
  for (int q = lane; q < NC * area; q += 32) {
    const int c = q / area, pix = q % area;
    const Rect& R = roi[c];
    if (rect_empty(R)) continue;
    const int w = R.cmax - R.cmin, h = R.rmax - R.rmin;
    if (w <= 0 || h <= 0 || pix >= w * h) continue;
    const int row = R.rmin + pix / w, col = R.cmin + pix % w;
    const double u = S.uvc[2 * c], vv = S.uvc[2 * c + 1];
    const int prmin = (int)floor(vv - v.r_px), prmax = (int)ceil(vv + v.r_px + 1);
    const int pcmin = (int)floor(u - v.r_px), pcmax = (int)ceil(u + v.r_px + 1);
    Real pred = (Real)0;
    if (row >= prmin && row < prmax && col >= pcmin && col < pcmax)
      pred = gauss<Real>(col, row, u, vv, S.otf + 5 * c);
    const Real d = S.aug[c * area + pix] - pred;
    if ((sizeof(Real) == 8 && v.exact_sums))
      S.dd[c * area + pix] = (double)d * (double)d;
    else
      part[c] += d * d;
  }
  if ((sizeof(Real) == 8 && v.exact_sums)) {
    __syncwarp();
    if (lane < NC) {
      const Rect& R = roi[lane];
      const int n = rect_empty(R) ? 0 : (R.cmax - R.cmin) * (R.rmax - R.rmin);
      double sse = 0.0;
      for (int i = 0; i < n; ++i) sse += S.dd[lane * area + i];
      mse[0] = n > 0 ? sse / (double)n : 0.0;
    }
    double m0 = mse[0];
    for (int c = 0; c < NC; ++c) mse[c] = __shfl_sync(0xffffffffu, m0, c);
    __syncwarp();
  } else {
    for (int c = 0; c < NC; ++c) {
      Real s = part[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      const Rect& R = roi[c];
      const int n = rect_empty(R) ? 0 : (R.cmax - R.cmin) * (R.rmax - R.rmin);
      mse[c] = n > 0 ? (double)s / (double)n : 0.0;
    }
  }
  double cost = 0.0;
  int used = 0;
  for (int c = 0; c < NC; ++c) {
    if (!v.cams[c].is_active) continue;
    const Rect& R = roi[c];
    const int nr = R.rmax - R.rmin, nc = R.cmax - R.cmin;
    if (nr <= 0 || nc <= 0) continue;
    cost += mse[c];
    ++used;
  }
  return used > 1 ? cost / (double)used : __longlong_as_double(0x7ff0000000000000LL);
}

// Three trial points at once (the -delta / 0 / +delta evaluations of one axis):
// lanes 3 x n_cam project point j = lane / n_cam on camera lane % n_cam; slot j of
// the geometry arrays receives it (slot 0 is the one eval_geom uses).
template <typename Real, int NC>
__device__ void eval_geom3(const ShakeView& v, const double P[3], int ax, double x0,
                           const double rel[3], Smem<Real>& S) {
  const int lane = threadIdx.x & 31;
  constexpr int C = NC;
  if (lane < 3 * C) {
    const int j = lane / C, c = lane % C;
    double Q[3] = {P[0], P[1], P[2]};
    Q[ax] = x0 + rel[j];
    double u, w;
    cam_project(v.cams[c], Q[0], Q[1], Q[2], u, w);
    S.uvc[2 * lane] = u;
    S.uvc[2 * lane + 1] = w;
    double q[5];
    otf_param(v.otf, c, Q[0], Q[1], Q[2], q);
    for (int k = 0; k < 5; ++k) S.otf[5 * lane + k] = (Real)q[k];
  }
  __syncwarp();
}

// calShakeResidue for the K points in the geometry slots 0 .. K - 1 (K = 3: the points
// of eval_geom3; K = 1: the point of eval_geom), production path: per camera, each
// lane visits the pixels q = lane, lane + 32, ... of the reference loop over all
// cameras' ROI pixels, in that order, so the sums are those of single evaluations bit
// for bit; the K points run interleaved.
template <typename Real, int NC, int K>
__device__ void residueK(const ShakeView& v, const Rect* roi, Smem<Real>& S, double f[K]) {
  const int lane = threadIdx.x & 31;
  const int area = v.roi_area;
  constexpr int C = NC;
  double cost[K];
#pragma unroll
  for (int j = 0; j < K; ++j) cost[j] = 0.0;
  int used = 0;
  // kept rolled: one copy of the pixel loop instead of one per camera (the kernel is
  // bound by instruction fetch; the unrolled form measured 10% slower)
#pragma unroll 1
  for (int c = 0; c < C; ++c) {
    const Rect R = roi[c];
    if (rect_empty(R)) continue;
    const int w = R.cmax - R.cmin, h = R.rmax - R.rmin;
    if (w <= 0 || h <= 0) continue;
    double u[K], vv[K];
    int prmin[K], prmax[K], pcmin[K], pcmax[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      u[j] = S.uvc[2 * (j * C + c)];
      vv[j] = S.uvc[2 * (j * C + c) + 1];
      prmin[j] = (int)floor(vv[j] - v.r_px);
      prmax[j] = (int)ceil(vv[j] + v.r_px + 1);
      pcmin[j] = (int)floor(u[j] - v.r_px);
      pcmax[j] = (int)ceil(u[j] + v.r_px + 1);
    }
    // the pixels of camera c that this lane visits in the single evaluation's loop
    // over q = lane, lane + 32, ... < C * area, in the same order
    int first = lane - (c * area) % 32;
    if (first < 0) first += 32;
    Real part[K];
#pragma unroll
    for (int j = 0; j < K; ++j) part[j] = (Real)0;
    for (int pix = first; pix < area; pix += 32) {
      if (pix >= w * h) continue;
      const int row = R.rmin + pix / w, col = R.cmin + pix % w;
      const Real a = S.aug[c * area + pix];
#pragma unroll
      for (int j = 0; j < K; ++j) {
        Real pred = (Real)0;
        if (row >= prmin[j] && row < prmax[j] && col >= pcmin[j] && col < pcmax[j])
          pred = gauss<Real>(col, row, u[j], vv[j], S.otf + 5 * (j * C + c));
        const Real d = a - pred;
        part[j] += d * d;
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part[j] += __shfl_xor_sync(0xffffffffu, part[j], o);
    if (!v.cams[c].is_active) continue;
    const int n = w * h;
#pragma unroll
    for (int j = 0; j < K; ++j) cost[j] += (double)part[j] / (double)n;
    ++used;
  }
#pragma unroll
  for (int j = 0; j < K; ++j)
    f[j] = used > 1 ? cost[j] / (double)used : __longlong_as_double(0x7ff0000000000000LL);
}

// myMATH::polyfit order 2 (myMATH.cpp:490-534): (X^T X)^-1 X^T y with the
// reference's operation order.
__device__ void polyfit2(const double* x, const double* y, int n, double coef[3]) {
  double X[5][3];
  for (int i = 0; i < n; ++i) {
    X[i][0] = 1.0;
    X[i][1] = x[i];
    X[i][2] = x[i] * x[i];
  }
  double A[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double s = 0;
      for (int i = 0; i < n; ++i) s += X[i][r] * X[i][c];
      A[3 * r + c] = s;
    }
  double Ai[9];
  gauss_inverse3(A, Ai);
  double B[3][5];
  for (int r = 0; r < 3; ++r)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += Ai[3 * r + k] * X[i][k];
      B[r][i] = s;
    }
  for (int r = 0; r < 3; ++r) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += B[r][i] * y[i];
    coef[r] = s;
  }
}

__device__ double median_small(double* a, int n) {
  if (n == 0) return 0.0;
  for (int i = 1; i < n; ++i) {
    double t = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > t) {
      a[j + 1] = a[j];
      --j;
    }
    a[j + 1] = t;
  }
  const int mid = n / 2;
  double m = a[mid];
  if ((n & 1) == 0) m = 0.5 * (m + a[mid - 1]);
  return m;
}

__device__ __forceinline__ bool in_roi(const Rect& R, double u, double w) {
  return R.cmin <= u && u < R.cmax && R.rmin <= w && w < R.rmax;
}

// MINB: resident blocks per SM the kernel is compiled for -- 8 (64 registers a thread)
// or 4 (128 registers)
template <typename Real, int NC, int MINB>
__global__ void __launch_bounds__(128, MINB) shake_kernel(const __grid_constant__ ShakeView v, int64_t n, double* xyz,
                                                    double* uv, const Real* otfp, double* score,
                                                    double delta, const uint8_t* active,
                                                    double* resid_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp_in_blk = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t o = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_in_blk;
  constexpr int C = NC;
  const int area = v.roi_area;
  const size_t per_warp = v.smem_per_warp;
  unsigned char* base = smem_raw + per_warp * warp_in_blk;
  Smem<Real> S;
  S.aug = reinterpret_cast<Real*>(base);
  S.dd = reinterpret_cast<double*>(base + v.off_dd);
  S.otf = reinterpret_cast<Real*>(base + v.off_otf);
  S.uvc = reinterpret_cast<double*>(base + v.off_uv);
  if (o >= n) return;
  if (active && !active[o]) return;  // held fixed (learned shake: not in this pass)

  double P[3] = {xyz[3 * o], xyz[3 * o + 1], xyz[3 * o + 2]};
  double f_final = 0.0;
  // ---- buildROIInfo (Shake.cpp:279-328)
  Rect roi[NC];
  const double* uvo = uv + o * C * 2;
  for (int c = 0; c < C; ++c) {
    roi[c] = Rect{0, 0, 0, 0};  // default-constructed PixelRange for skipped cameras
    if (!v.cams[c].is_active) continue;
    roi[c] = roi_bound(v.cams[c].n_row, v.cams[c].n_col, uvo[2 * c], uvo[2 * c + 1],
                       v.r_px * v.ratio, v.r_px * v.ratio);
  }
  // per camera: the projection window once, then the ROI's pixels over the lanes (each
  // pixel is independent, so the lane mapping does not change the values)
#pragma unroll 1
  for (int c = 0; c < C; ++c) {
    const Rect R = roi[c];
    if (!v.cams[c].is_active || rect_empty(R)) continue;
    const int w = R.cmax - R.cmin, h = R.rmax - R.rmin;
    const double u = uvo[2 * c], vv = uvo[2 * c + 1];
    const Rect pr = roi_bound(v.cams[c].n_row, v.cams[c].n_col, u, vv, v.r_px, v.r_px);
    const Real* res = reinterpret_cast<const Real*>(v.res[c].p);
    const int64_t rp = v.res[c].pitch / (int64_t)sizeof(Real);
    const Real* q5 = otfp + (o * C + c) * 5;
    for (int pix = lane; pix < w * h; pix += 32) {
      const int row = R.rmin + pix / w, col = R.cmin + pix % w;
      Real a = res[(int64_t)row * rp + col];
      if (row >= pr.rmin && row < pr.rmax && col >= pr.cmin && col < pr.cmax)
        a += gauss<Real>(col, row, u, vv, q5);
      S.aug[c * area + pix] = a > (Real)0 ? a : (Real)0;
    }
  }
  __syncwarp();

  // ---- shakeOneObject (Shake.cpp:409-665)
  double tmp[3] = {P[0], P[1], P[2]};
  for (int ax = 0; ax < 3; ++ax) {
    const double x0 = P[ax];
    const double rel[3] = {-delta, 0.0, delta};
    double f[3];
    // the projections of the three trial points stay in the warp's shared slots
    // (slot j = trial j) instead of per-lane copies
    if ((sizeof(Real) == 8 && v.exact_sums)) {
      for (int j = 2; j >= 0; --j) {  // slot 0 last: single evaluations write slot 0
        tmp[ax] = x0 + rel[j];
        eval_geom<Real, NC>(v, tmp, S);
        f[j] = residue<Real, NC>(v, roi, S);
        if (j > 0 && lane < 2 * C) S.uvc[2 * j * C + lane] = S.uvc[lane];
        __syncwarp();
      }
    } else {
      eval_geom3<Real, NC>(v, tmp, ax, x0, rel, S);
      residueK<Real, NC, 3>(v, roi, S, f);
      __syncwarp();
    }
    tmp[ax] = x0 + rel[2];  // as left by the last single evaluation
    auto su = [&](int j, int c) { return S.uvc[2 * (j * C + c)]; };
    auto sv = [&](int j, int c) { return S.uvc[2 * (j * C + c) + 1]; };
    auto sok = [&](int j, int c) { return in_roi(roi[c], su(j, c), sv(j, c)); };
    const double fL = f[0], f0 = f[1], fR = f[2];
    const double tol = 1e-3 * fmax(1.0, f0);
    const bool mono_dec = (fL > f0 + tol) && (f0 > fR + tol);
    const bool mono_inc = (fR > f0 + tol) && (f0 > fL + tol);
    const bool mono = mono_dec || mono_inc;
    int s = mono_dec ? +1 : (mono_inc ? -1 : 0);
    const double kappa = (fL - 2.0 * f0 + fR);
    const double g = (fR - fL) / fmax(2.0 * delta, 1e-12);
    double cx[5] = {-delta, 0.0, delta, 0, 0};
    double cf[5] = {fL, f0, fR, 0, 0};
    double ca[5] = {x0 + -delta, x0, x0 + delta, 0, 0};
    int nc = 3;
    bool skip_expand = false, allow_xhat = true;
    if (kappa > 0.0) {
      const double x3 = delta * (fL - fR) / (2.0 * kappa);
      if (fabs(x3) <= 0.95 * delta) {
        const double a = kappa / (delta * delta + 1e-12);
        const double rho_pred = (g * g) / (2.0 * a * fmax(f0, 1.0));
        skip_expand = true;
        if (rho_pred < 8e-4) allow_xhat = false;
      }
    }
    if (!skip_expand && mono) {
      double J[NC], M[NC];
      int nJ = 0, nM = 0;
      for (int c = 0; c < C; ++c) {
        if (sok(0, c) && sok(2, c)) {
          const double du = su(2, c) - su(0, c), dv = sv(2, c) - sv(0, c);
          J[nJ++] = hypot(du, dv) / fmax(2.0 * delta, 1e-12);
        }
        if (sok(1, c)) {
          const Rect& R = roi[c];
          const double mu = fmin(su(1, c) - R.cmin, R.cmax - 1.0 - su(1, c));
          const double mv = fmin(sv(1, c) - R.rmin, R.rmax - 1.0 - sv(1, c));
          M[nM++] = fmin(mu, mv);
        }
      }
      const double Jx = median_small(J, nJ);
      const double mpx = median_small(M, nM);
      const double Delta_roi = (Jx > 0.0 && mpx > 0.0) ? (0.5 * mpx / Jx) : 0.0;
      double Delta_try = 0.0;
      if (kappa > 0.0) {
        const double x3 = delta * (fL - fR) / (2.0 * kappa);
        if (fabs(x3) > delta) {
          s = (x3 > 0.0 ? +1 : -1);
          if (Jx > 0.0 && fabs(x3) > (1.0 / Jx))
            Delta_try = 1.0 / Jx;
          else
            Delta_try = 1.15 * fabs(x3);
        }
      }
      if (Delta_try <= 0.0 && Jx > 0.0) Delta_try = 1.0 / Jx;
      const double Dp = (Delta_try > 0.0 && Delta_roi > 0.0) ? fmin(Delta_try, Delta_roi) : 0.0;
      if (Dp > 0.0) {
        const double dx_exp = (s >= 0 ? +Dp : -Dp);
        tmp[ax] = x0 + dx_exp;
        eval_geom<Real, NC>(v, tmp, S);
        bool out = false;
        for (int c = 0; c < C; ++c)
          if (!in_roi(roi[c], S.uvc[2 * c], S.uvc[2 * c + 1])) {
            out = true;
            break;
          }
        if (!out) {
          const double fexp = residue<Real, NC>(v, roi, S);
          cx[nc] = dx_exp;
          cf[nc] = fexp;
          ca[nc] = x0 + dx_exp;
          ++nc;
        }
        __syncwarp();
      }
    }
    double coef[3];
    polyfit2(cx, cf, nc, coef);
    if (allow_xhat && coef[2] > 0.0) {
      const double x_hat = -coef[1] / (2.0 * coef[2]);
      double xmin = cx[0], xmax = cx[0];
      for (int t = 0; t < nc; ++t) {
        xmin = fmin(xmin, cx[t]);
        xmax = fmax(xmax, cx[t]);
      }
      if (x_hat >= xmin && x_hat <= xmax) {
        tmp[ax] = x0 + x_hat;
        eval_geom<Real, NC>(v, tmp, S);
        bool out = false;
        for (int c = 0; c < C; ++c)
          if (!in_roi(roi[c], S.uvc[2 * c], S.uvc[2 * c + 1])) {
            out = true;
            break;
          }
        if (!out) {
          const double fhat = residue<Real, NC>(v, roi, S);
          cx[nc] = x_hat;
          cf[nc] = fhat;
          ca[nc] = x0 + x_hat;
          ++nc;
        }
        __syncwarp();
      }
    }
    int best = 0;
    double bf = cf[0];
    for (int t = 1; t < nc; ++t)
      if (cf[t] < bf) {
        bf = cf[t];
        best = t;
      }
    P[ax] = ca[best];
    f_final = bf;  // after the last axis: the residue at the final position
  }

  // ---- final projection + calObjectScore (Shake.cpp:668-782)
  eval_geom<Real, NC>(v, P, S);
  double numer_c[NC], denom_c[NC], peak_c[NC];
  Rect sr[NC];
  int use[NC];
  int n_used = 0;
  for (int c = 0; c < C; ++c) {
    use[c] = 0;
    sr[c] = Rect{1, 0, 1, 0};
    if (!v.cams[c].is_active) continue;
    sr[c] = roi_bound(v.cams[c].n_row, v.cams[c].n_col, S.uvc[2 * c], S.uvc[2 * c + 1], v.r_px,
                      v.r_px);
    if (rect_empty(sr[c])) continue;
    use[c] = 1;
    ++n_used;
  }
  // per camera: peak over the rect, sum of max(0, meas), sum of predictions (in
  // row-major order, one lane per camera)
  if (lane < C) {
    const int c = lane;
    double pk = 0.0, nu = 0.0, de = 0.0;
    if (use[c]) {
      const Rect& R = sr[c];
      const Rect& Q = roi[c];
      const bool qv = (Q.rmax - Q.rmin) > 0 && (Q.cmax - Q.cmin) > 0;
      const Real* res = reinterpret_cast<const Real*>(v.res[c].p);
      const int64_t rp = v.res[c].pitch / (int64_t)sizeof(Real);
      const int qw = Q.cmax - Q.cmin;
      for (int r = R.rmin; r < R.rmax; ++r)
        for (int cc = R.cmin; cc < R.cmax; ++cc) {
          const bool inq = qv && r >= Q.rmin && r < Q.rmax && cc >= Q.cmin && cc < Q.cmax;
          const double val = inq ? (double)S.aug[c * area + (r - Q.rmin) * qw + (cc - Q.cmin)]
                                 : (double)res[(int64_t)r * rp + cc];
          if (val > pk) pk = val;
          nu += fmax(0.0, val);
          de += (double)gauss<Real>(cc, r, S.uvc[2 * c], S.uvc[2 * c + 1], S.otf + 5 * c);
        }
    }
    peak_c[0] = pk;
    numer_c[0] = nu;
    denom_c[0] = de;
  }
  {
    const double pk = peak_c[0], nu = numer_c[0], de = denom_c[0];
    for (int c = 0; c < C; ++c) {
      peak_c[c] = __shfl_sync(0xffffffffu, pk, c);
      numer_c[c] = __shfl_sync(0xffffffffu, nu, c);
      denom_c[c] = __shfl_sync(0xffffffffu, de, c);
    }
  }
  double sc;
  if (n_used < 2) {
    sc = 1e-12;
  } else {
    if (n_used > 2) {
      int max_id = -1;
      double max_v = -__longlong_as_double(0x7ff0000000000000LL);
      for (int c = 0; c < C; ++c)
        if (use[c] && peak_c[c] > max_v) {
          max_v = peak_c[c];
          max_id = c;
        }
      if (max_id >= 0) use[max_id] = 0;
    }
    double tn = 0.0, td = 0.0;
    for (int c = 0; c < C; ++c) {
      if (!use[c]) continue;
      tn += numer_c[c];
      td += denom_c[c];
    }
    double ratio = (td > 1e-12) ? (tn / td) : 1.0;
    ratio = fmax(2.0 / 3.0, fmin(1.5, ratio));
    sc = sqrt(ratio);
  }
  if (lane == 0) {
    xyz[3 * o] = P[0];
    xyz[3 * o + 1] = P[1];
    xyz[3 * o + 2] = P[2];
    score[o] *= sc;
    if (resid_out) resid_out[o] = f_final;
  }
  if (lane < C) {
    uv[(o * C + lane) * 2] = S.uvc[2 * lane];
    uv[(o * C + lane) * 2 + 1] = S.uvc[2 * lane + 1];
  }
}

// ---------------------------------------------------------------- repeated / ghost
__global__ void hash_key_kernel(const double* xyz, int n, double cell, int n_buckets, int* key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long cx = (long long)floor(xyz[3 * i] / cell);
  const long long cy = (long long)floor(xyz[3 * i + 1] / cell);
  const long long cz = (long long)floor(xyz[3 * i + 2] / cell);
  unsigned long long h = (unsigned long long)(cx * 73856093LL) ^ (unsigned long long)(cy * 19349663LL) ^
                         (unsigned long long)(cz * 83492791LL);
  key[i] = (int)(h % (unsigned long long)n_buckets);
}

// number of neighbours j != i with squared distance < r2 (nanoflann radius test)
__global__ void neighbour_kernel(const double* xyz, int n, double cell, int n_buckets,
                                 const int* start, const int* items, double r2, int* has_nb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double X = xyz[3 * i], Y = xyz[3 * i + 1], Z = xyz[3 * i + 2];
  const long long cx = (long long)floor(X / cell), cy = (long long)floor(Y / cell),
                  cz = (long long)floor(Z / cell);
  int cnt = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        unsigned long long h = (unsigned long long)((cx + dx) * 73856093LL) ^
                               (unsigned long long)((cy + dy) * 19349663LL) ^
                               (unsigned long long)((cz + dz) * 83492791LL);
        const int b = (int)(h % (unsigned long long)n_buckets);
        for (int q = start[b]; q < start[b + 1]; ++q) {
          const int j = items[q];
          if (j == i) continue;
          const double ddx = xyz[3 * j] - X, ddy = xyz[3 * j + 1] - Y, ddz = xyz[3 * j + 2] - Z;
          const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
          if (d2 < r2) ++cnt;
        }
      }
  has_nb[i] = cnt > 0 ? 1 : 0;
}

// Greedy in index order (Shake.cpp:802-822): an object that is not itself marked
// marks every neighbour within the radius.  Only objects with neighbours do work.
// `list` holds, in ascending order, the objects that have any neighbour (list_n[0]
// of them); objects without neighbours mark nothing, so skipping them keeps the
// greedy identical.
__global__ void repeat_greedy_kernel(const double* xyz, int n, double cell, int n_buckets,
                                     const int* start, const int* items, double r2,
                                     const int* list, const int* list_n, uint8_t* rep) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int m = list_n[0];
  for (int q0 = 0; q0 < m; ++q0) {
    const int i = list[q0];
    if (i >= n - 1 || rep[i]) continue;
    const double X = xyz[3 * i], Y = xyz[3 * i + 1], Z = xyz[3 * i + 2];
    const long long cx = (long long)floor(X / cell), cy = (long long)floor(Y / cell),
                    cz = (long long)floor(Z / cell);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          unsigned long long h = (unsigned long long)((cx + dx) * 73856093LL) ^
                                 (unsigned long long)((cy + dy) * 19349663LL) ^
                                 (unsigned long long)((cz + dz) * 83492791LL);
          const int b = (int)(h % (unsigned long long)n_buckets);
          for (int q = start[b]; q < start[b + 1]; ++q) {
            const int j = items[q];
            if (j == i) continue;
            const double ddx = xyz[3 * j] - X, ddy = xyz[3 * j + 1] - Y, ddz = xyz[3 * j + 2] - Z;
            if (ddx * ddx + ddy * ddy + ddz * ddz < r2) rep[j] = 1;
          }
        }
  }
}

// Shake.cpp:118-136: the ghost rule against the mean score of the non-repeated
// objects, which the reference sums in index order.  The flags are first decided with
// a tree-summed mean; a score within the bound by which the sequential and the tree
// sum can differ (|S_seq - S_tree| <= 2 n 2^-53 sum|x|) of the threshold marks the
// result ambiguous, and only then does ghost_kernel redo the sequential sum.
constexpr int kScoreBlocks = 296;

__global__ void score_partial_kernel(const double* score, const uint8_t* rep, int n,
                                     double* part) {
  __shared__ double s1[256], s2[256], s3[256];
  double a = 0.0, b = 0.0, c = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (!rep[i]) {
      a += score[i];
      b += fabs(score[i]);
      c += 1.0;
    }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  s3[threadIdx.x] = c;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) {
      s1[threadIdx.x] += s1[threadIdx.x + k];
      s2[threadIdx.x] += s2[threadIdx.x + k];
      s3[threadIdx.x] += s3[threadIdx.x + k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = s1[0];
    part[3 * blockIdx.x + 1] = s2[0];
    part[3 * blockIdx.x + 2] = s3[0];
  }
}

__global__ void ghost_flag_kernel(const double* score, const uint8_t* rep, int n, double thred,
                                  const double* part, int nb, uint8_t* flags, int* amb) {
  __shared__ double st[3];
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += part[3 * b + threadIdx.x];
    st[threadIdx.x] = t;
  }
  __syncthreads();
  const double cnt = st[2];
  const double m = cnt > 0 ? st[0] / cnt : 0.0;
  const double thr = m * thred;
  const double e = cnt > 0 ? (2.0 * (double)n * 1.1102230246251565e-16 * st[1]) / cnt : 0.0;
  const double band = 2.0 * (e * fabs(thred) + fabs(thr) * 4.5e-16);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double sc = score[i];
  uint8_t f = rep[i] ? 2 : 0;
  if (sc == 0.0 || sc < thr - band) {
    f |= 1;
  } else if (!(sc >= thr + band)) {
    atomicOr(amb, 1);
    if (sc < thr) f |= 1;
  }
  flags[i] = f;
}

__global__ void ghost_kernel(const double* score, const uint8_t* rep, int n, double thred,
                             uint8_t* flags, const int* amb) {
  if (!*amb) return;
  __shared__ double s_mean;
  if (threadIdx.x < 32) {
    // warp 0 streams the scores in; lane 0 adds them strictly in index order
    const int lane = threadIdx.x;
    double sum = 0.0;
    long long cnt = 0;
    for (int base = 0; base < n; base += 32) {
      const int i = base + lane;
      const bool valid = i < n && !rep[i];
      const double x = valid ? score[i] : 0.0;
      const unsigned ball = __ballot_sync(0xffffffffu, valid);
#pragma unroll 4
      for (int j = 0; j < 32; ++j) {
        const double y = __shfl_sync(0xffffffffu, x, j);
        if (lane == 0 && (ball >> j) & 1u) sum += y;
      }
      cnt += __popc(ball);
    }
    if (lane == 0) s_mean = cnt ? sum / (double)cnt : 0.0;
  }
  __syncthreads();
  const double m = s_mean;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    uint8_t f = rep[i] ? 2 : 0;
    if (score[i] < m * thred || score[i] == 0.0) f |= 1;
    flags[i] = f;
  }
}

// has_nb[i] is 0 or 1 after neighbour_kernel; pos = exclusive scan of it
__global__ void compact_kernel(const int* flag, const int* pos, int n, int* list) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flag[i]) list[pos[i]] = i;
}

__global__ void fill_kernel(double* p, int64_t n, double v) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

}  // namespace

// ---------------------------------------------------------------- host drivers
// ---------------------------------------------------------------- learned shake
// correction in units of scale (mm); keep = not a ghost by the network's logit
__global__ void learned_apply_kernel(double* xyz, const float* o, int64_t n, double scale,
                                     float ghost_logit, int* keep) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* oi = o + 4 * i;
  const bool fin = isfinite(oi[0]) && isfinite(oi[1]) && isfinite(oi[2]) && isfinite(oi[3]);
  if (fin)
    for (int d = 0; d < 3; ++d) xyz[3 * i + d] += (double)oi[d] * scale;
  keep[i] = (fin && oi[3] <= ghost_logit) ? 1 : 0;
}

__global__ void compact_xyz_kernel(const int* keep, const int* pos, int64_t n, const double* a,
                                   double* a_out, const double* b, double* b_out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || !keep[i]) return;
  const int64_t k = pos[i];
  for (int d = 0; d < 3; ++d) {
    a_out[3 * k + d] = a[3 * i + d];
    b_out[3 * k + d] = b[3 * i + d];
  }
}

// objects whose residue after the refinement, divided by the mean squared OTF
// amplitude over the active cameras, exceeds thr (or is not finite) restart the
// full shake from their stereo position
template <typename Real>
__global__ void fallback_kernel(const double* res, const Real* otfp, const CamDev* cams, int C,
                                int64_t n, double thr, uint8_t* act, double* xyz,
                                const double* start, double* score, int* count) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a2 = 0.0;
  int k = 0;
  for (int c = 0; c < C; ++c) {
    if (!cams[c].is_active) continue;
    const double a = (double)otfp[(i * C + c) * 5];
    a2 += a * a;
    ++k;
  }
  a2 = k > 0 ? a2 / k : 1.0;
  const double r = res[i] / (a2 > 1e-12 ? a2 : 1e-12);
  const bool fb = !(r <= thr);
  act[i] = fb ? 1 : 0;
  if (fb) {
    for (int d = 0; d < 3; ++d) xyz[3 * i + d] = start[3 * i + d];
    score[i] = 1.0;
    atomicAdd(count, 1);
  }
}

// refined objects carry a score over refine_loops iterations: bring it to the
// n_shake_loop scale of the plain schedule
__global__ void score_scale_kernel(double* score, const uint8_t* act, int64_t n, double expo) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || act[i]) return;
  score[i] = pow(score[i], expo);
}

static ShakeView make_view(olpt_ctx* ctx, const ShakeParams& sp, bool fp64) {
  ShakeView v{};
  v.n_cam = ctx->n_cam;
  v.cams = ctx->cams_d.as<CamDev>();
  v.otf = otf_view(ctx);
  v.r_px = sp.radius_obj;
  v.ratio = (double)sp.ratio_augimg;
  const int side = (int)std::lround(2.0 * sp.radius_obj * sp.ratio_augimg);
  OLPT_REQUIRE(side >= 1 && side <= 16, OLPT_ERR_UNSUPPORTED,
               "augmented ROI side round(2 * radius_obj * ratio_augimg) must be in [1, 16]");
  v.roi_area = side * side;
  v.win_w = v.win_h = (int)std::lround(2.0 * sp.radius_obj);
  OLPT_REQUIRE(v.win_w >= 1 && v.win_w < kTile, OLPT_ERR_UNSUPPORTED,
               "projection window round(2 * radius_obj) must be below 32 px");
  v.exact_sums = fp64 ? 1 : 0;
  int tiles = 0;
  for (int c = 0; c < ctx->n_cam; ++c) {
    const CamDev& cm = ctx->cams_h[c];
    v.tile_base[c] = tiles;
    tiles += ((cm.n_row + kTile - 1) / kTile) * ((cm.n_col + kTile - 1) / kTile);
    const ImagePlane& im = ctx->img[c];
    OLPT_REQUIRE(im.buf.p, OLPT_ERR_INVALID_ARG, "no image for camera");
    OLPT_REQUIRE(im.H == cm.n_row && im.W == cm.n_col, OLPT_ERR_INVALID_ARG,
                 "image size differs from the camera's n_row x n_col");
    v.orig[c] = PlaneView{im.buf.as<unsigned char>(), im.pitch, im.H, im.W, im.dtype};
  }
  v.n_tiles = tiles;
  const size_t rsz = fp64 ? 8 : 4;
  size_t off = 0;
  off += (size_t)v.n_cam * v.roi_area * rsz;
  off = (off + 15) / 16 * 16;
  v.off_dd = off;
  if (fp64) off += (size_t)v.n_cam * v.roi_area * 8;
  off = (off + 15) / 16 * 16;
  v.off_otf = off;
  off += 3 * (size_t)v.n_cam * 5 * rsz;  // three trial points (slot 0: single evaluations)
  off = (off + 15) / 16 * 16;
  v.off_uv = off;
  off += 3 * (size_t)v.n_cam * 2 * 8;
  v.smem_per_warp = (off + 15) / 16 * 16;
  return v;
}

static void ensure_residual_planes(olpt_ctx* ctx, ShakeView& v, bool fp64) {
  const int dt = fp64 ? OLPT_F64 : OLPT_F32;
  const int esz = fp64 ? 8 : 4;
  for (int c = 0; c < ctx->n_cam; ++c) {
    ImagePlane& r = ctx->resid[c];
    const CamDev& cm = ctx->cams_h[c];
    const int64_t pitch = ((int64_t)cm.n_col * esz + 15) / 16 * 16;
    r.buf.ensure((size_t)pitch * cm.n_row + 64, ctx->stream);
    r.dtype = dt;
    r.H = cm.n_row;
    r.W = cm.n_col;
    r.pitch = pitch;
    v.res[c] = PlaneView{r.buf.as<unsigned char>(), r.pitch, r.H, r.W, dt};
  }
}

template <typename Real>
static void residual_pass(olpt_ctx* ctx, ShakeView& v, const uint8_t* flags, int all_cams,
                          int clamp) {
  cudaStream_t s = ctx->stream;
  ShakeWork& W = ctx->shk;
  const int64_t n = ctx->obj.n;
  const int C = ctx->n_cam;
  W.otfp.ensure((n * C + 1) * 5 * sizeof(Real), s);
  W.pair_key.ensure((n * C + 1) * sizeof(int), s);
  if (n > 0)
    prep_kernel<Real><<<OLPT_G(nblk(n, 128)), 128, 0, s>>>(v, ctx->obj.xyz.as<double>(), n,
                                                   ctx->obj.uv.as<double>(), W.otfp.as<Real>(),
                                                   W.pair_key.as<int>(), flags, all_cams);
  OLPT_CUDA(cudaGetLastError());
  W.bins.build(W.pair_key.as<int>(), (int)(n * C), v.n_tiles, s);
  // algorithmic bytes: read the image, write the residual, for every computed camera
  double bytes = 0;
  for (int c = 0; c < C; ++c) {
    if (!(all_cams || ctx->cams_h[c].is_active)) continue;
    const int d = v.orig[c].dtype;
    const int esz = d == OLPT_U8 ? 1 : d == OLPT_U16 ? 2 : d == OLPT_F32 ? 4 : 8;
    bytes += (double)v.orig[c].H * v.orig[c].W * (esz + sizeof(Real));
  }
  const int pid = ctx->prof.begin(PROF_RESIDUAL, s);
  residual_kernel<Real><<<OLPT_G(v.n_tiles), ctx->tune.residual_threads, 0, s>>>(v, ctx->obj.uv.as<double>(), W.otfp.as<Real>(),
                                                  W.bins.start.as<int>(), W.bins.items.as<int>(),
                                                  clamp, all_cams);
  ctx->prof.end(PROF_RESIDUAL, pid, s, bytes);
  OLPT_CUDA(cudaGetLastError());
}

// shake_kernel instantiated per camera count (per-camera arrays in registers)
template <typename Real, int NC, int MINB>
static void launch_shake_nb(int grid, int block, size_t smem, cudaStream_t s, const ShakeView& v,
                            int64_t n, double* xyz, double* uv, const Real* otfp, double* score,
                            double delta, const uint8_t* active, double* resid_out) {
  OLPT_CUDA(cudaFuncSetAttribute(shake_kernel<Real, NC, MINB>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  shake_kernel<Real, NC, MINB><<<OLPT_G(grid), block, smem, s>>>(v, n, xyz, uv, otfp, score,
                                                                 delta, active, resid_out);
}

// the kernel variant of the context's register budget (64 or 128 a thread)
template <typename Real, int NC>
static void launch_shake_nc(int grid, int block, size_t smem, cudaStream_t s, const ShakeView& v,
                            int64_t n, double* xyz, double* uv, const Real* otfp, double* score,
                            double delta, const uint8_t* active, double* resid_out, int regs) {
  if (regs >= 128)
    launch_shake_nb<Real, NC, 4>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active,
                                 resid_out);
  else
    launch_shake_nb<Real, NC, 8>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active,
                                 resid_out);
}

template <typename Real>
static void launch_shake(int C, int grid, int block, size_t smem, cudaStream_t s,
                         const ShakeView& v, int64_t n, double* xyz, double* uv, const Real* otfp,
                         double* score, double delta, const uint8_t* active, double* resid_out,
                         int regs) {
  switch (C) {
    case 2: launch_shake_nc<Real, 2>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active, resid_out, regs); break;
    case 3: launch_shake_nc<Real, 3>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active, resid_out, regs); break;
    case 4: launch_shake_nc<Real, 4>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active, resid_out, regs); break;
    case 5: launch_shake_nc<Real, 5>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active, resid_out, regs); break;
    case 6: launch_shake_nc<Real, 6>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active, resid_out, regs); break;
    case 7: launch_shake_nc<Real, 7>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active, resid_out, regs); break;
    default: launch_shake_nc<Real, 8>(grid, block, smem, s, v, n, xyz, uv, otfp, score, delta, active, resid_out, regs); break;
  }
}

// n_loop shake iterations from the width delta (halved per iteration, clamped at the
// minimum); objects with active[o] == 0 stay fixed but still enter the residual
template <typename Real>
static void shake_iterations(olpt_ctx* ctx, const ShakeParams& sp, ShakeView& v, int n_loop,
                             double delta, const uint8_t* active, double* resid_out) {
  cudaStream_t s = ctx->stream;
  const int64_t n = ctx->obj.n;
  const int C = ctx->n_cam;
  ShakeWork& W = ctx->shk;
  double dmin = sp.shakewidth_min;
  dmin = (dmin > 0) ? dmin : sp.shake_width / 20;
  const int warps_per_blk = ctx->tune.shake_warps_per_block;  // 1, 2 or 4 (bound: 128 threads)
  const size_t smem = v.smem_per_warp * warps_per_blk;

  for (int it = 0; it < n_loop; ++it) {
    residual_pass<Real>(ctx, v, nullptr, 0, 0);
    // algorithmic bytes: the augmented ROI of every active camera plus the object
    // state (xyz, projections, OTF parameters, score) read and written once
    int n_act = 0;
    for (int c = 0; c < C; ++c) n_act += ctx->cams_h[c].is_active;
    const double bytes = (double)n * (n_act * v.roi_area * (double)sizeof(Real) +
                                      2.0 * (3 * 8 + C * 2 * 8 + 8) + C * 5.0 * sizeof(Real));
    const int pid = ctx->prof.begin(PROF_SHAKE, s);
    if (n > 0)
      launch_shake<Real>(C, nblk(n, warps_per_blk), 32 * warps_per_blk, smem, s, v, n,
                         ctx->obj.xyz.as<double>(), ctx->obj.uv.as<double>(), W.otfp.as<Real>(),
                         ctx->obj.score.as<double>(), delta, active, resid_out,
                         ctx->tune.shake_regs);
    ctx->prof.end(PROF_SHAKE, pid, s, bytes);
    OLPT_CUDA(cudaGetLastError());
    delta *= 0.5;
    if (delta < dmin) delta = dmin;
  }
}

// Shake::runShake (Shake.cpp:103-136): repeated objects (greedy over the tol_3d
// neighbourhood) and ghosts (score below thred_ghost x mean score)
static void shake_flags(olpt_ctx* ctx, const ShakeParams& sp) {
  cudaStream_t s = ctx->stream;
  const int64_t n = ctx->obj.n;
  ShakeWork& W = ctx->shk;
  W.rep.ensure(n + 16, s);
  OLPT_CUDA(cudaMemsetAsync(W.rep.p, 0, n + 16, s));
  if (n > 0) {
    const double cell = std::max(sp.tol_3d_mm, 1e-9);
    const int nb = (int)std::max<int64_t>(1024, 2 * n);
    W.hkey.ensure((n + 1) * sizeof(int), s);
    W.has_nb.ensure((n + 1) * sizeof(int), s);
    hash_key_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.xyz.as<double>(), (int)n, cell, nb,
                                             W.hkey.as<int>());
    W.hash.build(W.hkey.as<int>(), (int)n, nb, s);
    const double r2 = sp.tol_3d_mm * sp.tol_3d_mm;
    neighbour_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.xyz.as<double>(), (int)n, cell, nb,
                                              W.hash.start.as<int>(), W.hash.items.as<int>(), r2,
                                              W.has_nb.as<int>());
    // ascending list of the objects that have neighbours (order-preserving compaction)
    W.nb_pos.ensure((n + 1) * sizeof(int), s);
    W.nb_list.ensure((n + 1) * sizeof(int), s);
    exclusive_scan(W.has_nb.as<int>(), (int)n, W.nb_pos.as<int>(), W.scan_tmp, s);
    compact_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(W.has_nb.as<int>(), W.nb_pos.as<int>(), (int)n,
                                                  W.nb_list.as<int>());
    repeat_greedy_kernel<<<OLPT_G(1), 32, 0, s>>>(ctx->obj.xyz.as<double>(), (int)n, cell, nb,
                                          W.hash.start.as<int>(), W.hash.items.as<int>(), r2,
                                          W.nb_list.as<int>(), W.nb_pos.as<int>() + n,
                                          W.rep.as<uint8_t>());
    const int sb = std::max(1, std::min(kScoreBlocks, nblk(n)));
    W.gpart.ensure((size_t)sb * 3 * sizeof(double) + sizeof(int) + 64, s);
    int* amb = reinterpret_cast<int*>(W.gpart.as<double>() + 3 * sb);
    OLPT_CUDA(cudaMemsetAsync(amb, 0, sizeof(int), s));
    score_partial_kernel<<<OLPT_G(sb), 256, 0, s>>>(ctx->obj.score.as<double>(),
                                                    W.rep.as<uint8_t>(), (int)n,
                                                    W.gpart.as<double>());
    ghost_flag_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.score.as<double>(),
                                                      W.rep.as<uint8_t>(), (int)n, sp.thred_ghost,
                                                      W.gpart.as<double>(), sb,
                                                      ctx->obj.flags.as<uint8_t>(), amb);
    ghost_kernel<<<OLPT_G(1), 1024, 0, s>>>(ctx->obj.score.as<double>(), W.rep.as<uint8_t>(), (int)n,
                                    sp.thred_ghost, ctx->obj.flags.as<uint8_t>(), amb);
    OLPT_CUDA(cudaGetLastError());
  }
}

template <typename Real>
static void shake_impl(olpt_ctx* ctx, const ShakeParams& sp) {
  const bool fp64 = sizeof(Real) == 8;
  cudaStream_t s = ctx->stream;
  ShakeView v = make_view(ctx, sp, fp64);
  ensure_residual_planes(ctx, v, fp64);
  const int64_t n = ctx->obj.n;
  ctx->obj.ensure(std::max<int64_t>(n, 1), ctx->n_cam, s);
  if (n > 0) fill_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.score.as<double>(), n, 1.0);
  shake_iterations<Real>(ctx, sp, v, sp.n_shake_loop, sp.shake_width, nullptr, nullptr);
  shake_flags(ctx, sp);
}

template <typename Real>
static void learned_impl(olpt_ctx* ctx, const ShakeParams& sp) {
  const bool fp64 = sizeof(Real) == 8;
  cudaStream_t s = ctx->stream;
  MlpWork& M = ctx->mlp;
  const LearnedParams& lp = M.lp;
  ShakeView v = make_view(ctx, sp, fp64);
  ensure_residual_planes(ctx, v, fp64);
  int64_t n = ctx->obj.n;
  const int C = ctx->n_cam;
  if (n > 0) {
    // 1. residual with every candidate at its stereo position, features, network
    residual_pass<Real>(ctx, v, nullptr, 0, 0);
    M.x.ensure((size_t)n * M.dims.in_pad * 2, s);
    mlp_features_device(ctx, sp, M.x.as<__nv_bfloat16>(), nullptr);
    M.o.ensure((size_t)n * kMlpOut * 4, s);
    mlp_infer_device(ctx, M.x.as<__nv_bfloat16>(), n, M.o.as<float>());
    // 2. correction, and the network's ghosts leave before any shaking
    M.keep.ensure((size_t)(n + 1) * sizeof(int), s);
    M.pos.ensure((size_t)(n + 1) * sizeof(int), s);
    M.start_xyz.ensure((size_t)n * 3 * sizeof(double), s);
    OLPT_CUDA(cudaMemcpyAsync(M.start_xyz.p, ctx->obj.xyz.p, (size_t)n * 3 * sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
    learned_apply_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.xyz.as<double>(), M.o.as<float>(),
                                                        n, lp.out_scale_mm, (float)lp.ghost_logit,
                                                        M.keep.as<int>());
    exclusive_scan(M.keep.as<int>(), (int)n, M.pos.as<int>(), ctx->shk.scan_tmp, s);
    int kept = 0;
    OLPT_CUDA(cudaMemcpyAsync(&kept, M.pos.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    // compacted copies (through the scratch pair act / nres, then back)
    M.act.ensure((size_t)(n + 1) * 3 * sizeof(double), s);
    M.nres.ensure((size_t)(n + 1) * 3 * sizeof(double), s);
    compact_xyz_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(
        M.keep.as<int>(), M.pos.as<int>(), n, ctx->obj.xyz.as<double>(), M.act.as<double>(),
        M.start_xyz.as<double>(), M.nres.as<double>());
    OLPT_CUDA(cudaGetLastError());
    n = kept;
    ctx->obj.n = n;
    if (n > 0) {
      OLPT_CUDA(cudaMemcpyAsync(ctx->obj.xyz.p, M.act.p, (size_t)n * 3 * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
      OLPT_CUDA(cudaMemcpyAsync(M.start_xyz.p, M.nres.p, (size_t)n * 3 * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
    }
  }
  ctx->obj.ensure(std::max<int64_t>(n, 1), C, s);
  if (n > 0) {
    // 3. short plain refinement from the corrected positions
    fill_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->obj.score.as<double>(), n, 1.0);
    M.nres.ensure((size_t)(n + 1) * sizeof(double), s);
    shake_iterations<Real>(ctx, sp, v, lp.refine_loops, lp.refine_width_mm, nullptr,
                           M.nres.as<double>());
    // 4. fallback: the full plain shake for objects whose residue stays high
    M.act.ensure((size_t)n + 16, s);
    M.fb.ensure(16, s);
    int* cnt = M.fb.as<int>();
    OLPT_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
    fallback_kernel<Real><<<OLPT_G(nblk(n)), 256, 0, s>>>(
        M.nres.as<double>(), ctx->shk.otfp.as<Real>(), ctx->cams_d.as<CamDev>(), C, n,
        lp.fallback_residual, M.act.as<uint8_t>(), ctx->obj.xyz.as<double>(),
        M.start_xyz.as<double>(), ctx->obj.score.as<double>(), cnt);
    OLPT_CUDA(cudaGetLastError());
    int n_fb = 0;
    OLPT_CUDA(cudaMemcpyAsync(&n_fb, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    M.n_fallback += n_fb;
    M.n_learned += n;
    if (n_fb > 0)
      shake_iterations<Real>(ctx, sp, v, sp.n_shake_loop, sp.shake_width, M.act.as<uint8_t>(),
                             nullptr);
    if (lp.refine_loops > 0 && lp.refine_loops != sp.n_shake_loop)
      score_scale_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(
          ctx->obj.score.as<double>(), M.act.as<uint8_t>(), n,
          (double)sp.n_shake_loop / (double)lp.refine_loops);
    OLPT_CUDA(cudaGetLastError());
  }
  shake_flags(ctx, sp);
}

void residual_all_device(olpt_ctx* ctx, const ShakeParams& sp) {
  const bool fp64 = sp.precision == 1;
  ShakeView v = make_view(ctx, sp, fp64);
  ensure_residual_planes(ctx, v, fp64);
  if (fp64)
    residual_pass<double>(ctx, v, nullptr, 0, 0);
  else
    residual_pass<float>(ctx, v, nullptr, 0, 0);
}

void learned_shake_device(olpt_ctx* ctx, const ShakeParams& sp) {
  OLPT_REQUIRE(ctx->mlp.ready, OLPT_ERR_INVALID_ARG, "learned shake: network not initialised");
  OLPT_REQUIRE(ctx->n_cam == ctx->mlp.dims.cams, OLPT_ERR_UNSUPPORTED,
               "learned shake: the network was built for " + std::to_string(ctx->mlp.dims.cams) +
                   " cameras, the rig has " + std::to_string(ctx->n_cam));
  if (sp.precision == 1)
    learned_impl<double>(ctx, sp);
  else
    learned_impl<float>(ctx, sp);
}

void shake_device(olpt_ctx* ctx, const ShakeParams& sp) {
  OLPT_REQUIRE(ctx->n_cam >= 2, OLPT_ERR_INVALID_ARG, "shake needs at least 2 cameras");
  if (sp.precision == 1)
    shake_impl<double>(ctx, sp);
  else
    shake_impl<float>(ctx, sp);
}

// Shake::calResidualImage (output_ipr = true): every camera, clamped at 0, objects
// flagged Ghost/Repeated skipped when use_flags.  The result replaces the current
// images when make_current.
void residual_device(olpt_ctx* ctx, const ShakeParams& sp, bool use_flags, bool make_current) {
  const bool fp64 = sp.precision == 1;
  ShakeView v = make_view(ctx, sp, fp64);
  ensure_residual_planes(ctx, v, fp64);
  const uint8_t* fl = use_flags ? ctx->obj.flags.as<uint8_t>() : nullptr;
  if (fp64)
    residual_pass<double>(ctx, v, fl, 1, 1);
  else
    residual_pass<float>(ctx, v, fl, 1, 1);
  if (make_current)
    for (int c = 0; c < ctx->n_cam; ++c) std::swap(ctx->img[c], ctx->resid[c]);
}

}  // namespace olpt
