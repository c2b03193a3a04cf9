// Kernel family (d): the Shake-the-Box frame loop -- track prediction, repeat
// check, nearest-neighbour linking over device hash grids, linear-fit pruning and
// the initial-phase predictive field.
//
// Reference: STB::processFrame / runInitPhase / buildTrackFromPredField /
// predictNext / findNN / runConvPhase / checkRepeat / linkShortTrack /
// checkLinearFit / saveTracks / loadTracks (src/srcSTB/STB.cpp:40-1076),
// PredField (src/srcSTB/PredField.cpp), Object3D::isReconstructable
// (src/srcObject/ObjectInfo.cpp:3-30).
//
// Layout: the track containers stay on the host in the reference's order (four
// deques, the same moves between them); per frame the per-track numerics run on
// the device over packed arrays:
//  * predict_kernel: one thread per long track, the Wiener/LMS filter in FP64, then
//    the view-volume test and the camera-visibility test;
//  * the predictions go through the device shake and residual (shake.cu), the
//    residual through the device IPR (ipr.cu);
//  * repeat_kernel / link_kernel / nn_kernel: radius and nearest-neighbour queries
//    over CSR hash grids (cell >= the query radius, 27 cells) that stand in for
//    nanoflann; nearest-neighbour ties go to the lowest index;
//  * linfit_kernel: one thread per track;
//  * pf_node_kernel: one CTA per predictive-field node, neighbour lists from hash
//    grids, the displacement PDF in shared memory, peak and 3-point Gaussian fit;
//    pf_smooth_kernel: the separable Gaussian smoothing.
// Exactness: every per-track formula follows the reference's operation order in
// FP64.  Two sums have no fixed order in the reference's own terms -- the
// neighbour-track averages of linkShortTrack (nanoflann traversal order) and the
// PDF bins -- and are summed here in grid order and by shared-memory atomics:
// equal up to rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_otf.cuh"
#include "olpt_scan.cuh"
#include "olpt_stb.h"

namespace olpt {
namespace {

inline int nblk(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

// Margin on hash-grid cells so that every point within the query radius lies in
// one of the 27 cells around the query despite the rounding of x / cell.
constexpr double kCellMargin = 1.001;
constexpr int kLinkIters = 5;              // linkShortTrack(track, 5, ...), STB.cpp:497
constexpr int kLenLongTrack = 7;           // LEN_LONG_TRACK, STBCommons.h
constexpr double kMaxErrLinearFit = 5e-2;  // MAX_ERR_LINEARFIT, STBCommons.h:31

// ---------------------------------------------------------------- hash grid
struct HashGrid {
  double cell;
  int n_buckets;
  const int* start;
  const int* items;
  const double* pts;  // n x 3, the points the grid was built from (null: empty)
};

__device__ __forceinline__ int hash_bucket(long long cx, long long cy, long long cz, int nb) {
  const unsigned long long h = (unsigned long long)(cx * 73856093LL) ^
                               (unsigned long long)(cy * 19349663LL) ^
                               (unsigned long long)(cz * 83492791LL);
  return (int)(h % (unsigned long long)nb);
}

__global__ void hash_keys_kernel(const double* pts, int n, double cell, int nb, int* key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = hash_bucket((long long)floor(pts[3 * i] / cell), (long long)floor(pts[3 * i + 1] / cell),
                       (long long)floor(pts[3 * i + 2] / cell), nb);
}

// The distinct buckets of the 27 cells around q (a bucket shared by two cells is
// scanned once).
__device__ __forceinline__ int cell_buckets(const HashGrid& g, const double q[3], int out[27]) {
  if (!g.pts) return 0;
  const long long cx = (long long)floor(q[0] / g.cell), cy = (long long)floor(q[1] / g.cell),
                  cz = (long long)floor(q[2] / g.cell);
  int n = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int b = hash_bucket(cx + dx, cy + dy, cz + dz, g.n_buckets);
        bool dup = false;
        for (int e = 0; e < n; ++e) dup |= (out[e] == b);
        if (!dup) out[n++] = b;
      }
  return n;
}

// nanoflann L2_Simple_Adaptor::evalMetric: the squared differences summed in
// dimension order.
__device__ __forceinline__ double l2sq(const double* a, const double* b) {
  double r = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double t = a[d] - b[d];
    r += t * t;
  }
  return r;
}

// STB::findNN (STB.cpp:318-335): the nearest point, accepted when its squared
// distance is below radius^2; -1 (UNLINKED) otherwise.
__device__ int grid_nearest(const HashGrid& g, const double q[3], double r2) {
  int bk[27];
  const int nb = cell_buckets(g, q, bk);
  int best = -1;
  double bd = 0.0;
  for (int e = 0; e < nb; ++e)
    for (int s = g.start[bk[e]]; s < g.start[bk[e] + 1]; ++s) {
      const int j = g.items[s];
      const double d2 = l2sq(q, g.pts + 3 * (int64_t)j);
      if (best < 0 || d2 < bd || (d2 == bd && j < best)) {
        best = j;
        bd = d2;
      }
    }
  return (best >= 0 && bd < r2) ? best : -1;
}

// ---------------------------------------------------------------- prediction
// STB::predictNext (STB.cpp:233-316) on the last min(len, 6) points of each track,
// then AxisLimit::check (STBCommons.h:142-150) and Object3D::isReconstructable
// (ObjectInfo.cpp:3-30; y is compared with the column count there, kept as is).
__global__ void predict_kernel(const double* pts, const int* npts, int n, StbView v,
                               double* pred, int* in_range) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int len = npts[i];
  const double* P = pts + (int64_t)i * 18;
  const int order = (len < 6) ? len - 1 : 5;
  const int start = len - 1 - order;
  double out[3];
  for (int axis = 0; axis < 3; ++axis) {
    double s[6];
    for (int j = 0; j <= order; ++j) s[j] = P[3 * (start + j) + axis];
    bool shifted = false;
    if (fabs(s[order]) < 1.0) {
      shifted = true;
      for (int j = 0; j <= order; ++j) s[j] += 10.0;
    }
    double denom = 0.0;
    for (int j = 0; j < order; ++j) denom += s[j] * s[j];
    const double step = (denom > 1e-12) ? (1.0 / denom) : 0.0;
    double f[5] = {0, 0, 0, 0, 0};
    double prediction = 0.0;
    double error = s[order] - prediction;
    int iter = 0;
    while (fabs(error) > 1e-8 && iter < 5000 && step > 0.0) {
      prediction = 0.0;
      for (int j = 0; j < order; ++j) {
        f[j] += step * s[j] * error;
        prediction += f[j] * s[j];
      }
      error = s[order] - prediction;
      ++iter;
    }
    if (order >= 1 && step == 0.0) {
      prediction = s[order] + (s[order] - s[order - 1]);
    } else {
      prediction = 0.0;
      for (int j = 0; j < order; ++j) prediction += f[j] * s[j + 1];
    }
    if (shifted) prediction -= 10.0;
    out[axis] = prediction;
  }
  pred[3 * i] = out[0];
  pred[3 * i + 1] = out[1];
  pred[3 * i + 2] = out[2];
  int ok = !(out[0] > v.limit[1] || out[0] < v.limit[0] || out[1] > v.limit[3] ||
             out[1] < v.limit[2] || out[2] > v.limit[5] || out[2] < v.limit[4]);
  if (ok) {
    int n_out = 0;
    for (int c = 0; c < v.n_cam; ++c) {
      double x, y;
      cam_project(v.cams[c], out[0], out[1], out[2], x, y);
      if (x < 0 || x >= v.cams[c].n_col || y < 0 || y >= v.cams[c].n_col) {
        ++n_out;
        if (v.n_cam - n_out < 2) {
          ok = 0;
          break;
        }
      }
    }
  }
  in_range[i] = ok;
}

// ---------------------------------------------------------------- repeat check
// STB::checkRepeat (STB.cpp:698-741): an object within tol (Pt3D::norm <= tol,
// tracers have no radius) of any active long track's last point is Repeated.
__global__ void repeat_kernel(const double* obj, int n, HashGrid g, double tol, int* rep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = obj + 3 * (int64_t)i;
  int bk[27];
  const int nb = cell_buckets(g, p, bk);
  int r = 0;
  for (int e = 0; e < nb && !r; ++e)
    for (int s = g.start[bk[e]]; s < g.start[bk[e] + 1]; ++s) {
      const double* q = g.pts + 3 * (int64_t)g.items[s];
      const double d0 = p[0] - q[0], d1 = p[1] - q[1], d2 = p[2] - q[2];
      if (sqrt(d0 * d0 + d1 * d1 + d2 * d2) <= tol) {
        r = 1;
        break;
      }
    }
  rep[i] = r;
}

// ---------------------------------------------------------------- linking
// STB::linkShortTrack (STB.cpp:743-872) for every active short track.  tg: grid
// over the long tracks' second-to-last points rounded to float (TrackCloud,
// inc/libSTB/Track.h:49-62), disp: their last displacement; go: grid over the new
// objects.  len: points in the short track (an empty track is UNLINKED).
__global__ void link_kernel(const double* p_last, const int* len, int n_sa, HashGrid tg,
                            const double* disp, HashGrid go, double base_r, int* link) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_sa) return;
  if (len[i] == 0 || !(base_r > 0.0)) {
    link[i] = -1;
    return;
  }
  const double* p = p_last + 3 * (int64_t)i;
  int bk[27];
  const int nb = cell_buckets(tg, p, bk);
  // the radius of every step (factor 1, 1.1, 1.1 * 1.1, ...); the neighbour sums of all
  // steps are accumulated in one scan each (same neighbour order as one scan per step,
  // so the same sums)
  double fac[kLinkIters], r2[kLinkIters];
#pragma unroll
  for (int st = 0; st < kLinkIters; ++st) {
    fac[st] = (st == 0) ? 1.0 : fac[st - 1] * 1.1;
    const double r_track = (3.0 * base_r) * fac[st];
    r2[st] = r_track * r_track;
  }
  int cnt[kLinkIters];
  double mean_d2[kLinkIters];
#pragma unroll
  for (int st = 0; st < kLinkIters; ++st) {
    cnt[st] = 0;
    mean_d2[st] = 0.0;
  }
  for (int e = 0; e < nb; ++e)
    for (int s = tg.start[bk[e]]; s < tg.start[bk[e] + 1]; ++s) {
      const double d2 = l2sq(p, tg.pts + 3 * (int64_t)tg.items[s]);
#pragma unroll
      for (int st = 0; st < kLinkIters; ++st)
        if (d2 < r2[st]) {
          ++cnt[st];
          mean_d2[st] += d2;
        }
    }
  double beta2[kLinkIters];
  bool any = false;
#pragma unroll
  for (int st = 0; st < kLinkIters; ++st) {
    beta2[st] = 0.0;
    if (cnt[st] > 0) {
      any = true;
      const double m = mean_d2[st] / (double)cnt[st];
      const double alpha = 0.8;
      double L2 = (alpha * alpha) * m;
      const double R = base_r * fac[st];
      const double Lmin2 = (0.1 * R) * (0.1 * R);
      const double Lmax2 = (0.8 * R) * (0.8 * R);
      L2 = (L2 < Lmin2) ? Lmin2 : ((Lmax2 < L2) ? Lmax2 : L2);  // std::clamp
      beta2[st] = 1.0 / (L2 + 1e-12);
    }
  }
  double sum_w[kLinkIters], sx[kLinkIters], sy[kLinkIters], sz[kLinkIters];
#pragma unroll
  for (int st = 0; st < kLinkIters; ++st) sum_w[st] = sx[st] = sy[st] = sz[st] = 0.0;
  if (any)
    for (int e = 0; e < nb; ++e)
      for (int s = tg.start[bk[e]]; s < tg.start[bk[e] + 1]; ++s) {
        const int j = tg.items[s];
        const double d2 = l2sq(p, tg.pts + 3 * (int64_t)j);
        if (!(d2 < r2[kLinkIters - 1])) continue;
        const double dx = disp[3 * (int64_t)j], dy = disp[3 * (int64_t)j + 1],
                     dz = disp[3 * (int64_t)j + 2];
#pragma unroll
        for (int st = 0; st < kLinkIters; ++st) {
          if (cnt[st] == 0 || !(d2 < r2[st])) continue;
          const double w = 1.0 / (1.0 + d2 * beta2[st]);
          sum_w[st] += w;
          sx[st] += w * dx;
          sy[st] += w * dy;
          sz[st] += w * dz;
        }
      }
  int obj_id = -1;
#pragma unroll
  for (int st = 0; st < kLinkIters; ++st) {
    double vel[3] = {0.0, 0.0, 0.0};
    if (cnt[st] > 0 && sum_w[st] > 0.0) {
      const double inv = 1.0 / sum_w[st];
      vel[0] = sx[st] * inv;
      vel[1] = sy[st] * inv;
      vel[2] = sz[st] * inv;
    }
    const double est[3] = {p[0] + vel[0], p[1] + vel[1], p[2] + vel[2]};
    const double r_obj = base_r * fac[st];
    obj_id = grid_nearest(go, est, r_obj * r_obj);
    if (obj_id >= 0) break;
    if (cnt[st] == 0) {
      obj_id = grid_nearest(go, p, r_obj * r_obj);
      if (obj_id >= 0) break;
    }
  }
  link[i] = obj_id;
}

// Nearest object within the radius for every query point (initial phase).
__global__ void nn_kernel(const double* q, int n, HashGrid go, double r2, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = grid_nearest(go, q + 3 * (int64_t)i, r2);
}

// ---------------------------------------------------------------- linear fit
// STB::checkLinearFit (STB.cpp:874-924): least-squares line through the last n_pts
// points (kern = inverse(X^T X) X^T, 2 x n_pts); kept when the distance of the last
// point to the fitted one is not above MAX_ERR_LINEARFIT.
__global__ void linfit_kernel(const double* pts, const int* len, int n, int n_pts,
                              const double* kern, int* ok) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (len[i] < n_pts) {
    ok[i] = 0;
    return;
  }
  const double* P = pts + (int64_t)i * 12;
  double est[3];
  for (int d = 0; d < 3; ++d) {
    double c0 = 0.0, c1 = 0.0;
    for (int j = 0; j < n_pts; ++j) c0 += kern[j] * P[3 * j + d];
    for (int j = 0; j < n_pts; ++j) c1 += kern[n_pts + j] * P[3 * j + d];
    est[d] = c0 + (n_pts - 1) * c1;
  }
  const double* L = P + 3 * (n_pts - 1);
  // myMATH::dist (myMATH.cpp:257-268, 325-328)
  double r = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double t = est[d] - L[d];
    r += t * t;
  }
  r = (r < 0.0) ? 0.0 : r;
  ok[i] = !(sqrt(r) > kMaxErrLinearFit);
}

// ---------------------------------------------------------------- predictive field
constexpr int kPfMaxNb = 4096;  // objects of one frame inside one search cube

// PredField::calPredField (PredField.cpp:20-90), one grid node per CTA:
// findNeighbor (|d| < r on every axis, :205-231), updateDispPDF (:247-283),
// findPDFPeakID / findPDFPeakLoc / fitPeakBinLocGauss (:286-369).
__global__ void __launch_bounds__(256) pf_node_kernel(PfView pf, HashGrid gp, HashGrid gc,
                                                      double* field, int* overflow) {
  extern __shared__ __align__(16) unsigned char pf_smem[];
  double* pdf = reinterpret_cast<double*>(pf_smem);
  int* lp = reinterpret_cast<int*>(pdf + pf.nbin_tot);
  int* lc = lp + kPfMaxNb;
  __shared__ int n_nb[2];
  __shared__ int s_peak;
  __shared__ double s_peakv;
  const int g = blockIdx.x;
  const int zi = g % pf.nz, yi = (g / pf.nz) % pf.ny, xi = g / (pf.ny * pf.nz);
  // myMATH::linspace nodes (myMATH.cpp:9-33)
  const double node[3] = {pf.lo[0] + pf.d[0] * xi, pf.lo[1] + pf.d[1] * yi,
                          pf.lo[2] + pf.d[2] * zi};
  if (threadIdx.x < 2) n_nb[threadIdx.x] = 0;
  for (int b = threadIdx.x; b < pf.nbin_tot; b += blockDim.x) pdf[b] = 0.0;
  __syncthreads();
  for (int which = 0; which < 2; ++which) {
    const HashGrid& G = which == 0 ? gp : gc;
    int* list = which == 0 ? lp : lc;
    int bk[27];
    const int nb = cell_buckets(G, node, bk);
    for (int e = threadIdx.x / 32; e < nb; e += blockDim.x / 32)
      for (int s = G.start[bk[e]] + (threadIdx.x & 31); s < G.start[bk[e] + 1]; s += 32) {
        const int j = G.items[s];
        const double* q = G.pts + 3 * (int64_t)j;
        const double dx = q[0] - node[0], dy = q[1] - node[1], dz = q[2] - node[2];
        if (dx < pf.r && dx > -pf.r && dy < pf.r && dy > -pf.r && dz < pf.r && dz > -pf.r) {
          const int slot = atomicAdd(&n_nb[which], 1);
          if (slot < kPfMaxNb) list[slot] = j;
        }
      }
  }
  __syncthreads();
  const int n_p = n_nb[0], n_c = n_nb[1];
  if (n_p > kPfMaxNb || n_c > kPfMaxNb) {
    if (threadIdx.x == 0) atomicExch(overflow, 1);
    return;
  }
  double* out = field + 3 * (int64_t)g;
  if (n_p == 0 || n_c == 0) {
    if (threadIdx.x < 3) out[threadIdx.x] = 0.0;
    return;
  }
  const int nyz = pf.nbin[1] * pf.nbin[2];
  const int n_pair = n_p * n_c;
  for (int t = threadIdx.x; t < n_pair; t += blockDim.x) {
    const double* a = gc.pts + 3 * (int64_t)lc[t / n_p];
    const double* b = gp.pts + 3 * (int64_t)lp[t % n_p];
    const double xb = pf.m[0] * (a[0] - b[0]) + pf.c[0];
    const double yb = pf.m[1] * (a[1] - b[1]) + pf.c[1];
    const double zb = pf.m[2] * (a[2] - b[2]) + pf.c[2];
    const int xi0 = (int)round(xb), yi0 = (int)round(yb), zi0 = (int)round(zb);
    for (int i = max(0, xi0 - 1); i <= min(pf.nbin[0] - 1, xi0 + 1); ++i) {
      const double xx = i - xb;
      for (int j = max(0, yi0 - 1); j <= min(pf.nbin[1] - 1, yi0 + 1); ++j) {
        const double yy = j - yb;
        for (int k = max(0, zi0 - 1); k <= min(pf.nbin[2] - 1, zi0 + 1); ++k) {
          const double zz = k - zb;
          atomicAdd(&pdf[i * nyz + j * pf.nbin[2] + k], exp(-(xx * xx + yy * yy + zz * zz)));
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // std::max_element: the first maximum
    int bi = 0;
    double bv = pdf[0];
    for (int b = 1; b < pf.nbin_tot; ++b)
      if (bv < pdf[b]) {
        bv = pdf[b];
        bi = b;
      }
    s_peak = bi;
    s_peakv = bv;
  }
  __syncthreads();
  if (threadIdx.x >= 3) return;
  const int ax = threadIdx.x;
  int pk[3] = {-1, -1, -1};
  if (s_peakv > 1e-1) {
    pk[0] = s_peak / nyz;
    pk[1] = (s_peak - pk[0] * nyz) / pf.nbin[2];
    pk[2] = s_peak % pf.nbin[2];
  }
  double res;
  if (pk[ax] < 0) {
    res = 0.0;
  } else if (pk[ax] == 0) {
    res = -2 * pf.r;
  } else if (pk[ax] == pf.nbin[ax] - 1) {
    res = 2 * pf.r;
  } else {
    int a1[3] = {pk[0], pk[1], pk[2]}, a3[3] = {pk[0], pk[1], pk[2]};
    a1[ax] -= 1;
    a3[ax] += 1;
    const double v1 = pdf[a1[0] * nyz + a1[1] * pf.nbin[2] + a1[2]];
    const double v2 = pdf[pk[0] * nyz + pk[1] * pf.nbin[2] + pk[2]];
    const double v3 = pdf[a3[0] * nyz + a3[1] * pf.nbin[2] + a3[2]];
    const double y1 = pk[ax] - 1, y2 = pk[ax], y3 = pk[ax] + 1;
    const double l1 = v1 < 1e-4 ? log(1e-4) : log(v1);
    const double l2 = v2 < 1e-4 ? log(1e-4) : log(v2);
    const double l3 = v3 < 1e-4 ? log(1e-4) : log(v3);
    double yc = -0.5 *
                ((l1 * double((y2 * y2) - (y3 * y3))) - (l2 * double((y1 * y1) - (y3 * y3))) +
                 (l3 * double((y1 * y1) - (y2 * y2)))) /
                ((l1 * double(y3 - y2)) - (l3 * double(y1 - y2)) + (l2 * double(y1 - y3)));
    if (!isfinite(yc)) yc = y2;
    res = (yc - pf.c[ax]) / pf.m[ax];
  }
  out[ax] = res;
}

// One pass of PredField::applyGaussian (PredField.cpp:372-452): component `comp`
// convolved along axis `dir` (src -> dst).
__global__ void pf_smooth_kernel(PfView pf, const double* src, double* dst, int comp, int dir,
                                 const double* kern, int radius) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= pf.nx * pf.ny * pf.nz) return;
  const int z = g % pf.nz, y = (g / pf.nz) % pf.ny, x = g / (pf.ny * pf.nz);
  const int n[3] = {pf.nx, pf.ny, pf.nz};
  const int pos[3] = {x, y, z};
  double sum = 0.0;
  for (int k = -radius; k <= radius; ++k) {
    const int idx = pos[dir] + k;
    if (idx >= 0 && idx < n[dir]) {
      int q[3] = {x, y, z};
      q[dir] = idx;
      sum += src[3 * (q[0] * pf.ny * pf.nz + q[1] * pf.nz + q[2]) + comp] * kern[k + radius];
    }
  }
  dst[3 * g + comp] = sum;
}

// PredField::getDisp (PredField.cpp:94-150): trilinear interpolation of the field
// (myMATH::triLinearInterp).
__device__ void pf_disp(const PfView& pf, const double* field, const double P[3], double out[3]) {
  const int n[3] = {pf.nx, pf.ny, pf.nz};
  double t[3];
  int id[3];
  for (int k = 0; k < 3; ++k) {
    double p = P[k] < pf.lo[k] ? pf.lo[k] : P[k];  // std::min(std::max(p, lo), hi)
    p = pf.hi[k] < p ? pf.hi[k] : p;
    int i = (int)floor((p - pf.lo[k]) / pf.d[k]);
    i = i < 0 ? 0 : i;
    i = i > n[k] - 2 ? n[k] - 2 : i;
    id[k] = i;
    const double lo = pf.lo[k] + pf.d[k] * i;
    const double hi = pf.lo[k] + pf.d[k] * (i + 1);
    const double v = (p - lo) / (hi - lo);
    t[k] = fmax(0.0, fmin(1.0, v));
  }
  const int nyz = pf.ny * pf.nz;
  const int x0 = id[0], y0 = id[1], z0 = id[2];
  const int g[8] = {x0 * nyz + y0 * pf.nz + z0,
                    (x0 + 1) * nyz + y0 * pf.nz + z0,
                    (x0 + 1) * nyz + y0 * pf.nz + z0 + 1,
                    x0 * nyz + y0 * pf.nz + z0 + 1,
                    x0 * nyz + (y0 + 1) * pf.nz + z0,
                    (x0 + 1) * nyz + (y0 + 1) * pf.nz + z0,
                    (x0 + 1) * nyz + (y0 + 1) * pf.nz + z0 + 1,
                    x0 * nyz + (y0 + 1) * pf.nz + z0 + 1};
  for (int c = 0; c < 3; ++c) {
    double v[8];
    for (int k = 0; k < 8; ++k) v[k] = field[3 * g[k] + c];
    out[c] = otf_lerp8(v, t[0], t[1], t[2]);
  }
}

// Initial-phase link queries: last point + the field's displacement there.
__global__ void pf_query_kernel(PfView pf, const double* field, const double* last, int n,
                                double* q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = last + 3 * (int64_t)i;
  double d[3];
  pf_disp(pf, field, p, d);
  q[3 * i] = p[0] + d[0];
  q[3 * i + 1] = p[1] + d[1];
  q[3 * i + 2] = p[2] + d[2];
}

__global__ void init_pred_kernel(uint8_t* flags, double* score, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flags[i] = 0;
  score[i] = 1.0;
}

// Camera::project of points on every camera (the 2D columns of the track files).
__global__ void project_all_kernel(const CamDev* cams, int n_cam, const double* xyz, int64_t n,
                                   double* uv) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < n_cam; ++c) {
    double x, y;
    cam_project(cams[c], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], x, y);
    uv[(i * n_cam + c) * 2] = x;
    uv[(i * n_cam + c) * 2 + 1] = y;
  }
}

}  // namespace

// ======================================================================== host
namespace {

template <class T>
T* upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s) {
  b.ensure((v.size() + 1) * sizeof(T), s);
  if (!v.empty())
    OLPT_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return b.as<T>();
}

template <class T>
std::vector<T> download(const T* p, size_t n, cudaStream_t s) {
  std::vector<T> v(n);
  if (n) OLPT_CUDA(cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  return v;
}

HashGrid build_grid(Csr& csr, DevBuf& keys, const double* d_pts, int n, double radius,
                    cudaStream_t s) {
  HashGrid g;
  g.cell = std::max(radius, 1e-9) * kCellMargin;
  g.n_buckets = std::max(1024, 2 * n);
  keys.ensure((n + 1) * sizeof(int), s);
  if (n > 0)
    hash_keys_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(d_pts, n, g.cell, g.n_buckets, keys.as<int>());
  csr.build(keys.as<int>(), n, g.n_buckets, s);
  OLPT_CUDA(cudaGetLastError());
  g.start = csr.start.as<int>();
  g.items = csr.items.as<int>();
  g.pts = n > 0 ? d_pts : nullptr;
  return g;
}

PfView pf_view(const StbParams& p) {
  PfView pf{};
  pf.nx = p.pf_n[0];
  pf.ny = p.pf_n[1];
  pf.nz = p.pf_n[2];
  const int n[3] = {pf.nx, pf.ny, pf.nz};
  for (int k = 0; k < 3; ++k) {
    pf.lo[k] = p.limit[2 * k];
    pf.hi[k] = p.limit[2 * k + 1];
    pf.d[k] = (pf.hi[k] - pf.lo[k]) / (n[k] - 1);
    pf.nbin[k] = p.pf_nbin[k];
    pf.m[k] = (pf.nbin[k] - 1) / (4 * p.pf_r);
    pf.c[k] = (double)((pf.nbin[k] - 1) / 2);
  }
  pf.nbin_tot = pf.nbin[0] * pf.nbin[1] * pf.nbin[2];
  pf.r = p.pf_r;
  return pf;
}

// myMATH::createGaussianKernel (myMATH.cpp:537-557)
std::vector<double> gaussian_kernel(int radius, double sigma) {
  const int size = 2 * radius + 1;
  std::vector<double> k(size);
  double sum = 0.0;
  for (int i = 0; i < size; ++i) {
    const int x = i - radius;
    k[i] = std::exp(-(x * x) / (2 * sigma * sigma));
    sum += k[i];
  }
  for (int i = 0; i < size; ++i) k[i] /= sum;
  return k;
}

// myMATH::inverse with the "gauss" method (myMATH.h:182-255, 357-377): Gauss
// elimination with scaled partial pivoting on the row order, then forward and
// back substitution of every identity column.  a, out: n x n row-major.
void gauss_inverse_host(const double* a, int n, double* out) {
  std::vector<double> u(a, a + n * n), b(n * n, 0.0), maxrow(n);
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) {
    idx[i] = i;
    maxrow[i] = *std::max_element(u.begin() + i * n, u.begin() + (i + 1) * n);
    b[i * n + i] = 1.0;
  }
  for (int y = 0; y < n - 1; ++y) {
    double max_pivot = 0;
    int t = 0;
    for (int x = y; x < n; ++x) {
      const double pivot = std::fabs(u[idx[x] * n + y] / maxrow[idx[x]]);
      if (pivot > max_pivot) {
        max_pivot = pivot;
        t = x;
      }
    }
    std::swap(idx[t], idx[y]);
    for (int x = y + 1; x < n; ++x) {
      const double m = u[idx[x] * n + y] / u[idx[y] * n + y];
      u[idx[x] * n + y] = m;
      for (int it = y + 1; it < n; ++it) u[idx[x] * n + it] -= m * u[idx[y] * n + it];
    }
  }
  std::vector<double> res(b);
  for (int it = 0; it < n; ++it) {
    for (int y = 0; y < n - 1; ++y)
      for (int x = y + 1; x < n; ++x) b[idx[x] * n + it] -= u[idx[x] * n + y] * b[idx[y] * n + it];
    res[(n - 1) * n + it] = b[idx[n - 1] * n + it] / u[idx[n - 1] * n + n - 1];
    for (int x = n - 2; x > -1; --x) {
      double z = b[idx[x] * n + it];
      for (int y = x + 1; y < n; ++y) z -= u[idx[x] * n + y] * res[y * n + it];
      res[x * n + it] = z / u[idx[x] * n + x];
    }
  }
  std::copy(res.begin(), res.end(), out);
}

// The 2 x n_pts matrix inverse(X^T X) X^T of STB::checkLinearFit, X = [1, i]
// (Matrix::operator* accumulates from 0 in index order).
std::vector<double> linfit_matrix(int n_pts) {
  double A[4];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 2; ++c) {
      double acc = 0.0;
      for (int i = 0; i < n_pts; ++i) {
        const double xr = r == 0 ? 1.0 : (double)i, xc = c == 0 ? 1.0 : (double)i;
        acc += xr * xc;
      }
      A[2 * r + c] = acc;
    }
  double inv[4];
  gauss_inverse_host(A, 2, inv);
  std::vector<double> k(2 * n_pts);
  for (int r = 0; r < 2; ++r)
    for (int j = 0; j < n_pts; ++j) {
      double acc = 0.0;
      acc += inv[2 * r] * 1.0;
      acc += inv[2 * r + 1] * (double)j;
      k[r * n_pts + j] = acc;
    }
  return k;
}

// The last k points of a track, packed.
void last_points(const TrackH& tr, int k, double* dst) {
  std::copy(tr.xyz.end() - 3 * k, tr.xyz.end(), dst);
}

// The frame loop's temporary track lists reuse the capacity of earlier frames' lists:
// a list of 10^5 tracks is tens of MB, and an allocation that size is fresh pages (and
// their faults) on every frame.
TrackList take_list(TrackList& spare, size_t n) {
  TrackList t;
  t.swap(spare);
  t.clear();
  t.reserve(n);
  return t;
}

void give_list(TrackList& spare, TrackList& t) {
  t.clear();
  if (t.capacity() > spare.capacity()) spare.swap(t);
}

// Copy of the current images: what STB::processFrame leaves in img_list (the input
// in the initial phase, the residual of the shaken predictions in the convergence
// phase; the IPR works on its own copy).
void snapshot_images(olpt_ctx* ctx) {
  for (int c = 0; c < ctx->n_cam; ++c) {
    const ImagePlane& src = ctx->img[c];
    ImagePlane& dst = ctx->stb.frame_img[c];
    const size_t bytes = (size_t)src.pitch * src.H;
    dst.buf.ensure(bytes + 16, ctx->stream);
    dst.dtype = src.dtype;
    dst.H = src.H;
    dst.W = src.W;
    dst.pitch = src.pitch;
    if (bytes)
      OLPT_CUDA(cudaMemcpyAsync(dst.buf.p, src.buf.p, bytes, cudaMemcpyDeviceToDevice,
                                ctx->stream));
  }
}

// IPR::runIPR on the current images; the objects come back to the host.
std::vector<double> run_ipr_host(olpt_ctx* ctx) {
  ipr_device(ctx, ctx->stb.ipr);
  return download(ctx->ipr.out_xyz.as<double>(), (size_t)ctx->ipr.n_out * 3, ctx->stream);
}

// STB::saveTracks (STB.cpp:967-1004) + Track::saveTrack + Tracer3D::saveObject3D
// (ObjectInfo.cpp:76-94).  The 2D columns are each point's projection on every
// camera: the reference's objects always hold projectObject2D of their centre
// (end of Shake::shakeOneObject, buildTrackFromPredField, loadTrack).  The points go
// to the device in passes of at most kMaxRowsPerPass rows, are projected and
// formatted there (trackio.cu), and the file is written by the context's writer.
void save_tracks_file(olpt_ctx* ctx, const TrackList& tracks, const std::string& file) {
  const int C = ctx->n_cam;
  std::string o = "TrackID,FrameID,WorldX,WorldY,WorldZ";
  for (int i = 0; i < C; ++i)
    o += ",cam" + std::to_string(i) + "_x(col),cam" + std::to_string(i) + "_y(row)";
  o += "\n";
  cudaStream_t s = ctx->stream;
  TrackIoWork& W = ctx->tio;
  std::vector<int> ids;
  std::vector<double> xyz;
  size_t tr_i = 0, pt_k = 0;  // next point to pack: track tr_i, its point pt_k
  for (;;) {
    ids.clear();
    xyz.clear();
    while (tr_i < tracks.size() && (int64_t)ids.size() < 2 * kMaxRowsPerPass) {
      const TrackH& tr = tracks[tr_i];
      if (pt_k >= tr.size()) {
        ++tr_i;
        pt_k = 0;
        continue;
      }
      ids.push_back((int)tr_i);  // static_cast<int>(i) of the list index
      ids.push_back(tr.t[pt_k]);
      xyz.insert(xyz.end(), tr.xyz.begin() + 3 * pt_k, tr.xyz.begin() + 3 * pt_k + 3);
      ++pt_k;
    }
    const int64_t n = (int64_t)ids.size() / 2;
    if (n == 0) break;
    const int* d_ids = upload(W.ints, ids, s);
    const double* d_x = upload(W.xyz, xyz, s);
    W.uv.ensure((size_t)(n * C * 2 + 1) * sizeof(double), s);
    project_all_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(ctx->cams_d.as<CamDev>(), C, d_x, n,
                                                      W.uv.as<double>());
    OLPT_CUDA(cudaGetLastError());
    format_rows_device(ctx, d_ids, 2, d_x, 3, W.uv.as<double>(), 2 * C, n, o);
  }
  write_file(ctx, file, std::move(o));
}

// STB::saveTracksAll (STB.cpp:926-965).
void save_tracks_all(olpt_ctx* ctx, const std::string& folder, int frame) {
  namespace fs = std::filesystem;
  StbState& S = ctx->stb;
  const fs::path dir(folder);
  const std::string s = std::to_string(frame);
  // the reference's saveTracks fails on a folder it cannot write into; here before
  // anything is queued
  OLPT_REQUIRE(fs::is_directory(dir), OLPT_ERR_INVALID_ARG,
               "Cannot open file: " + (dir / ("LongTrackActive_" + s + ".csv")).string());
  // runs on the writer thread, after the files posted before it
  auto remove_with_prefix = [dir](const std::string& prefix) {
    if (!fs::exists(dir)) return;
    for (const auto& e : fs::directory_iterator(dir)) {
      if (!e.is_regular_file()) continue;
      const std::string name = e.path().filename().string();
      if (name.size() >= prefix.size() + 4 && name.compare(0, prefix.size(), prefix) == 0 &&
          name.rfind(".csv") == name.size() - 4) {
        std::error_code ec;
        fs::remove(e.path(), ec);
      }
    }
  };
  ctx->tio.writer.post([remove_with_prefix] {
    remove_with_prefix("LongTrackActive_");
    remove_with_prefix("ShortTrackActive_");
  });
  save_tracks_file(ctx, S.long_active, (dir / ("LongTrackActive_" + s + ".csv")).string());
  save_tracks_file(ctx, S.short_active, (dir / ("ShortTrackActive_" + s + ".csv")).string());
  save_tracks_file(ctx, S.exited, (dir / ("ExitTrack_" + s + ".csv")).string());
  save_tracks_file(ctx, S.long_inactive, (dir / ("LongTrackInactive_" + s + ".csv")).string());
}

// PredField::saveDispField -> Matrix::write (src/srcMath/Matrix.hpp:266-279):
// scientific with SAVEPRECISION (8) digits, comma separated, one node per row.
void save_pred_field(const std::vector<double>& f, const std::string& file) {
  std::FILE* fp = std::fopen(file.c_str(), "w");
  OLPT_REQUIRE(fp, OLPT_ERR_INVALID_ARG, "Cannot open file: " + file);
  std::string o;
  char b[64];
  for (size_t g = 0; g < f.size() / 3; ++g)
    for (int c = 0; c < 3; ++c) {
      const int n = std::snprintf(b, sizeof b, c < 2 ? "%.8e," : "%.8e\n", f[3 * g + c]);
      o.append(b, n);
    }
  std::fwrite(o.data(), 1, o.size(), fp);
  std::fclose(fp);
}

// PredField::calPredField between the initial frames i-1 and i; the (smoothed)
// field stays in W.field.
const double* cal_pred_field(olpt_ctx* ctx, int i) {
  StbState& S = ctx->stb;
  StbWork& W = S.w;
  cudaStream_t s = ctx->stream;
  const PfView pf = pf_view(S.p);
  const int n_grid = pf.nx * pf.ny * pf.nz;
  const double* d_prev = upload(W.a, S.ipr_xyz[i - 1], s);
  const double* d_curr = upload(W.c, S.ipr_xyz[i], s);
  const int np = (int)(S.ipr_xyz[i - 1].size() / 3), nc = (int)(S.ipr_xyz[i].size() / 3);
  HashGrid gp = build_grid(W.g1, W.k1, d_prev, np, pf.r, s);
  HashGrid gc = build_grid(W.g2, W.k2, d_curr, nc, pf.r, s);
  W.field.ensure((3 * (size_t)n_grid + 1) * sizeof(double), s);
  W.field2.ensure((3 * (size_t)n_grid + 1) * sizeof(double), s);
  W.flag.ensure(sizeof(int), s);
  OLPT_CUDA(cudaMemsetAsync(W.flag.p, 0, sizeof(int), s));
  const size_t smem = pf.nbin_tot * sizeof(double) + 2 * kPfMaxNb * sizeof(int);
  OLPT_REQUIRE(smem <= 200 * 1024, OLPT_ERR_UNSUPPORTED, "predictive field: too many PDF bins");
  OLPT_CUDA(cudaFuncSetAttribute(pf_node_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  const int pid = ctx->prof.begin(PROF_PF, s);
  pf_node_kernel<<<OLPT_G(n_grid), 256, smem, s>>>(pf, gp, gc, W.field.as<double>(),
                                                   W.flag.as<int>());
  ctx->prof.end(PROF_PF, pid, s, (double)(np + nc) * 24.0 + n_grid * 24.0);
  OLPT_CUDA(cudaGetLastError());
  const int ovf = download(W.flag.as<int>(), 1, s)[0];
  OLPT_REQUIRE(!ovf, OLPT_ERR_UNSUPPORTED,
               "predictive field: more than 4096 objects inside one search cube");
  double* A = W.field.as<double>();
  if (S.p.pf_smooth) {
    // PredField::smoothDispField (PredField.cpp:455-470): component c convolved
    // along x, y and z with the kernel of sigma[c]
    double* B = W.field2.as<double>();
    for (int comp = 0; comp < 3; ++comp) {
      const int radius = (int)std::round(3 * S.p.pf_sigma[comp]);
      const std::vector<double> kern = gaussian_kernel(radius, S.p.pf_sigma[comp]);
      const double* d_k = upload(W.kern, kern, s);
      for (int dir = 0; dir < 3; ++dir) {
        OLPT_CUDA(cudaMemcpyAsync(B, A, 3 * (size_t)n_grid * sizeof(double),
                                  cudaMemcpyDeviceToDevice, s));
        pf_smooth_kernel<<<OLPT_G(nblk(n_grid)), 256, 0, s>>>(pf, B, A, comp, dir, d_k, radius);
      }
      OLPT_CUDA(cudaStreamSynchronize(s));  // the kernel buffer is rewritten next
    }
    OLPT_CUDA(cudaGetLastError());
  }
  if (!S.p.output_path.empty()) {
    const int fid = i + S.p.frame_start;  // named as in runInitPhase (STB.cpp:121-123)
    save_pred_field(download(A, 3 * (size_t)n_grid, s),
                    S.p.output_path + "PredField_" + std::to_string(fid) + "_" +
                        std::to_string(fid + 1) + ".csv");
  }
  return A;
}

// STB::buildTrackFromPredField (STB.cpp:160-231).
void build_from_pf(olpt_ctx* ctx, int idx, const double* d_field, int frame) {
  StbState& S = ctx->stb;
  StbWork& W = S.w;
  cudaStream_t s = ctx->stream;
  const std::vector<double>& objs = S.ipr_xyz[idx];
  std::vector<char>& tracked = S.ipr_tracked[idx];
  const int n_obj = (int)(objs.size() / 3);
  if (idx > 0) {
    const int n_sa = (int)S.short_active.size();
    std::vector<int> link(n_sa, -1);
    if (n_sa > 0 && n_obj > 0) {
      std::vector<double> last(3 * (size_t)n_sa);
      for (int j = 0; j < n_sa; ++j) last_points(S.short_active[j], 1, &last[3 * j]);
      const double* d_last = upload(W.d, last, s);
      W.b.ensure((3 * (size_t)n_sa + 1) * sizeof(double), s);
      pf_query_kernel<<<OLPT_G(nblk(n_sa)), 256, 0, s>>>(pf_view(S.p), d_field, d_last, n_sa,
                                                        W.b.as<double>());
      const double* d_obj = upload(W.c, objs, s);
      const double r = S.p.radius_search_obj;
      HashGrid go = build_grid(W.g1, W.k1, d_obj, n_obj, r, s);
      W.link.ensure((n_sa + 1) * sizeof(int), s);
      nn_kernel<<<OLPT_G(nblk(n_sa)), 256, 0, s>>>(W.b.as<double>(), n_sa, go, r * r,
                                                  W.link.as<int>());
      OLPT_CUDA(cudaGetLastError());
      link = download(W.link.as<int>(), n_sa, s);
    }
    TrackList kept;
    for (int j = 0; j < n_sa; ++j) {
      if (link[j] < 0) continue;
      tracked[link[j]] = 1;
      TrackH& tr = S.short_active[j];
      tr.xyz.insert(tr.xyz.end(), &objs[3 * link[j]], &objs[3 * link[j]] + 3);
      tr.t.push_back(frame);
      kept.push_back(std::move(tr));
    }
    S.short_active.swap(kept);
  }
  for (int i = 0; i < n_obj; ++i) {
    if (tracked[i]) continue;
    tracked[i] = 1;
    TrackH tr;
    tr.xyz.assign(&objs[3 * i], &objs[3 * i] + 3);
    tr.t.push_back(frame);
    S.short_active.push_back(std::move(tr));
  }
}

// STB::runInitPhase (STB.cpp:91-158)
void init_phase(olpt_ctx* ctx, int frame) {
  StbState& S = ctx->stb;
  snapshot_images(ctx);
  std::vector<double> xyz = run_ipr_host(ctx);
  PhaseTimer pt(ctx->prof, PH_TRACK);
  S.ipr_tracked.emplace_back(xyz.size() / 3, 0);
  S.ipr_xyz.push_back(std::move(xyz));
  S.last_xyz = S.ipr_xyz.back();
  S.last_new = (int64_t)(S.ipr_xyz.back().size() / 3);
  S.last_extended = 0;
  if (frame - S.p.frame_start != S.p.n_initial_frames - 1) return;
  for (int i = 0; i < S.p.n_initial_frames; ++i) {
    const int fid = i + S.p.frame_start;
    build_from_pf(ctx, i, i == 0 ? nullptr : cal_pred_field(ctx, i), fid);
  }
  const size_t need = (size_t)S.p.n_initial_frames;
  TrackList still_short;
  for (TrackH& tr : S.short_active) {
    if (tr.size() >= need)
      S.long_active.push_back(std::move(tr));
    else
      still_short.push_back(std::move(tr));
  }
  S.short_active.swap(still_short);
  if (!S.p.output_path.empty()) save_tracks_all(ctx, S.p.output_path + "InitialTrack/", frame);
}

// STB::runConvPhase (STB.cpp:337-696; without the volume self-calibration).
void conv_phase(olpt_ctx* ctx, int frame) {
  StbState& S = ctx->stb;
  StbWork& W = S.w;
  cudaStream_t s = ctx->stream;
  const int C = ctx->n_cam;
  auto t_track = std::chrono::steady_clock::now();
  double track_ms = 0.0;
  auto pause = [&] {
    track_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_track)
                    .count();
  };
  auto resume = [&] { t_track = std::chrono::steady_clock::now(); };
  // the parts of the track work (the shake and the IPR excluded)
  auto t_part = std::chrono::steady_clock::now();
  auto part = [&](int ph) {
    const auto now = std::chrono::steady_clock::now();
    ctx->prof.add_phase(ph, std::chrono::duration<double, std::milli>(now - t_part).count());
    t_part = now;
  };

  // 1. prediction of the active long tracks
  int n_la = (int)S.long_active.size();
  std::vector<double> pred;
  if (n_la > 0) {
    std::vector<double> pts((size_t)n_la * 18, 0.0);
    std::vector<int> np(n_la);
    for (int i = 0; i < n_la; ++i) {
      const TrackH& tr = S.long_active[i];
      OLPT_REQUIRE(tr.size() >= 3, OLPT_ERR_UNSUPPORTED,
                   "active long track with fewer than 3 points (the reference dereferences "
                   "a null prediction)");
      np[i] = (int)std::min<size_t>(tr.size(), 6);
      last_points(tr, np[i], &pts[(size_t)18 * i]);
    }
    StbView v{};
    v.n_cam = C;
    v.cams = ctx->cams_d.as<CamDev>();
    for (int q = 0; q < 6; ++q) v.limit[q] = S.p.limit[q];
    const double* d_pts = upload(W.a, pts, s);
    const int* d_np = upload(W.ia, np, s);
    W.b.ensure((3 * (size_t)n_la + 1) * sizeof(double), s);
    W.link.ensure((n_la + 1) * sizeof(int), s);
    predict_kernel<<<OLPT_G(nblk(n_la, 128)), 128, 0, s>>>(d_pts, d_np, n_la, v, W.b.as<double>(),
                                                          W.link.as<int>());
    OLPT_CUDA(cudaGetLastError());
    pred = download(W.b.as<double>(), 3 * (size_t)n_la, s);
    const std::vector<int> in_range = download(W.link.as<int>(), n_la, s);
    TrackList kept = take_list(S.spare_long, n_la);
    size_t w = 0;
    for (int i = 0; i < n_la; ++i) {
      if (!in_range[i]) {
        if (S.long_active[i].size() >= (size_t)kLenLongTrack)
          S.exited.push_back(std::move(S.long_active[i]));
      } else {
        kept.push_back(std::move(S.long_active[i]));
        std::copy(&pred[3 * i], &pred[3 * i] + 3, &pred[3 * w]);
        ++w;
      }
    }
    S.long_active.swap(kept);
    give_list(S.spare_long, kept);
    n_la = (int)w;
    pred.resize(3 * w);
  }

  part(PH_TR_PREDICT);
  // 2. shake the predictions; residual without the ghost / repeated ones; extend
  int64_t extended = 0;
  S.last_xyz.clear();
  if (n_la > 0) {
    ctx->obj.ensure(n_la, C, s);
    ctx->obj.n = n_la;
    OLPT_CUDA(cudaMemcpyAsync(ctx->obj.xyz.p, pred.data(), pred.size() * sizeof(double),
                              cudaMemcpyHostToDevice, s));
    init_pred_kernel<<<OLPT_G(nblk(n_la)), 256, 0, s>>>(ctx->obj.flags.as<uint8_t>(),
                                                       ctx->obj.score.as<double>(), n_la);
    // with the learned proposal configured, the predictions go through the learned
    // shake, which drops the network's ghosts (they end like ghost-flagged tracks)
    const bool learned = ctx->mlp.lp.enable != 0;
    pause();
    part(PH_TR_EXTEND);
    if (learned)
      learned_shake_device(ctx, S.ipr.shake);
    else
      shake_device(ctx, S.ipr.shake);
    residual_device(ctx, S.ipr.shake, true, true);
    resume();
    t_part = std::chrono::steady_clock::now();
    const int64_t n_out = ctx->obj.n;
    const std::vector<double> sx0 = download(ctx->obj.xyz.as<double>(), 3 * (size_t)n_out, s);
    const std::vector<uint8_t> fl0 = download(ctx->obj.flags.as<uint8_t>(), (size_t)n_out, s);
    std::vector<double> sx(3 * (size_t)n_la, 0.0);
    std::vector<uint8_t> fl(n_la, 1);
    if (learned) {
      const std::vector<int> keep = download(ctx->mlp.keep.as<int>(), n_la, s);
      int64_t j = 0;
      for (int i = 0; i < n_la; ++i)
        if (keep[i] && j < n_out) {
          std::copy(&sx0[3 * j], &sx0[3 * j] + 3, &sx[3 * i]);
          fl[i] = fl0[j++];
        }
    } else {
      sx = sx0;
      fl = fl0;
    }
    TrackList kept = take_list(S.spare_long, n_la);
    for (int i = 0; i < n_la; ++i) {
      TrackH& tr = S.long_active[i];
      if (fl[i] == 0) {
        S.last_xyz.insert(S.last_xyz.end(), &sx[3 * i], &sx[3 * i] + 3);
        tr.xyz.insert(tr.xyz.end(), &sx[3 * i], &sx[3 * i] + 3);
        tr.t.push_back(frame);
        kept.push_back(std::move(tr));
        ++extended;
      } else if (tr.size() >= (size_t)kLenLongTrack) {
        S.long_inactive.push_back(std::move(tr));
      }
    }
    S.long_active.swap(kept);
    give_list(S.spare_long, kept);
    n_la = (int)S.long_active.size();
  }

  // 3. IPR on the residual images
  snapshot_images(ctx);
  pause();
  part(PH_TR_EXTEND);
  std::vector<double> oxyz = run_ipr_host(ctx);
  resume();
  t_part = std::chrono::steady_clock::now();
  int n_obj = (int)(oxyz.size() / 3);

  // 4. drop the objects close to an active long track's last point
  if (n_obj > 0 && n_la > 0) {
    std::vector<double> lastp(3 * (size_t)n_la);
    for (int i = 0; i < n_la; ++i) last_points(S.long_active[i], 1, &lastp[3 * i]);
    const double tol = S.ipr.sm.tol_3d_mm;
    const double* d_last = upload(W.a, lastp, s);
    HashGrid g = build_grid(W.g1, W.k1, d_last, n_la, tol, s);
    const double* d_obj = upload(W.c, oxyz, s);
    W.link.ensure((n_obj + 1) * sizeof(int), s);
    repeat_kernel<<<OLPT_G(nblk(n_obj)), 256, 0, s>>>(d_obj, n_obj, g, tol, W.link.as<int>());
    OLPT_CUDA(cudaGetLastError());
    const std::vector<int> rep = download(W.link.as<int>(), n_obj, s);
    size_t w = 0;
    for (int i = 0; i < n_obj; ++i)
      if (!rep[i]) {
        std::copy(&oxyz[3 * i], &oxyz[3 * i] + 3, &oxyz[3 * w]);
        ++w;
      }
    oxyz.resize(3 * w);
    n_obj = (int)w;
  }

  // 5. link the active short tracks to the new objects
  if (n_obj > 0) {
    const int n_sa = (int)S.short_active.size();
    std::vector<int> link(n_sa, -1);
    if (n_sa > 0) {
      std::vector<double> plast(3 * (size_t)n_sa, 0.0);
      std::vector<int> slen(n_sa);
      for (int i = 0; i < n_sa; ++i) {
        slen[i] = (int)S.short_active[i].size();
        if (slen[i] > 0) last_points(S.short_active[i], 1, &plast[3 * i]);
      }
      std::vector<double> key(3 * (size_t)n_la), disp(3 * (size_t)n_la);
      for (int j = 0; j < n_la; ++j) {
        const TrackH& tr = S.long_active[j];
        const size_t L = tr.size();
        const double* a = &tr.xyz[3 * (L - 1)];
        const double* b = &tr.xyz[3 * (L - 2)];
        for (int d = 0; d < 3; ++d) {
          key[3 * j + d] = (double)(float)b[d];
          disp[3 * j + d] = a[d] - b[d];
        }
      }
      const double base_r = S.p.radius_search_track;
      const double r_max = base_r * 1.1 * 1.1 * 1.1 * 1.1;
      const double* d_key = upload(W.a, key, s);
      const double* d_disp = upload(W.b, disp, s);
      const double* d_pl = upload(W.d, plast, s);
      const int* d_len = upload(W.ia, slen, s);
      const double* d_obj = upload(W.c, oxyz, s);
      HashGrid tg = build_grid(W.g1, W.k1, d_key, n_la, 3.0 * r_max, s);
      HashGrid go = build_grid(W.g2, W.k2, d_obj, n_obj, r_max, s);
      W.link.ensure((n_sa + 1) * sizeof(int), s);
      link_kernel<<<OLPT_G(nblk(n_sa, 128)), 128, 0, s>>>(d_pl, d_len, n_sa, tg, d_disp, go, base_r,
                                                         W.link.as<int>());
      OLPT_CUDA(cudaGetLastError());
      link = download(W.link.as<int>(), n_sa, s);
    }
    // first come, first served
    std::vector<int> owner(n_obj, -1);
    for (int j = 0; j < n_sa; ++j) {
      const int lid = link[j];
      if (lid < 0 || lid >= n_obj) continue;
      if (owner[lid] == -1)
        owner[lid] = j;
      else
        link[j] = -1;
    }
    std::vector<char> used(n_obj, 0);
    TrackList keep = take_list(S.spare_short, (size_t)n_sa + n_obj);
    for (int i = 0; i < n_sa; ++i) {
      const int lid = link[i];
      if (lid < 0 || lid >= n_obj) continue;
      used[lid] = 1;
      TrackH& tr = S.short_active[i];
      tr.xyz.insert(tr.xyz.end(), &oxyz[3 * lid], &oxyz[3 * lid] + 3);
      tr.t.push_back(frame);
      if ((int)tr.size() >= S.p.n_initial_frames)
        S.long_active.push_back(std::move(tr));
      else
        keep.push_back(std::move(tr));
    }
    S.short_active.swap(keep);
    give_list(S.spare_short, keep);
    S.short_active.reserve(S.short_active.size() + n_obj);
    for (int i = 0; i < n_obj; ++i) {
      if (used[i]) continue;
      TrackH tr;
      tr.xyz.assign(&oxyz[3 * i], &oxyz[3 * i] + 3);
      tr.t.push_back(frame);
      S.short_active.push_back(std::move(tr));
    }
  }

  part(PH_TR_LINK);
  // 6. linear-fit pruning of the active long tracks
  n_la = (int)S.long_active.size();
  if (n_la > 0) {
    const int n_pts = S.p.n_initial_frames > 4 ? 4 : S.p.n_initial_frames;
    std::vector<double> pts((size_t)n_la * 12, 0.0);
    std::vector<int> len(n_la);
    for (int i = 0; i < n_la; ++i) {
      const TrackH& tr = S.long_active[i];
      len[i] = (int)tr.size();
      if (len[i] >= n_pts) last_points(tr, n_pts, &pts[(size_t)12 * i]);
    }
    const double* d_pts = upload(W.a, pts, s);
    const int* d_len = upload(W.ia, len, s);
    const double* d_k = upload(W.kern, S.linfit_kernel, s);
    W.link.ensure((n_la + 1) * sizeof(int), s);
    linfit_kernel<<<OLPT_G(nblk(n_la)), 256, 0, s>>>(d_pts, d_len, n_la, n_pts, d_k,
                                                    W.link.as<int>());
    OLPT_CUDA(cudaGetLastError());
    const std::vector<int> ok = download(W.link.as<int>(), n_la, s);
    TrackList kept = take_list(S.spare_long, n_la);
    for (int i = 0; i < n_la; ++i) {
      TrackH& tr = S.long_active[i];
      if (ok[i])
        kept.push_back(std::move(tr));
      else if (tr.size() >= (size_t)kLenLongTrack)
        S.long_inactive.push_back(std::move(tr));
    }
    S.long_active.swap(kept);
    give_list(S.spare_long, kept);
  }
  S.last_extended = extended;
  S.last_new = n_obj;
  S.last_xyz.insert(S.last_xyz.end(), oxyz.begin(), oxyz.end());

  // every 500 frames the reference writes all tracks and forgets the inactive and
  // exited ones
  if (frame % 500 == 0) {
    if (!S.p.output_path.empty()) save_tracks_all(ctx, S.p.output_path + "ConvergeTrack/", frame);
    S.long_inactive.clear();
    S.exited.clear();
  }
  pause();
  part(PH_TR_PRUNE);
  ctx->prof.add_phase(PH_TRACK, track_ms);
}

}  // namespace

void stb_configure(olpt_ctx* ctx, const StbParams& p, const IprParams& ipr) {
  OLPT_REQUIRE(p.frame_end >= p.frame_start, OLPT_ERR_INVALID_ARG, "frame_end < frame_start");
  OLPT_REQUIRE(p.n_initial_frames >= 4, OLPT_ERR_INVALID_ARG,
               "n_initial_frames must be >= 4 (the reference's config reader enforces it)");
  for (int k = 0; k < 3; ++k) {
    OLPT_REQUIRE(p.pf_n[k] >= 2, OLPT_ERR_INVALID_ARG, "predictive-field grid needs >= 2 nodes");
    OLPT_REQUIRE(p.pf_nbin[k] >= 2, OLPT_ERR_INVALID_ARG, "predictive-field PDF needs >= 2 bins");
    OLPT_REQUIRE(p.pf_sigma[k] > 0, OLPT_ERR_INVALID_ARG, "smoothing sigma must be positive");
  }
  OLPT_REQUIRE(p.pf_r > 0, OLPT_ERR_INVALID_ARG, "predictive-field radius must be positive");
  StbState& S = ctx->stb;
  S.p = p;
  S.ipr = ipr;
  S.short_active.clear();
  S.long_active.clear();
  S.long_inactive.clear();
  S.exited.clear();
  S.ipr_xyz.clear();
  S.ipr_tracked.clear();
  S.last_new = S.last_extended = 0;
  S.linfit_kernel = linfit_matrix(p.n_initial_frames > 4 ? 4 : p.n_initial_frames);
  if (!p.output_path.empty()) {
    std::filesystem::create_directories(p.output_path);
    std::filesystem::create_directories(p.output_path + "InitialTrack/");
    std::filesystem::create_directories(p.output_path + "ConvergeTrack/");
  }
  S.configured = true;
}

// STB::processFrame (STB.cpp:40-89) on the context's current images.  In the
// convergence phase they become the residual of the shaken predictions (the
// reference's img_list), which the IPR then reduces further in place.
void stb_process_frame(olpt_ctx* ctx, int frame) {
  StbState& S = ctx->stb;
  OLPT_REQUIRE(S.configured, OLPT_ERR_INVALID_ARG, "configure the STB first");
  OLPT_REQUIRE(frame >= S.p.frame_start && frame <= S.p.frame_end, OLPT_ERR_INVALID_ARG,
               "Frame number is out of range");
  if (frame - S.p.frame_start < S.p.n_initial_frames)
    init_phase(ctx, frame);
  else
    conv_phase(ctx, frame);
  if (frame == S.p.frame_end && frame % 500 != 0 && !S.p.output_path.empty())
    save_tracks_all(ctx, S.p.output_path + "ConvergeTrack/", frame);
}

TrackList& stb_list(olpt_ctx* ctx, int which) {
  StbState& S = ctx->stb;
  switch (which) {
    case OLPT_TRACK_LONG_ACTIVE: return S.long_active;
    case OLPT_TRACK_SHORT_ACTIVE: return S.short_active;
    case OLPT_TRACK_LONG_INACTIVE: return S.long_inactive;
    case OLPT_TRACK_EXIT: return S.exited;
    default: throw ApiError{OLPT_ERR_INVALID_ARG, "unknown track list"};
  }
}

void stb_save_tracks(olpt_ctx* ctx, int which, const std::string& path) {
  save_tracks_file(ctx, stb_list(ctx, which), path);
}

// STB::loadTracks (STB.cpp:1006-1047) + Track::loadTrack (Track.cpp:30-68): a
// track id creates every slot up to it; X, Y, Z are parsed with std::stod.
void stb_load_tracks(olpt_ctx* ctx, int which, const std::string& path) {
  std::ifstream fin(path);
  OLPT_REQUIRE(fin.is_open(), OLPT_ERR_INVALID_ARG, "LoadTracks: cannot open file: " + path);
  TrackList& tracks = stb_list(ctx, which);
  tracks.clear();
  std::string line;
  std::getline(fin, line);  // header
  while (std::getline(fin, line)) {
    if (line.empty()) continue;
    std::istringstream row(line);
    std::string s_tid, s_fid, sx, sy, sz;
    if (!std::getline(row, s_tid, ',') || !std::getline(row, s_fid, ',')) continue;
    int tid, fid;
    try {
      tid = std::stoi(s_tid);
      fid = std::stoi(s_fid);
    } catch (...) {
      continue;
    }
    OLPT_REQUIRE(std::getline(row, sx, ',') && std::getline(row, sy, ',') &&
                     std::getline(row, sz, ','),
                 OLPT_ERR_INVALID_ARG, "Tracer3D::loadObject3D: insufficient 3D columns");
    OLPT_REQUIRE(tid >= 0, OLPT_ERR_INVALID_ARG, "negative track id");
    while ((int)tracks.size() <= tid) tracks.emplace_back();
    TrackH& tr = tracks[tid];
    tr.xyz.push_back(std::stod(sx));
    tr.xyz.push_back(std::stod(sy));
    tr.xyz.push_back(std::stod(sz));
    tr.t.push_back(fid);
  }
}

}  // namespace olpt
