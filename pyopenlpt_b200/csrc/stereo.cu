// Kernel family (b): stereo matching on the device.
//
// Reference: StereoMatch (src/srcSTB/StereoMatch.cpp): IDMap grid (:1413-1437),
// strip intersection (:1471-1570), point visit (:1572-1627), DFS build (:184-444),
// candidate enumeration (:449-498), back-projection (:1206-1227), quick
// triangulation gate (:1083-1141), camera selection (:1307-1411), check (:504-609).
//
// B200 mapping.
//  * Grid: a counting sort per camera (histogram -> scan -> scatter -> per-cell
//    ascending pid order), i.e. the reference's bucket lists as CSR arrays.
//  * Every detection's line of sight and its image line on every other camera are
//    computed once (same FP64 functions the reference calls on the fly, so the
//    values are bit-identical) and reused by every path that touches the point.
//  * The depth-first search over build cameras is expanded breadth-first: level k
//    holds all partial paths with k chosen cameras and the target camera of their
//    next choice.  One warp expands one path: lanes take rows of cells, replicate the
//    reference's per-row span arithmetic exactly, visit the cells and apply the exact
//    point-line test, back-projection test and quick triangulation gate.  Children
//    are appended with atomics; the final candidate list is sorted by ids on the
//    host, so append order never shows.
//  * The whole set of candidates (ids, e_check) is therefore identical to the
//    reference's.  Decisions that pass through acos/sin (only when the minimum
//    parallax is below 6 degrees) can differ by one ulp; those are the only
//    non-bit-exact inputs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_prune.h"
#include "olpt_scan.cuh"
#include "olpt_stereo.h"

namespace olpt {

struct SmView {
  int n_cam, m, n_active;
  int active[OLPT_MAX_CAM];
  int cell;
  int rows[OLPT_MAX_CAM], cols[OLPT_MAX_CAM];
  double Wd[OLPT_MAX_CAM], Hd[OLPT_MAX_CAM];
  const int* cell_start[OLPT_MAX_CAM];
  const int* cell_items[OLPT_MAX_CAM];
  const double* x[OLPT_MAX_CAM];
  const double* y[OLPT_MAX_CAM];
  int64_t n[OLPT_MAX_CAM];
  const double* los[OLPT_MAX_CAM];                  // n x 6
  const double* l2d[OLPT_MAX_CAM][OLPT_MAX_CAM];    // [c][t]: n[c] x 6 (pt, unit, U)
  // cell-ordered copies of camera t's detections (position q of cell_items[t]):
  // their coordinates, and the first four values of their image lines on camera c
  const double2* cxy[OLPT_MAX_CAM];
  const double* cbp[OLPT_MAX_CAM][OLPT_MAX_CAM];    // [t][c]: n[t] x 4
  double tol2d, tol3d;
  double limit[6];
  // near-tolerance log (off when near_band == 0): 2D tests whose distance lies within
  // near_band px of tol2d are appended to near_rec
  double near_band;
  olpt_near_record* near_rec;
  unsigned long long* near_count;
  long long near_cap;
};

struct Path {
  int ids[OLPT_MAX_CAM];
  signed char cams[OLPT_MAX_CAM];
  int k;
  int target;
};

// A partial path of exactly N chosen points, as the level kernels pass it on: the
// chosen detection ids, their cameras packed 4 bits each (point i in bits 4i..4i+3)
// and the next camera.  16 bytes for N = 2 (the 30 M first-level children of a 2048^2
// frame) instead of the 48 of a full Path.
template <int N>
struct alignas(16) PathN {
  int ids[N];
  unsigned cams;
  int target;
  __host__ __device__ int cam(int i) const { return (int)((cams >> (4 * i)) & 15u); }
};

namespace {

inline int nblk(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------- grid
__global__ void cell_hist_kernel(const double* x, const double* y, int64_t n, int cell, int rows,
                                 int cols, int* cell_of, int* counts) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  // IDMap::rebuild (StereoMatch.cpp:1423-1437)
  int cx = (int)floor(x[i] / (double)cell);
  int cy = (int)floor(y[i] / (double)cell);
  if (cx < 0 || cy < 0 || cx >= cols || cy >= rows) {
    cell_of[i] = -1;
    return;
  }
  int c = cy * cols + cx;
  cell_of[i] = c;
  atomicAdd(&counts[c], 1);
}

__global__ void cell_scatter_kernel(const int* cell_of, int64_t n, const int* start, int* cursor,
                                    int* items) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = cell_of[i];
  if (c < 0) return;
  int pos = start[c] + atomicAdd(&cursor[c], 1);
  items[pos] = (int)i;
}

// ascending pid order inside every cell (the reference pushes pids in order)
__global__ void cell_sort_kernel(const int* start, int n_cells, int* items) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  int b = start[c], e = start[c + 1];
  for (int i = b + 1; i < e; ++i) {
    int v = items[i];
    int j = i - 1;
    while (j >= b && items[j] > v) {
      items[j + 1] = items[j];
      --j;
    }
    items[j + 1] = v;
  }
}

// ---------------------------------------------------------------- per-detection lines
__global__ void lines_kernel(const CamDev* cams, int c, const double* x, const double* y, int64_t n,
                             int n_cam, const int* active, double* los, double* const* l2d) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  Line3 L;
  cam_los(cams[c], x[i], y[i], L);
  for (int k = 0; k < 3; ++k) {
    los[6 * i + k] = L.p[k];
    los[6 * i + 3 + k] = L.u[k];
  }
  for (int t = 0; t < n_cam; ++t) {
    if (t == c || !active[t]) continue;
    double o[4];
    los_to_line2d(cams[t], L, o);
    double* d = l2d[t] + 6 * i;
    d[0] = o[0];
    d[1] = o[1];
    d[2] = o[2];
    d[3] = o[3];
    // IDMap::normalized (StereoMatch.cpp:1441-1451)
    const double n2 = o[2] * o[2] + o[3] * o[3];
    if (n2 <= 1e-24) {
      d[4] = 1.0;
      d[5] = 0.0;
    } else {
      const double inv = 1.0 / sqrt(n2);
      d[4] = o[2] * inv;
      d[5] = o[3] * inv;
    }
  }
}

// Cell-ordered copies of camera t's detections for the enumeration's inner loop:
// coordinates, and for every other active camera c the point and direction of the
// detection's image line on c.
__global__ void cell_pack_kernel(const int* items, int64_t n, const double* x, const double* y,
                                 double2* cxy, double* const* bp_out, const double* const* l2d,
                                 int n_cam, int t) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int pid = items[q];
  cxy[q] = make_double2(x[pid], y[pid]);
  for (int c = 0; c < n_cam; ++c) {
    double* o = bp_out[c];
    if (c == t || !o) continue;
    const double* L = l2d[c] + 6 * (int64_t)pid;
    o[4 * q] = L[0];
    o[4 * q + 1] = L[1];
    o[4 * q + 2] = L[2];
    o[4 * q + 3] = L[3];
  }
}

__device__ __forceinline__ void load_line3(const double* p, Line3& L) {
  L.p[0] = p[0];
  L.p[1] = p[1];
  L.p[2] = p[2];
  L.u[0] = p[3];
  L.u[1] = p[4];
  L.u[2] = p[5];
}

// StereoMatch::selectSecondCameraByLineLength segment length (StereoMatch.cpp:1309-1357)
__device__ double seg_len(const double* L, double W, double H) {
  const double px = L[0], py = L[1], ux = L[2], uy = L[3];
  double qx[4], qy[4];
  int n = 0;
  auto push_if = [&](double a, double b) {
    if (a >= 0.0 && a <= W && b >= 0.0 && b <= H) {
      qx[n] = a;
      qy[n] = b;
      ++n;
    }
  };
  if (fabs(ux) > 1e-12) {
    double t = (0.0 - px) / ux;
    push_if(0.0, py + t * uy);
    t = (W - 1 - px) / ux;
    push_if(W - 1, py + t * uy);
  }
  if (fabs(uy) > 1e-12) {
    double t = (0.0 - py) / uy;
    push_if(px + t * ux, 0.0);
    t = (H - 1 - py) / uy;
    push_if(px + t * ux, H - 1);
  }
  double ux2[4], uy2[4];
  int m = 0;
  for (int i = 0; i < n; ++i) {
    bool dup = false;
    for (int j = 0; j < m; ++j)
      if (fabs(ux2[j] - qx[i]) < 1e-9 && fabs(uy2[j] - qy[i]) < 1e-9) {
        dup = true;
        break;
      }
    if (!dup) {
      ux2[m] = qx[i];
      uy2[m] = qy[i];
      ++m;
    }
  }
  if (m < 2) return 0.0;
  const double dx = ux2[0] - ux2[1], dy = uy2[0] - uy2[1];
  return sqrt(dx * dx + dy * dy);
}

// seed level: one path per reference detection with its second build camera
__global__ void seed_kernel(const __grid_constant__ SmView v, int ref, PathN<1>* out, int* out_count,
                            int cap) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= v.n[ref]) return;
  int best = -1;
  double best_len = __longlong_as_double(0x7ff0000000000000LL);
  for (int cam = 0; cam < v.n_cam; ++cam) {
    if (!v.active[cam] || cam == ref) continue;
    const double L = seg_len(v.l2d[ref][cam] + 6 * i, v.Wd[cam], v.Hd[cam]);
    if (L < best_len - 1e-9) {
      best_len = L;
      best = cam;
    }
  }
  if (best < 0) return;
  int slot = atomicAdd(out_count, 1);
  if (slot >= cap) return;
  PathN<1> p;
  p.ids[0] = (int)i;
  p.cams = (unsigned)ref;
  p.target = best;
  out[slot] = p;
}

// (I - n n^T) of one line of sight, in myMATH::triangulation's element order.
__device__ __forceinline__ void normal_terms(const double u[3], double t[9]) {
  const double nx = u[0], ny = u[1], nz = u[2];
  t[0] = 1 - nx * nx;
  t[1] = -nx * ny;
  t[2] = -nx * nz;
  t[3] = -nx * ny;
  t[4] = 1 - ny * ny;
  t[5] = -ny * nz;
  t[6] = -nx * nz;
  t[7] = -ny * nz;
  t[8] = 1 - nz * nz;
}

// Angle in degrees between two unit directions (StereoMatch.cpp:1077-1083).
__device__ __forceinline__ double pair_deg(const double a[3], const double b[3]) {
  double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  dot = fmax(-1.0, fmin(1.0, dot));
  return acos(dot) * 180.0 / M_PI;
}

// StereoMatch::calTriangulateTol (StereoMatch.cpp:1103-1126) from the min parallax.
__device__ __forceinline__ double quick_tol_from_deg(double min_deg, int k, int m, double tol3d) {
  const int kk = k > 2 ? k : 2;
  const int mm = m > 2 ? m : 2;
  const double alpha_depth = sqrt(double(mm) / double(kk));
  const double th = fmax(min_deg, 1.0);
  const double num = sin(6.0 * M_PI / 180.0);
  const double den = fmax(1e-6, sin(th * M_PI / 180.0));
  const double alpha_angle = fmax(1.0, fmin(2.0, num / den));
  return tol3d * alpha_depth * alpha_angle;
}

// One line's contribution to the triangulation error (myMATH.cpp:396-418);
// false where the reference throws (squared distance below -1e-8).
__device__ __forceinline__ bool line_error_term(const double X[3], const double p[3],
                                                const double u[3], double& e) {
  const double d0 = X[0] - p[0], d1 = X[1] - p[1], d2 = X[2] - p[2];
  const double nrm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  const double dt = d0 * u[0] + d1 * u[1] + d2 * u[2];
  double h = nrm * nrm - dt * dt;
  if (h < 0.0 && h >= -1e-8) {
    h = 0.0;
  } else if (h < -1e-8) {
    return false;
  } else {
    h = sqrt(h);
  }
  e += h * h;
  return true;
}

__device__ __forceinline__ double clamped_dot(const double a[3], const double b[3]) {
  const double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  return fmax(-1.0, fmin(1.0, dot));
}

// cos(6 deg): the quick-gate angle factor of calTriangulateTol is exactly 1 whenever
// the smallest pairwise parallax lies inside (6, 174) degrees.
constexpr double kCos6 = 0.99452189536827329;

// A path and one of its candidates on the target camera that passed the 2D tests.
struct Pair {
  int path;
  int pid;
};

// Slot in an append buffer for every active lane, one atomic per warp.
__device__ __forceinline__ int append_slot(int* counter) {
  const unsigned m = __activemask();
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(m, base, leader);
  return base + __popc(m & ((1u << lane) - 1u));
}

// Appends one near-tolerance 2D decision to the log (rare: only tests whose
// distance is within near_band px of the tolerance).
__device__ __noinline__ void near_append(const SmView& v, int kind, int k, int cam, int id,
                                         int other_cam, int other_id, double margin) {
  const unsigned long long slot = atomicAdd(v.near_count, 1ull);
  if ((long long)slot >= v.near_cap) return;
  olpt_near_record r;
  r.kind = kind;
  r.n_chosen = k;
  r.cam = cam;
  r.id = id;
  r.other_cam = other_cam;
  r.other_id = other_id;
  r.margin_px = margin;
  v.near_rec[slot] = r;
}

// Expand one level, first half: each path has K chosen cameras; its candidates on
// the target camera are enumerated over rows of cells and kept when they pass the
// strip test (IDMap::visitPointsInRowSpans) and the back-projection test.  WARP: one
// warp per path, lanes take rows (the single long strip of K = 1); otherwise one
// thread per path (K >= 2, where the strips intersect in a few rows).
template <int K, bool WARP>
__global__ void __launch_bounds__(256, K == 1 ? 4 : 2) enum_kernel(const __grid_constant__ SmView v, const void* in_v, int n_in,
                                                   Pair* pairs, int* pair_count, int pair_cap) {
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int pidx = WARP ? (gtid >> 5) : gtid;
  const int r0 = WARP ? (threadIdx.x & 31) : 0;
  // thread-per-path levels keep every lane of a warp to the end (the items of the
  // warp's paths are shared out over all lanes); a lane without a path has no rows
  const bool live = pidx < n_in;
  if (WARP && !live) return;
  const PathN<K>* in = static_cast<const PathN<K>*>(in_v);
  PathN<K> P{};
  if (live) P = in[pidx];
  const int t = P.target;
  // image lines of the chosen points on the target camera
  double lp[K][2], lU[K][2];
  double cpt[K][2];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    lp[i][0] = lp[i][1] = lU[i][0] = cpt[i][0] = cpt[i][1] = 0.0;
    lU[i][1] = 1.0;
    if (!live) continue;
    const int c = P.cam(i);
    const double* L = v.l2d[c][t] + 6 * (int64_t)P.ids[i];
    lp[i][0] = L[0];
    lp[i][1] = L[1];
    lU[i][0] = L[4];
    lU[i][1] = L[5];
    cpt[i][0] = v.x[c][P.ids[i]];
    cpt[i][1] = v.y[c][P.ids[i]];
  }
  const int rows = v.rows[t], cols = v.cols[t];
  const double cellp = (double)v.cell;
  const double hw = 0.5 * v.cell, hh = 0.5 * v.cell;
  const double tol_grow = v.tol2d + 1e-6;
  const double tol2 = v.tol2d * v.tol2d;
  const int* cstart = v.cell_start[t];
  const int* citems = v.cell_items[t];
  const double2* cxy = v.cxy[t];
  const double* cbp[K];
#pragma unroll
  for (int i = 0; i < K; ++i) cbp[i] = live ? v.cbp[t][P.cam(i)] : nullptr;

  // Rows that can hold a non-empty span: with two or more strips, the cell-centre rows
  // inside the y-extent of the first two strips' intersection parallelogram (plus one
  // row each side).  Rows outside it have an empty exact span, so skipping them leaves
  // the visited set unchanged.
  int row_lo = 0, row_hi = live ? rows - 1 : -1;
  if (K >= 2 && live) {
    const double n00 = -lU[0][1], n01 = lU[0][0], n10 = -lU[1][1], n11 = lU[1][0];
    const double d0 = -(n00 * lp[0][0] + n01 * lp[0][1]);
    const double d1 = -(n10 * lp[1][0] + n11 * lp[1][1]);
    const double T0 = tol_grow + fabs(n00) * hw + fabs(n01) * hh;
    const double T1 = tol_grow + fabs(n10) * hw + fabs(n11) * hh;
    const double det = n00 * n11 - n01 * n10;
    if (fabs(det) > 1e-9) {
      double ymin = 1e300, ymax = -1e300;
#pragma unroll
      for (int s0 = -1; s0 <= 1; s0 += 2)
#pragma unroll
        for (int s1 = -1; s1 <= 1; s1 += 2) {
          const double y = (n00 * (s1 * T1 - d1) - n10 * (s0 * T0 - d0)) / det;
          ymin = fmin(ymin, y);
          ymax = fmax(ymax, y);
        }
      if (isfinite(ymin) && isfinite(ymax)) {
        const double lo = floor(ymin / cellp - 0.5) - 1.0, hi = ceil(ymax / cellp - 0.5) + 1.0;
        row_lo = (int)fmax(0.0, fmin((double)(rows - 1), lo));
        row_hi = (int)fmax(-1.0, fmin((double)(rows - 1), hi));
      }
    }
  }

  // IDMap::computeStripIntersection, one row: a cell range [xmin, xmax] (empty when
  // xmin > xmax) that contains the reference's.  The range only selects the items that
  // the exact FP64 tests below then decide, and every item that passes them lies in a
  // cell of the reference's range, so any superset of that range gives the same
  // accepted set.  It is evaluated in FP32 with the strip widened by 0.01 px and the
  // cell bounds widened by 1e-3 cells (FP32 errors here stay below 1e-3 px), and the
  // division by n0 folded into one reciprocal per strip.
  float sn0[K], sn1[K], sd[K], sT[K], sinv[K];
  bool shz[K];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const double n0 = -lU[i][1], n1 = lU[i][0];
    sn0[i] = (float)n0;
    sn1[i] = (float)n1;
    sd[i] = (float)(-(n0 * lp[i][0] + n1 * lp[i][1]));
    sT[i] = (float)(tol_grow + fabs(n0) * hw + fabs(n1) * hh) + 0.01f;
    shz[i] = fabs(n0) < 1e-12;
    sinv[i] = shz[i] ? 0.0f : 1.0f / (float)n0;
  }
  const float cellf = (float)cellp, to_index_f = 1.0f / cellf;
  auto row_span = [&](int cy, int& xmin, int& xmax) {
    xmin = 0;
    xmax = cols - 1;
    const float y_c = ((float)cy + 0.5f) * cellf;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const float C = fmaf(sn1[i], y_c, sd[i]);
      int a = 0, b = cols - 1;
      if (shz[i]) {
        if (fabsf(C) > sT[i]) {
          xmin = 1;
          xmax = 0;
        }
      } else {
        float xl = (-sT[i] - C) * sinv[i];
        float xr = (sT[i] - C) * sinv[i];
        if (xl > xr) {
          const float s_ = xl;
          xl = xr;
          xr = s_;
        }
        a = (int)ceilf(xl * to_index_f - 0.5f - 1e-3f);
        b = (int)floorf(xr * to_index_f - 0.5f + 1e-3f);
        a = a > 0 ? a : 0;
        b = b < cols - 1 ? b : cols - 1;
      }
      xmin = xmin > a ? xmin : a;
      xmax = xmax < b ? xmax : b;
    }
  };
  // IDMap::visitPointsInRowSpans precise test and checkBackProjection of the item at
  // cell-ordered position q; true when the pair passes both
  auto item_ok = [&](int q) -> bool {
    const double2 xy = cxy[q];
    bool ok = true;
    // IDMap::visitPointsInRowSpans precise test
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const double dx = xy.x - lp[i][0], dy = xy.y - lp[i][1];
      const double z = dy * lU[i][0] - dx * lU[i][1];
      ok = ok && !(z * z > tol2);
      if (v.near_band > 0.0) {
        const double m = fabs(z) - v.tol2d;
        if (fabs(m) < v.near_band)
          near_append(v, 0, K, t, citems[q], P.cam(i), P.ids[i], m);
      }
    }
    if (!ok) return false;
    // checkBackProjection (StereoMatch.cpp:1206-1227)
#pragma unroll
    for (int i = 0; i < K; ++i) {
      if (!ok) break;
      const double2 a = reinterpret_cast<const double2*>(cbp[i])[2 * q];
      const double2 b = reinterpret_cast<const double2*>(cbp[i])[2 * q + 1];
      const double d0 = cpt[i][0] - a.x, d1 = cpt[i][1] - a.y;
      const double z = d1 * b.x - d0 * b.y;
      ok = !(z * z > tol2);
      if (v.near_band > 0.0) {
        const double m = fabs(z) - v.tol2d;
        if (fabs(m) < v.near_band)
          near_append(v, 1, K, t, citems[q], P.cam(i), P.ids[i], m);
      }
    }
    return ok;
  };

  if constexpr (WARP) {
    // one warp per path: 32 rows at a time (lane = row), then the rows' item ranges
    // flattened over the lanes (consecutive items of a row are adjacent in memory, so
    // the loads coalesce and no lane idles on a short row)
    for (int base = row_lo; base <= row_hi; base += 32) {
      const int cy = base + r0;
      int q0 = 0, cnt = 0;
      if (cy <= row_hi) {
        int xmin, xmax;
        row_span(cy, xmin, xmax);
        if (xmin <= xmax) {
          q0 = cstart[cy * cols + xmin];
          cnt = cstart[cy * cols + xmax + 1] - q0;
        }
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t_ = __shfl_up_sync(0xffffffffu, incl, o);
        if (r0 >= o) incl += t_;
      }
      const int excl = incl - cnt;
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + r0;
        // the row holding item k: the largest lane r with excl[r] <= k
        int r = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int e = __shfl_sync(0xffffffffu, excl, r + step);
          if (e <= k) r += step;
        }
        const int qr = __shfl_sync(0xffffffffu, q0, r);
        const int er = __shfl_sync(0xffffffffu, excl, r);
        if (k >= total) continue;
        const int q = qr + (k - er);
        if (!item_ok(q)) continue;
        const int slot = append_slot(pair_count);
        if (slot < pair_cap) pairs[slot] = Pair{pidx, citems[q]};
      }
    }
  } else {
    // K >= 2, one path per lane: row j of every lane's path at a time, the 32 rows'
    // item ranges flattened over the warp; an item is tested against its owner lane's
    // lines and points (fetched by shuffles), so no lane waits on another's long row
    const int lane = threadIdx.x & 31;
    const int nrow = row_hi >= row_lo ? row_hi - row_lo + 1 : 0;
    const int maxrow = __reduce_max_sync(0xffffffffu, nrow);
    for (int j = 0; j < maxrow; ++j) {
      int q0 = 0, cnt = 0;
      if (j < nrow) {
        const int cy = row_lo + j;
        int xmin, xmax;
        row_span(cy, xmin, xmax);
        if (xmin <= xmax) {
          q0 = cstart[cy * cols + xmin];
          cnt = cstart[cy * cols + xmax + 1] - q0;
        }
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t_ = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t_;
      }
      const int excl = incl - cnt;
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        int r = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int e = __shfl_sync(0xffffffffu, excl, r + step);
          if (e <= k) r += step;
        }
        const int qr = __shfl_sync(0xffffffffu, q0, r);
        const int er = __shfl_sync(0xffffffffu, excl, r);
        const int ot = __shfl_sync(0xffffffffu, t, r);
        const int opidx = __shfl_sync(0xffffffffu, pidx, r);
        double Lp[K][2], LU[K][2], Cp[K][2];
        const double* Cb[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
          Lp[i][0] = __shfl_sync(0xffffffffu, lp[i][0], r);
          Lp[i][1] = __shfl_sync(0xffffffffu, lp[i][1], r);
          LU[i][0] = __shfl_sync(0xffffffffu, lU[i][0], r);
          LU[i][1] = __shfl_sync(0xffffffffu, lU[i][1], r);
          Cp[i][0] = __shfl_sync(0xffffffffu, cpt[i][0], r);
          Cp[i][1] = __shfl_sync(0xffffffffu, cpt[i][1], r);
          Cb[i] = reinterpret_cast<const double*>(__shfl_sync(
              0xffffffffu, reinterpret_cast<unsigned long long>(cbp[i]), r));
        }
        if (k >= total) continue;
        const int q = qr + (k - er);
        const double2 xy = v.cxy[ot][q];
        bool ok = true;
        // IDMap::visitPointsInRowSpans precise test
#pragma unroll
        for (int i = 0; i < K; ++i) {
          const double dx = xy.x - Lp[i][0], dy = xy.y - Lp[i][1];
          const double z = dy * LU[i][0] - dx * LU[i][1];
          ok = ok && !(z * z > tol2);
          if (v.near_band > 0.0) {
            const double m = fabs(z) - v.tol2d;
            if (fabs(m) < v.near_band)
              near_append(v, 0, K, ot, v.cell_items[ot][q], in[opidx].cam(i), in[opidx].ids[i], m);
          }
        }
        if (!ok) continue;
        // checkBackProjection (StereoMatch.cpp:1206-1227)
#pragma unroll
        for (int i = 0; i < K; ++i) {
          if (!ok) break;
          const double2 a = reinterpret_cast<const double2*>(Cb[i])[2 * q];
          const double2 b = reinterpret_cast<const double2*>(Cb[i])[2 * q + 1];
          const double d0 = Cp[i][0] - a.x, d1 = Cp[i][1] - a.y;
          const double z = d1 * b.x - d0 * b.y;
          ok = !(z * z > tol2);
          if (v.near_band > 0.0) {
            const double m = fabs(z) - v.tol2d;
            if (fabs(m) < v.near_band)
              near_append(v, 1, K, ot, v.cell_items[ot][q], in[opidx].cam(i), in[opidx].ids[i], m);
          }
        }
        if (!ok) continue;
        const int slot = append_slot(pair_count);
        if (slot < pair_cap) pairs[slot] = Pair{opidx, v.cell_items[ot][q]};
      }
    }
  }
}

// Expand one level, second half: one thread per (path, candidate) pair.  The quick
// triangulation gate (computeMinParallaxDeg, calTriangulateTol,
// TriangulationCheckWithTol: StereoMatch.cpp:1072-1141) on the path's lines plus the
// candidate's, then the child path (terminal, or with its next target camera).
template <int K>
__global__ void __launch_bounds__(256, 2) tri_kernel(const __grid_constant__ SmView v, const void* in_v,
                                                     const Pair* pairs, int n_pairs, void* out_v,
                                                     int* out_count, int out_cap, Path* term,
                                                     int* term_count, int term_cap) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= n_pairs) return;
  const Pair pr = pairs[gi];
  const PathN<K> P = static_cast<const PathN<K>*>(in_v)[pr.path];
  const int t = P.target;
  const int pid = pr.pid;
  double cp[K][3], cu[K][3];  // chosen lines of sight (build order)
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const double* S = v.los[P.cam(i)] + 6 * (int64_t)P.ids[i];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      cp[i][q] = S[q];
      cu[i][q] = S[3 + q];
    }
  }
  // Normal equations of the chosen lines, summed in build order: the candidate's
  // term is added last, which is the reference's summation order
  // (myMATH::triangulation sums lines in list order, myMATH.cpp:376-391).
  double Mc[9], bc[3];
#pragma unroll
  for (int q = 0; q < 9; ++q) Mc[q] = 0.0;
  bc[0] = bc[1] = bc[2] = 0.0;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    double tt[9];
    normal_terms(cu[i], tt);
#pragma unroll
    for (int r = 0; r < 3; ++r)
      bc[r] = bc[r] + (tt[3 * r] * cp[i][0] + tt[3 * r + 1] * cp[i][1] + tt[3 * r + 2] * cp[i][2]);
#pragma unroll
    for (int q = 0; q < 9; ++q) Mc[q] = Mc[q] + tt[q];
  }
  // largest pairwise dot (smallest parallax) among the chosen lines
  double maxdot_c = -2.0;
#pragma unroll
  for (int i = 0; i < K; ++i)
#pragma unroll
    for (int j = i + 1; j < K; ++j) maxdot_c = fmax(maxdot_c, clamped_dot(cu[i], cu[j]));

  {
    {
      {
        // extend the path; quick triangulation gate (computeMinParallaxDeg,
        // calTriangulateTol, TriangulationCheckWithTol: StereoMatch.cpp:1072-1141)
        double qp[3], qu[3];
        {
          const double* S = v.los[t] + 6 * (int64_t)pid;
          qp[0] = S[0];
          qp[1] = S[1];
          qp[2] = S[2];
          qu[0] = S[3];
          qu[1] = S[4];
          qu[2] = S[5];
        }
        constexpr int k1 = K + 1;
        double maxdot = maxdot_c;
#pragma unroll
        for (int i = 0; i < K; ++i) maxdot = fmax(maxdot, clamped_dot(cu[i], qu));
        double tq;
        if (maxdot <= kCos6 - 1e-9 && maxdot >= -kCos6 + 1e-9) {
          // min parallax in (6 + 5e-7, 174 - 5e-7) deg: the angle factor is exactly 1
          tq = v.tol3d * sqrt(double(v.m > 2 ? v.m : 2) / double(k1)) * 1.0;
        } else {
          // near the 6-degree knee or beyond: the reference's acos/sin path
          double min_deg = 180.0;
#pragma unroll
          for (int i = 0; i < k1; ++i)
#pragma unroll
            for (int j = i + 1; j < k1; ++j)
              min_deg = fmin(min_deg, pair_deg(i < K ? cu[i] : qu, j < K ? cu[j] : qu));
          tq = quick_tol_from_deg(min_deg, k1, v.m, v.tol3d);
        }
        double M[9], b[3];
        {
          double tt[9];
          normal_terms(qu, tt);
#pragma unroll
          for (int r = 0; r < 3; ++r)
            b[r] = bc[r] + (tt[3 * r] * qp[0] + tt[3 * r + 1] * qp[1] + tt[3 * r + 2] * qp[2]);
#pragma unroll
          for (int q2 = 0; q2 < 9; ++q2) M[q2] = Mc[q2] + tt[q2];
        }
        double Mi[9], X[3];
        gauss_inverse3(M, Mi);
#pragma unroll
        for (int r = 0; r < 3; ++r) X[r] = Mi[3 * r] * b[0] + Mi[3 * r + 1] * b[1] + Mi[3 * r + 2] * b[2];
        double e = 0.0;
        bool thrown = false;
#pragma unroll
        for (int i = 0; i < k1; ++i) {
          const double* pp = (i < K) ? cp[i] : qp;
          const double* uu = (i < K) ? cu[i] : qu;
          thrown |= !line_error_term(X, pp, uu, e);
        }
        if (thrown) return;  // the reference's triangulation throws; the check fails
        const double err = sqrt(e / k1);
        if (!(err <= tq)) return;
        PathN<K + 1> ch;
#pragma unroll
        for (int i = 0; i < K; ++i) ch.ids[i] = P.ids[i];
        ch.ids[K] = pid;
        ch.cams = P.cams | ((unsigned)t << (4 * K));
        if (k1 == v.m) {
          Path full;
#pragma unroll
          for (int i = 0; i < OLPT_MAX_CAM; ++i) {
            full.ids[i] = 0;
            full.cams[i] = 0;
          }
#pragma unroll
          for (int i = 0; i < K + 1; ++i) {
            full.ids[i] = ch.ids[i];
            full.cams[i] = (signed char)ch.cam(i);
          }
          full.k = k1;
          full.target = -1;
          const int slot = append_slot(term_count);
          if (slot < term_cap) term[slot] = full;
          return;
        }
        if (k1 >= OLPT_MAX_CAM) return;
        // StereoMatch::selectNextCameraByMaxPairAngle (StereoMatch.cpp:1375-1411)
        int best = -1;
        double best_score = -1.0;
        for (int cam = 0; cam < v.n_cam; ++cam) {
          if (!v.active[cam]) continue;
          bool used = false;
#pragma unroll
          for (int i = 0; i < K + 1; ++i) used |= (ch.cam(i) == cam);
          if (used) continue;
          double ux[K + 1], uy[K + 1];
#pragma unroll
          for (int i = 0; i < K + 1; ++i) {
            const double* L = v.l2d[ch.cam(i)][cam] + 6 * (int64_t)ch.ids[i];
            ux[i] = L[2];
            uy[i] = L[3];
          }
          double score = 0.0;
          if (k1 >= 2) {
#pragma unroll
            for (int i = 0; i < K + 1; ++i) {
#pragma unroll
              for (int j = i + 1; j < K + 1; ++j) {
                const double s = fabs(ux[i] * uy[j] - uy[i] * ux[j]);
                if (s > score) score = s;
                if (score >= 1.0 - 1e-12) break;
              }
              if (score >= 1.0 - 1e-12) break;
            }
          }
          if (score > best_score) {
            best_score = score;
            best = cam;
          }
        }
        if (best < 0) return;
        ch.target = best;
        const int slot = append_slot(out_count);
        if (slot < out_cap) static_cast<PathN<K + 1>*>(out_v)[slot] = ch;
      }
    }
  }
}


// StereoMatch::checkMatch, case "every active camera was used to build"
// (StereoMatch.cpp:520-540): triangulate in camera order, gate on tol_3d and limit.
__global__ void check_kernel(const __grid_constant__ SmView v, const Path* term, int n_term, int* cand_ids,
                             double* cand_e, double* cand_x, int* cand_count, int cap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_term) return;
  const Path P = term[i];
  int ids[OLPT_MAX_CAM];
  for (int c = 0; c < v.n_cam; ++c) ids[c] = -1;
  for (int j = 0; j < P.k; ++j) ids[P.cams[j]] = P.ids[j];
  Line3 Ls[OLPT_MAX_CAM];
  const Line3* Lp[OLPT_MAX_CAM];
  int n = 0;
  for (int c = 0; c < v.n_cam; ++c) {
    if (ids[c] < 0) continue;
    load_line3(v.los[c] + 6 * (int64_t)ids[c], Ls[n]);
    Lp[n] = &Ls[n];
    ++n;
  }
  double X[3], err;
  if (!triangulate<OLPT_MAX_CAM>(Lp, n, X, err)) return;  // the reference throws here
  if (err > v.tol3d) return;
  if (X[0] > v.limit[1] || X[0] < v.limit[0] || X[1] > v.limit[3] || X[1] < v.limit[2] ||
      X[2] > v.limit[5] || X[2] < v.limit[4])
    return;
  int slot = atomicAdd(cand_count, 1);
  if (slot >= cap) return;
  for (int c = 0; c < v.n_cam; ++c) cand_ids[(int64_t)slot * v.n_cam + c] = ids[c];
  cand_e[slot] = err;
  cand_x[3 * slot] = X[0];
  cand_x[3 * slot + 1] = X[1];
  cand_x[3 * slot + 2] = X[2];
}

}  // namespace

// ---------------------------------------------------------------- host driver
// Steps 2-6 of pruneMatch on the candidates in ctx->prune.ids_s / e_s (M x n_cam, in
// the reference's order): the kept flags end in ctx->prune.sel (device, M bytes) and,
// when selected is given, on the host.  False when the comparator sorts must run on
// the host (prune_candidates) instead.
bool prune_select_device(olpt_ctx* ctx, const PruneView& pv, int M, int n_cam,
                         int64_t total_points, char* selected) {
  cudaStream_t s = ctx->stream;
  PruneWork& P = ctx->prune;
  int G = 0;
  if (!prune_order_device(P, pv, M, n_cam, total_points, &G, s)) return false;
  P.sel.ensure((size_t)M + 16, s);
  if (greedy_device(P, M, G, n_cam, total_points, P.sel.as<uint8_t>(), s)) {
    if (selected && M > 0) {
      OLPT_CUDA(cudaMemcpyAsync(selected, P.sel.p, (size_t)M, cudaMemcpyDeviceToHost, s));
      OLPT_CUDA(cudaStreamSynchronize(s));
    }
    return true;
  }
  // a replacement fires: the sequential greedy over pinned staging
  PhaseTimer pg(ctx->prof, PH_GREEDY_HOST);
  const size_t b_ord = (size_t)G * sizeof(int), b_pts = (size_t)G * n_cam * sizeof(int);
  const size_t b_dbl = (size_t)G * sizeof(double);
  P.pin.ensure(b_ord + b_pts + 2 * b_dbl + G + 64);
  char* hp = P.pin.as<char>();
  double* g_pct = reinterpret_cast<double*>(hp);
  double* g_e = reinterpret_cast<double*>(hp + b_dbl);
  int* order = reinterpret_cast<int*>(hp + 2 * b_dbl);
  int* g_pts = reinterpret_cast<int*>(hp + 2 * b_dbl + b_ord);
  uint8_t* g_cnt = reinterpret_cast<uint8_t*>(hp + 2 * b_dbl + b_ord + b_pts);
  if (G > 0) {
    OLPT_CUDA(cudaMemcpyAsync(order, P.val.p, b_ord, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(g_pts, P.g_pts.p, b_pts, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(g_cnt, P.g_cnt.p, (size_t)G, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(g_pct, P.g_pct.p, b_dbl, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(g_e, P.g_e.p, b_dbl, cudaMemcpyDeviceToHost, s));
  }
  OLPT_CUDA(cudaStreamSynchronize(s));
  std::vector<char> sel(G, 0);
  greedy_select(G, n_cam, g_pts, g_cnt, g_pct, g_e, total_points, sel.data());
  std::vector<char> flags(M, 0);
  for (int i = 0; i < G; ++i)
    if (sel[i]) flags[order[i]] = 1;
  if (M > 0) {
    OLPT_CUDA(cudaMemcpyAsync(P.sel.p, flags.data(), (size_t)M, cudaMemcpyHostToDevice, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
  }
  if (selected) std::copy(flags.begin(), flags.end(), selected);
  return true;
}

void stereo_match_device(olpt_ctx* ctx, const SmParams& prm, StereoResult& res) {
  cudaStream_t s = ctx->stream;
  const int n_cam = ctx->n_cam;
  SmView v{};
  v.n_cam = n_cam;
  res.on_device = false;
  res.M = 0;
  int n_active = 0;
  for (int c = 0; c < n_cam; ++c) {
    v.active[c] = ctx->cams_h[c].is_active;
    n_active += v.active[c];
  }
  OLPT_REQUIRE(n_active >= 2, OLPT_ERR_INVALID_ARG, "preCheck: need at least 2 active cameras.");
  OLPT_REQUIRE(prm.match_cam_count >= 2 && prm.match_cam_count <= n_active, OLPT_ERR_INVALID_ARG,
               "preCheck: match_cam_count must be within [2," + std::to_string(n_active) + "].");
  v.n_active = n_active;
  v.m = std::min(std::max(2, prm.match_cam_count), n_active);
  OLPT_REQUIRE(v.m == n_active, OLPT_ERR_UNSUPPORTED,
               "match_cam_count below the number of active cameras: the reference aborts on this "
               "path (checkMatch leaves e_check NaN, StereoMatch.cpp:561-600 vs :129)");
  v.cell = std::max(1, prm.idmap_cell_px);
  v.tol2d = prm.tol_2d_px;
  v.tol3d = prm.tol_3d_mm;
  v.near_band = ctx->sm.near_band;
  if (v.near_band > 0.0) {
    v.near_rec = ctx->sm.near_rec.as<olpt_near_record>();
    v.near_count = ctx->sm.near_count.as<unsigned long long>();
    v.near_cap = ctx->sm.near_cap;
  }
  for (int q = 0; q < 6; ++q) v.limit[q] = prm.limit[q];

  StereoWork& W = ctx->sm;
  // reference camera: fewest detections among active (StereoMatch.cpp:70-85)
  int ref = -1;
  int64_t best = INT64_MAX;
  for (int c = 0; c < n_cam; ++c) {
    if (!v.active[c]) continue;
    if (ctx->det_counts_h[c] < best) {
      best = ctx->det_counts_h[c];
      ref = c;
    }
  }
  res.ref_cam = ref;

  // grids and lines
  for (int c = 0; c < n_cam; ++c) {
    const CamDev& cm = ctx->cams_h[c];
    const int64_t n = v.active[c] ? ctx->det_counts_h[c] : 0;
    v.n[c] = n;
    v.x[c] = ctx->dets[c].x.as<double>();
    v.y[c] = ctx->dets[c].y.as<double>();
    v.Wd[c] = (double)cm.n_col;
    v.Hd[c] = (double)cm.n_row;
    const int rows = std::max(1, cm.n_row / v.cell + (cm.n_row % v.cell ? 1 : 0));
    const int cols = std::max(1, cm.n_col / v.cell + (cm.n_col % v.cell ? 1 : 0));
    v.rows[c] = rows;
    v.cols[c] = cols;
    if (!v.active[c]) continue;
    const int ncell = rows * cols;
    W.cell_start[c].ensure((ncell + 1) * sizeof(int), s);
    W.cell_cursor[c].ensure(ncell * sizeof(int), s);
    W.cell_items[c].ensure((n + 1) * sizeof(int), s);
    W.cell_of[c].ensure((n + 1) * sizeof(int), s);
    W.los[c].ensure((n + 1) * 6 * sizeof(double), s);
    OLPT_CUDA(cudaMemsetAsync(W.cell_cursor[c].p, 0, ncell * sizeof(int), s));
    if (n > 0) {
      cell_hist_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(v.x[c], v.y[c], n, v.cell, rows, cols,
                                                W.cell_of[c].as<int>(), W.cell_cursor[c].as<int>());
    }
    exclusive_scan(W.cell_cursor[c].as<int>(), ncell, W.cell_start[c].as<int>(), W.scan_tmp, s);
    OLPT_CUDA(cudaMemsetAsync(W.cell_cursor[c].p, 0, ncell * sizeof(int), s));
    if (n > 0) {
      cell_scatter_kernel<<<OLPT_G(nblk(n)), 256, 0, s>>>(W.cell_of[c].as<int>(), n, W.cell_start[c].as<int>(),
                                                   W.cell_cursor[c].as<int>(), W.cell_items[c].as<int>());
      cell_sort_kernel<<<OLPT_G(nblk(ncell)), 256, 0, s>>>(W.cell_start[c].as<int>(), ncell,
                                                    W.cell_items[c].as<int>());
    }
    OLPT_CUDA(cudaGetLastError());
    v.cell_start[c] = W.cell_start[c].as<int>();
    v.cell_items[c] = W.cell_items[c].as<int>();
    v.los[c] = W.los[c].as<double>();
  }
  // image lines of every detection on every other active camera
  {
    W.l2d_ptrs.ensure(OLPT_MAX_CAM * OLPT_MAX_CAM * sizeof(double*), s);
    W.active_d.ensure(OLPT_MAX_CAM * sizeof(int), s);
    std::vector<double*> ptrs(OLPT_MAX_CAM * OLPT_MAX_CAM, nullptr);
    for (int c = 0; c < n_cam; ++c) {
      if (!v.active[c]) continue;
      for (int t = 0; t < n_cam; ++t) {
        if (t == c || !v.active[t]) continue;
        DevBuf& b = W.l2d[c * OLPT_MAX_CAM + t];
        b.ensure((v.n[c] + 1) * 6 * sizeof(double), s);
        ptrs[c * OLPT_MAX_CAM + t] = b.as<double>();
        v.l2d[c][t] = b.as<double>();
      }
    }
    OLPT_CUDA(cudaMemcpyAsync(W.l2d_ptrs.p, ptrs.data(), ptrs.size() * sizeof(double*),
                              cudaMemcpyHostToDevice, s));
    OLPT_CUDA(cudaMemcpyAsync(W.active_d.p, v.active, OLPT_MAX_CAM * sizeof(int),
                              cudaMemcpyHostToDevice, s));
    for (int c = 0; c < n_cam; ++c) {
      if (!v.active[c] || v.n[c] == 0) continue;
      lines_kernel<<<OLPT_G(nblk(v.n[c], 128)), 128, 0, s>>>(
          ctx->cams_d.as<CamDev>(), c, v.x[c], v.y[c], v.n[c], n_cam, W.active_d.as<int>(),
          W.los[c].as<double>(), W.l2d_ptrs.as<double*>() + c * OLPT_MAX_CAM);
      OLPT_CUDA(cudaGetLastError());
    }
    // cell-ordered copies for the enumeration
    W.cbp_ptrs.ensure(2 * OLPT_MAX_CAM * OLPT_MAX_CAM * sizeof(double*), s);
    std::vector<double*> bp(2 * OLPT_MAX_CAM * OLPT_MAX_CAM, nullptr);
    for (int t = 0; t < n_cam; ++t) {
      if (!v.active[t]) continue;
      W.cxy[t].ensure((v.n[t] + 1) * sizeof(double2), s);
      v.cxy[t] = W.cxy[t].as<double2>();
      for (int c = 0; c < n_cam; ++c) {
        if (c == t || !v.active[c]) continue;
        DevBuf& b = W.cbp[t * OLPT_MAX_CAM + c];
        b.ensure((v.n[t] + 1) * 4 * sizeof(double), s);
        bp[t * OLPT_MAX_CAM + c] = b.as<double>();
        v.cbp[t][c] = b.as<double>();
      }
      for (int c = 0; c < n_cam; ++c)
        bp[OLPT_MAX_CAM * OLPT_MAX_CAM + t * OLPT_MAX_CAM + c] = ptrs[t * OLPT_MAX_CAM + c];
    }
    OLPT_CUDA(cudaMemcpyAsync(W.cbp_ptrs.p, bp.data(), bp.size() * sizeof(double*),
                              cudaMemcpyHostToDevice, s));
    for (int t = 0; t < n_cam; ++t) {
      if (!v.active[t] || v.n[t] == 0) continue;
      double* const* outs = W.cbp_ptrs.as<double*>() + t * OLPT_MAX_CAM;
      const double* const* lines =
          W.cbp_ptrs.as<const double*>() + OLPT_MAX_CAM * OLPT_MAX_CAM + t * OLPT_MAX_CAM;
      cell_pack_kernel<<<OLPT_G(nblk(v.n[t])), 256, 0, s>>>(
          W.cell_items[t].as<int>(), v.n[t], v.x[t], v.y[t], W.cxy[t].as<double2>(), outs, lines,
          n_cam, t);
      OLPT_CUDA(cudaGetLastError());
    }
  }

  // breadth-first expansion of the build DFS
  W.counters.ensure(8 * sizeof(int), s);
  int* cnt = W.counters.as<int>();
  auto read_count = [&](int idx) {
    int h = 0;
    OLPT_CUDA(cudaMemcpyAsync(&h, cnt + idx, sizeof(int), cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    return h;
  };
  int64_t n_ref = v.n[ref];
  int cap_a = (int)std::max<int64_t>(n_ref, 1024);
  W.path_a.ensure(cap_a * sizeof(Path), s);
  OLPT_CUDA(cudaMemsetAsync(cnt, 0, 8 * sizeof(int), s));
  if (n_ref > 0)
    seed_kernel<<<OLPT_G(nblk(n_ref)), 256, 0, s>>>(v, ref, W.path_a.as<PathN<1>>(), cnt, cap_a);
  OLPT_CUDA(cudaGetLastError());
  int n_in = read_count(0);
  int term_cap = (int)std::max<int64_t>(4 * n_ref, 4096);
  W.term.ensure(term_cap * sizeof(Path), s);
  int n_term = 0;
  DevBuf* in_buf = &W.path_a;
  DevBuf* out_buf = &W.path_b;
  int out_cap = (int)std::max<int64_t>(16 * (int64_t)n_in, 4096);
  int pair_cap = (int)std::max<int64_t>(8 * (int64_t)n_in, 4096);
  for (int level = 1; level < v.m && n_in > 0; ++level) {
    // candidates of every path that pass the 2D tests
    int n_pairs = 0;
    // buffers are grow-only: their capacity from earlier calls avoids a redo
    pair_cap = (int)std::max<int64_t>(pair_cap, (int64_t)(W.pairs.bytes / sizeof(Pair)) - 1);
    for (;;) {
      W.pairs.ensure((size_t)pair_cap * sizeof(Pair), s);
      OLPT_CUDA(cudaMemsetAsync(cnt + 4, 0, sizeof(int), s));
      const int pid = ctx->prof.begin(PROF_STEREO, s);
      auto kern = enum_kernel<1, true>;
      switch (level) {
        case 1: kern = enum_kernel<1, true>; break;
        case 2: kern = enum_kernel<2, false>; break;
        case 3: kern = enum_kernel<3, false>; break;
        case 4: kern = enum_kernel<4, false>; break;
        case 5: kern = enum_kernel<5, false>; break;
        case 6: kern = enum_kernel<6, false>; break;
        default: kern = enum_kernel<7, false>; break;
      }
      const int64_t work = level == 1 ? (int64_t)n_in * 32 : (int64_t)n_in;
      kern<<<OLPT_G(nblk(work)), 256, 0, s>>>(v, in_buf->p, n_in, W.pairs.as<Pair>(), cnt + 4,
                                                pair_cap);
      ctx->prof.end(PROF_STEREO, pid, s, 0.0);
      OLPT_CUDA(cudaGetLastError());
      n_pairs = read_count(4);
      if (n_pairs > pair_cap) {  // grow and redo
        pair_cap = n_pairs + n_pairs / 4 + 1024;
        continue;
      }
      break;
    }
    // quick triangulation gate and the children
    out_cap = (int)std::max<int64_t>(out_cap, (int64_t)(out_buf->bytes / sizeof(Path)) - 1);
    term_cap = (int)std::max<int64_t>(term_cap, (int64_t)(W.term.bytes / sizeof(Path)) - 1);
    for (;;) {
      out_buf->ensure((size_t)out_cap * sizeof(Path), s);
      W.term.ensure((size_t)term_cap * sizeof(Path), s);
      // counters: [1] = children, [2] = terminals (terminals accumulate across levels)
      OLPT_CUDA(cudaMemsetAsync(cnt + 1, 0, sizeof(int), s));
      OLPT_CUDA(cudaMemcpyAsync(cnt + 2, &n_term, sizeof(int), cudaMemcpyHostToDevice, s));
      const int pid = ctx->prof.begin(PROF_STEREO, s);
      auto kern = tri_kernel<1>;
      switch (level) {
        case 1: kern = tri_kernel<1>; break;
        case 2: kern = tri_kernel<2>; break;
        case 3: kern = tri_kernel<3>; break;
        case 4: kern = tri_kernel<4>; break;
        case 5: kern = tri_kernel<5>; break;
        case 6: kern = tri_kernel<6>; break;
        default: kern = tri_kernel<7>; break;
      }
      if (n_pairs > 0)
        kern<<<OLPT_G(nblk(n_pairs)), 256, 0, s>>>(v, in_buf->p, W.pairs.as<Pair>(), n_pairs,
                                                   out_buf->p, cnt + 1, out_cap,
                                                   W.term.as<Path>(), cnt + 2, term_cap);
      ctx->prof.end(PROF_STEREO, pid, s, 0.0);
      OLPT_CUDA(cudaGetLastError());
      int h[2];
      OLPT_CUDA(cudaMemcpyAsync(h, cnt + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      OLPT_CUDA(cudaStreamSynchronize(s));
      if (h[0] > out_cap || h[1] > term_cap) {  // grow and redo this level
        out_cap = std::max(out_cap, h[0] + h[0] / 4 + 1024);
        term_cap = std::max(term_cap, h[1] + h[1] / 4 + 1024);
        continue;
      }
      n_in = h[0];
      n_term = h[1];
      break;
    }
    std::swap(in_buf, out_buf);
    out_cap = (int)std::max<int64_t>(4 * (int64_t)n_in, 4096);
  }

  // check + candidate list
  int cap_c = std::max(n_term, 1);
  W.cand_ids.ensure((size_t)cap_c * n_cam * sizeof(int), s);
  W.cand_e.ensure((size_t)cap_c * sizeof(double), s);
  W.cand_x.ensure((size_t)cap_c * 3 * sizeof(double), s);
  OLPT_CUDA(cudaMemsetAsync(cnt + 3, 0, sizeof(int), s));
  if (n_term > 0)
    check_kernel<<<OLPT_G(nblk(n_term, 128)), 128, 0, s>>>(v, W.term.as<Path>(), n_term, W.cand_ids.as<int>(),
                                              W.cand_e.as<double>(), W.cand_x.as<double>(), cnt + 3,
                                              cap_c);
  OLPT_CUDA(cudaGetLastError());
  const int M = read_count(3);
  res.n_cam = n_cam;
  PhaseTimer pt(ctx->prof, PH_PRUNE);
  std::vector<int> counts(n_cam);
  std::vector<int> active(n_cam);
  PruneView pv{};
  int64_t total_points = 0;
  int max_count = 0;
  for (int c = 0; c < n_cam; ++c) {
    counts[c] = (int)ctx->det_counts_h[c];
    active[c] = v.active[c];
    pv.active[c] = v.active[c];
    pv.count[c] = counts[c];
    pv.offset[c] = (int)total_points;
    total_points += counts[c];
    max_count = std::max(max_count, counts[c]);
  }
  res.M = M;
  PruneWork& P = ctx->prune;
  auto download = [&](const void* ids, const void* e, const void* X) {
    res.ids.resize((size_t)M * n_cam);
    res.e.resize(M);
    res.X.resize((size_t)M * 3);
    if (M == 0) return;
    OLPT_CUDA(cudaMemcpyAsync(res.ids.data(), ids, (size_t)M * n_cam * sizeof(int),
                              cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(res.e.data(), e, (size_t)M * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(res.X.data(), X, (size_t)M * 3 * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  };
  // candidate order, prune and greedy on the device
  if (sort_candidates_device(P, W.cand_ids.as<int>(), W.cand_e.as<double>(),
                             W.cand_x.as<double>(), M, n_cam, max_count - 1, s)) {
    if (prune_select_device(ctx, pv, M, n_cam, total_points, nullptr)) {
      res.ids.clear();
      res.e.clear();
      res.X.clear();
      res.selected.clear();
      res.on_device = true;  // downloaded on demand (stereo_result_to_host)
      return;
    }
    download(P.ids_s.p, P.e_s.p, P.X_s.p);
    OLPT_CUDA(cudaStreamSynchronize(s));
  } else {
    download(W.cand_ids.p, W.cand_e.p, W.cand_x.p);
    OLPT_CUDA(cudaStreamSynchronize(s));
    sort_candidates(res);
  }
  prune_candidates(res, counts, active);
}

__global__ void sel_count_kernel(const uint8_t* sel, int M, int* f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M) f[i] = sel[i] ? 1 : 0;
}

__global__ void sel_gather_kernel(const uint8_t* sel, const int* pos, int M, const double* X,
                                  double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M || !sel[i]) return;
  const int k = pos[i];
  out[3 * k] = X[3 * i];
  out[3 * k + 1] = X[3 * i + 1];
  out[3 * k + 2] = X[3 * i + 2];
}

void stereo_result_to_host(olpt_ctx* ctx, StereoResult& r) {
  if (!r.on_device) return;
  cudaStream_t s = ctx->stream;
  PruneWork& P = ctx->prune;
  const int64_t M = r.M;
  const int n = r.n_cam;
  r.ids.resize((size_t)M * n);
  r.e.resize(M);
  r.X.resize((size_t)M * 3);
  r.selected.resize(M);
  if (M > 0) {
    OLPT_CUDA(cudaMemcpyAsync(r.ids.data(), P.ids_s.p, (size_t)M * n * sizeof(int),
                              cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(r.e.data(), P.e_s.p, (size_t)M * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(r.X.data(), P.X_s.p, (size_t)M * 3 * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(r.selected.data(), P.sel.p, (size_t)M, cudaMemcpyDeviceToHost, s));
  }
  OLPT_CUDA(cudaStreamSynchronize(s));
  r.on_device = false;
}

int64_t stereo_objects(olpt_ctx* ctx, const StereoResult& r) {
  cudaStream_t s = ctx->stream;
  int64_t n = 0;
  if (r.on_device) {
    PruneWork& P = ctx->prune;
    const int M = (int)r.M;
    P.spos.ensure((size_t)(M + 1) * sizeof(int), s);
    P.scnt.ensure((size_t)(M + 1) * sizeof(int), s);
    if (M > 0)
      sel_count_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(P.sel.as<uint8_t>(), M, P.scnt.as<int>());
    exclusive_scan(P.scnt.as<int>(), M, P.spos.as<int>(), P.scan_tmp, s);
    int total = 0;
    OLPT_CUDA(cudaMemcpyAsync(&total, P.spos.as<int>() + M, sizeof(int), cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    n = total;
    ctx->obj.ensure(std::max<int64_t>(n, 1), ctx->n_cam, s);
    ctx->obj.n = n;
    if (n > 0)
      sel_gather_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(P.sel.as<uint8_t>(), P.spos.as<int>(), M,
                                                       P.X_s.as<double>(), ctx->obj.xyz.as<double>());
    OLPT_CUDA(cudaGetLastError());
    return n;
  }
  std::vector<double> xyz;
  for (size_t j = 0; j < r.selected.size(); ++j)
    if (r.selected[j]) xyz.insert(xyz.end(), &r.X[3 * j], &r.X[3 * j] + 3);
  n = (int64_t)(xyz.size() / 3);
  ctx->obj.ensure(std::max<int64_t>(n, 1), ctx->n_cam, s);
  ctx->obj.n = n;
  if (n > 0) {
    OLPT_CUDA(cudaMemcpyAsync(ctx->obj.xyz.p, xyz.data(), xyz.size() * sizeof(double),
                              cudaMemcpyHostToDevice, s));
    OLPT_CUDA(cudaStreamSynchronize(s));  // xyz is a local host buffer
  }
  return n;
}

}  // namespace olpt
