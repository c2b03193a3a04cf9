/*
 * Test infrastructure only -- C restatement of the reference's hot-path arithmetic
 * (see olpt_oracle.h).  FP64, IEEE, no FMA contraction.
 */
#include "olpt_oracle.h"

#include <float.h>
#include <math.h>

/* safe_ln and the 3-point log-parabola of ObjectFinder2D::findTracer2D
 * (src/srcObject/ObjectFinder.cpp:54-97). */
static double safe_ln(double v) { return log(v < 1e-4 ? 1e-4 : v); }

static int fit3(double l1, double l2, double l3, int p, double* out) {
  const int p1 = p - 1, p2 = p, p3 = p + 1;
  const double num = l1 * (double)((p2 * p2) - (p3 * p3)) - l2 * (double)((p1 * p1) - (p3 * p3)) +
                     l3 * (double)((p1 * p1) - (p2 * p2));
  const double den = l1 * (double)(p3 - p2) - l3 * (double)(p1 - p2) + l2 * (double)(p1 - p3);
  double c;
  if (den == 0.0) return 0;
  c = -0.5 * (num / den);
  if (!isfinite(c)) return 0;
  *out = c;
  return 1;
}

/* ObjectFinder2D::findTracer2D (ObjectFinder.cpp:37-111) with myMATH::isLocalMax
 * (inc/libMath/myMATH.h:399-435): raster order, border excluded, up/left reject on
 * strictly greater, down/right on greater-or-equal. */
int64_t oo_find_peaks(const double* img, int H, int W, double min_int, double* out_xy,
                      int64_t cap) {
  int64_t n = 0;
  int r, c;
  for (r = 1; r < H - 1; ++r) {
    for (c = 1; c < W - 1; ++c) {
      const double v = img[(int64_t)r * W + c];
      const double up = img[(int64_t)(r - 1) * W + c], dn = img[(int64_t)(r + 1) * W + c];
      const double lf = img[(int64_t)r * W + c - 1], rt = img[(int64_t)r * W + c + 1];
      double xc, yc;
      if (v < min_int) continue;
      if (up > v || lf > v || dn >= v || rt >= v) continue;
      if (!fit3(safe_ln(lf), safe_ln(v), safe_ln(rt), c, &xc)) continue;
      if (!fit3(safe_ln(up), safe_ln(v), safe_ln(dn), r, &yc)) continue;
      if (n < cap) {
        out_xy[2 * n] = xc;
        out_xy[2 * n + 1] = yc;
      }
      ++n;
    }
  }
  return n;
}

static int is_distorted(const oo_pinhole* c) {
  int k;
  for (k = 0; k < c->n_dist; ++k)
    if (c->dist[k] > 1e-8) return 1; /* Camera.cpp:55-67 */
  return 0;
}

/* Camera::worldToUndistImg (Camera.cpp:679-690) */
void oo_pinhole_world_to_undist(const oo_pinhole* c, const double X[3], double xy[2]) {
  double t0 = c->R[0] * X[0] + c->R[1] * X[1] + c->R[2] * X[2];
  double t1 = c->R[3] * X[0] + c->R[4] * X[1] + c->R[5] * X[2];
  double t2 = c->R[6] * X[0] + c->R[7] * X[1] + c->R[8] * X[2];
  t0 = t0 + c->T[0];
  t1 = t1 + c->T[1];
  t2 = t2 + c->T[2];
  xy[0] = (t2 != 0.0) ? (t0 / t2) : t0;
  xy[1] = (t2 != 0.0) ? (t1 / t2) : t1;
}

/* Camera::distort (Camera.cpp:913-966) */
void oo_pinhole_distort(const oo_pinhole* c, const double in[2], double uv[2]) {
  const double x = in[0], y = in[1];
  double xd = x, yd = y;
  if (is_distorted(c)) {
    const double* k = c->dist;
    const int nd = c->n_dist;
    const double r2 = x * x + y * y, r4 = r2 * r2, r6 = r4 * r2;
    const double a1 = 2 * x * y, a2 = r2 + 2 * x * x, a3 = r2 + 2 * y * y;
    double cdist = 1 + k[0] * r2 + k[1] * r4, icdist2 = 1.0;
    if (nd > 4) cdist += k[4] * r6;
    if (nd > 5) icdist2 = 1.0 / (1 + k[5] * r2 + k[6] * r4 + k[7] * r6);
    xd = x * cdist * icdist2 + k[2] * a1 + k[3] * a2;
    yd = y * cdist * icdist2 + k[2] * a3 + k[3] * a1;
    if (nd > 8) {
      xd += k[8] * r2 + k[9] * r4;
      yd += k[10] * r2 + k[11] * r4;
    }
  }
  uv[0] = xd * c->fx + c->cx;
  uv[1] = yd * c->fy + c->cy;
}

/* Camera::project, PINHOLE branch (Camera.cpp:648-653) */
void oo_pinhole_project(const oo_pinhole* c, const double X[3], double uv[2]) {
  double xy[2];
  oo_pinhole_world_to_undist(c, X, xy);
  oo_pinhole_distort(c, xy, uv);
}

/* Camera::undistort (Camera.cpp:1018-1094) */
void oo_pinhole_undistort(const oo_pinhole* c, const double uv[2], double out[2]) {
  const double u = uv[0], v = uv[1];
  double x = (u - c->cx) / c->fx, y = (v - c->cy) / c->fy;
  out[0] = x;
  out[1] = y;
  if (is_distorted(c)) {
    const double* k = c->dist;
    const int nd = c->n_dist;
    const double x0 = x, y0 = y;
    double err = DBL_MAX;
    int iter = 0;
    while (err > 1e-5 && iter < 50) {
      const double r2 = x * x + y * y;
      const double a1 = 2 * x * y, a2 = r2 + 2 * x * x, a3 = r2 + 2 * y * y;
      double icdist, dX, dY, p[2], q[2];
      if (nd == 4)
        icdist = 1 / (1 + (k[1] * r2 + k[0]) * r2);
      else if (nd == 5)
        icdist = 1 / (1 + ((k[4] * r2 + k[1]) * r2 + k[0]) * r2);
      else
        icdist = (1 + ((k[7] * r2 + k[6]) * r2 + k[5]) * r2) /
                 (1 + ((k[4] * r2 + k[1]) * r2 + k[0]) * r2);
      if (icdist < 0) {
        out[0] = (u - c->cx) / c->fx;
        out[1] = (v - c->cy) / c->fy;
        break;
      }
      dX = k[2] * a1 + k[3] * a2;
      dY = k[2] * a3 + k[3] * a1;
      if (nd > 8) {
        dX += k[8] * r2 + k[9] * r2 * r2;
        dY += k[10] * r2 + k[11] * r2 * r2;
      }
      x = (x0 - dX) * icdist;
      y = (y0 - dY) * icdist;
      out[0] = x;
      out[1] = y;
      p[0] = x;
      p[1] = y;
      oo_pinhole_distort(c, p, q);
      err = sqrt((q[0] - u) * (q[0] - u) + (q[1] - v) * (q[1] - v));
      ++iter;
    }
  }
}

/* Camera::pinholeLine (Camera.cpp:1096-1108) after undistort */
void oo_pinhole_los(const oo_pinhole* c, const double uv[2], double L[6]) {
  double xy[2], p[3], d[3], nrm;
  int i;
  oo_pinhole_undistort(c, uv, xy);
  for (i = 0; i < 3; ++i)
    p[i] = c->Rinv[3 * i] * xy[0] + c->Rinv[3 * i + 1] * xy[1] + c->Rinv[3 * i + 2] * 1.0;
  for (i = 0; i < 3; ++i) p[i] = p[i] + c->Tinv[i];
  for (i = 0; i < 3; ++i) d[i] = p[i] - c->Tinv[i];
  nrm = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (i = 0; i < 3; ++i) {
    L[i] = c->Tinv[i];
    L[3 + i] = d[i] / nrm;
  }
}

/* Camera::polyProject (Camera.cpp:969-990) */
void oo_poly_project(const oo_poly* c, const double X[3], double uv[2]) {
  double su = 0, sv = 0;
  int i, j;
  for (i = 0; i < c->n_coeff; ++i) {
    double a = c->u[4 * i], b = c->v[4 * i];
    for (j = 1; j < 4; ++j) {
      a *= pow(X[j - 1], c->u[4 * i + j]);
      b *= pow(X[j - 1], c->v[4 * i + j]);
    }
    su += a;
    sv += b;
  }
  uv[0] = su;
  uv[1] = sv;
}

/* myMATH::internal::gaussForward / gaussBackward, n = 3 (inc/libMath/myMATH.h:183-289) */
static void gauss_inverse3(const double A[9], double R[9]) {
  double u[9], b[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, maxrow[3];
  int idx[3], x, y, it, i;
  for (i = 0; i < 9; ++i) u[i] = A[i];
  for (x = 0; x < 3; ++x) {
    double m = u[3 * x];
    if (u[3 * x + 1] > m) m = u[3 * x + 1];
    if (u[3 * x + 2] > m) m = u[3 * x + 2];
    idx[x] = x;
    maxrow[x] = m;
  }
  for (y = 0; y < 2; ++y) {
    double maxp = 0;
    int t = 0, tmp;
    for (x = y; x < 3; ++x) {
      const double piv = fabs(u[3 * idx[x] + y] / maxrow[idx[x]]);
      if (piv > maxp) {
        maxp = piv;
        t = x;
      }
    }
    tmp = idx[t];
    idx[t] = idx[y];
    idx[y] = tmp;
    for (x = y + 1; x < 3; ++x) {
      const double m = u[3 * idx[x] + y] / u[3 * idx[y] + y];
      u[3 * idx[x] + y] = m;
      for (it = y + 1; it < 3; ++it) u[3 * idx[x] + it] -= m * u[3 * idx[y] + it];
    }
  }
  for (i = 0; i < 9; ++i) R[i] = b[i];
  for (it = 0; it < 3; ++it) {
    for (y = 0; y < 2; ++y)
      for (x = y + 1; x < 3; ++x) b[3 * idx[x] + it] -= u[3 * idx[x] + y] * b[3 * idx[y] + it];
    R[6 + it] = b[3 * idx[2] + it] / u[3 * idx[2] + 2];
    for (x = 1; x > -1; --x) {
      double z = b[3 * idx[x] + it];
      for (y = x + 1; y < 3; ++y) z -= u[3 * idx[x] + y] * R[3 * y + it];
      R[3 * x + it] = z / u[3 * idx[x] + x];
    }
  }
}

/* myMATH::triangulation (src/srcMath/myMATH.cpp:357-419); -1 where it throws. */
int oo_triangulate(const double* L, int k, double out[4]) {
  double M[9] = {0}, b[3] = {0}, Mi[9], X[3], e = 0.0;
  int i, r, q;
  for (i = 0; i < k; ++i) {
    const double* p = L + 6 * i;
    const double nx = p[3], ny = p[4], nz = p[5];
    double t[9];
    t[0] = 1 - nx * nx;
    t[1] = -nx * ny;
    t[2] = -nx * nz;
    t[3] = -nx * ny;
    t[4] = 1 - ny * ny;
    t[5] = -ny * nz;
    t[6] = -nx * nz;
    t[7] = -ny * nz;
    t[8] = 1 - nz * nz;
    for (r = 0; r < 3; ++r) b[r] = b[r] + (t[3 * r] * p[0] + t[3 * r + 1] * p[1] + t[3 * r + 2] * p[2]);
    for (q = 0; q < 9; ++q) M[q] = M[q] + t[q];
  }
  gauss_inverse3(M, Mi);
  for (r = 0; r < 3; ++r) X[r] = Mi[3 * r] * b[0] + Mi[3 * r + 1] * b[1] + Mi[3 * r + 2] * b[2];
  for (i = 0; i < k; ++i) {
    const double* p = L + 6 * i;
    const double d0 = X[0] - p[0], d1 = X[1] - p[1], d2 = X[2] - p[2];
    const double nrm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    const double dt = d0 * p[3] + d1 * p[4] + d2 * p[5];
    double h = nrm * nrm - dt * dt;
    if (h < 0.0 && h >= -1e-8)
      h = 0.0;
    else if (h < -1e-8)
      return -1;
    else
      h = sqrt(h);
    e += h * h;
  }
  out[0] = X[0];
  out[1] = X[1];
  out[2] = X[2];
  out[3] = sqrt(e / k);
  return 0;
}

/* OTF::getOTFParam (src/srcSTB/OTF.cpp:273-338), linspace (myMATH.cpp:9-33),
 * triLinearInterp (myMATH.cpp:131-214). table: [4][n_cam][nx*ny*nz]. */
void oo_otf_param(int nx, int ny, int nz, const double bd[6], const double* table, int n_cam,
                  int cam, const double X[3], double out[5]) {
  const int n[3] = {nx, ny, nz};
  const int ng = nx * ny * nz, nyz = ny * nz;
  double p[3], lo[3], hi[3], t[3], res[4];
  int id[3], k, q, g[8];
  for (k = 0; k < 3; ++k) {
    const double mn = bd[2 * k], mx = bd[2 * k + 1];
    const double d = (mx - mn) / (n[k] - 1);
    int i;
    p[k] = X[k] < mn ? mn : X[k];
    p[k] = p[k] > mx ? mx : p[k];
    i = (int)floor((p[k] - mn) / d);
    i = i < 0 ? 0 : i;
    i = i > n[k] - 2 ? n[k] - 2 : i;
    id[k] = i;
    lo[k] = mn + d * i;
    hi[k] = mn + d * (i + 1);
    t[k] = (p[k] - lo[k]) / (hi[k] - lo[k]);
    t[k] = t[k] < 0.0 ? 0.0 : (t[k] > 1.0 ? 1.0 : t[k]);
  }
  g[0] = id[0] * nyz + id[1] * nz + id[2];
  g[1] = (id[0] + 1) * nyz + id[1] * nz + id[2];
  g[2] = (id[0] + 1) * nyz + id[1] * nz + id[2] + 1;
  g[3] = id[0] * nyz + id[1] * nz + id[2] + 1;
  g[4] = id[0] * nyz + (id[1] + 1) * nz + id[2];
  g[5] = (id[0] + 1) * nyz + (id[1] + 1) * nz + id[2];
  g[6] = (id[0] + 1) * nyz + (id[1] + 1) * nz + id[2] + 1;
  g[7] = id[0] * nyz + (id[1] + 1) * nz + id[2] + 1;
  for (q = 0; q < 4; ++q) {
    const double* tb = table + ((int64_t)q * n_cam + cam) * ng;
    const double c00 = tb[g[0]] * (1 - t[0]) + tb[g[1]] * t[0];
    const double c01 = tb[g[3]] * (1 - t[0]) + tb[g[2]] * t[0];
    const double c10 = tb[g[4]] * (1 - t[0]) + tb[g[5]] * t[0];
    const double c11 = tb[g[7]] * (1 - t[0]) + tb[g[6]] * t[0];
    const double c0 = c00 * (1 - t[1]) + c10 * t[1];
    const double c1 = c01 * (1 - t[1]) + c11 * t[1];
    res[q] = c0 * (1 - t[2]) + c1 * t[2];
  }
  out[0] = res[0];
  out[1] = res[1];
  out[2] = res[2];
  out[3] = cos(res[3]);
  out[4] = sin(res[3]);
}

/* Shake::calROIBound (src/srcSTB/Shake.cpp:246-277) */
static int roi_bound(int H, int W, double cx, double cy, double dx, double dy, int r[4]) {
  int width, height;
  if (H <= 0 || W <= 0 || dx <= 0.0 || dy <= 0.0 || cx <= 0 || cy <= 0 || cx >= W || cy >= H)
    return 0;
  width = (int)round(2.0 * dx);
  height = (int)round(2.0 * dy);
  r[2] = (int)round(cx - (width - 1) / 2.0);
  r[0] = (int)round(cy - (height - 1) / 2.0);
  r[3] = r[2] + width;
  r[1] = r[0] + height;
  if (r[0] < 0) r[0] = 0;
  if (r[2] < 0) r[2] = 0;
  if (r[1] > H) r[1] = H;
  if (r[3] > W) r[3] = W;
  return !(r[1] < r[0] || r[3] < r[2]);
}

/* Shake::calResidueImage (Shake.cpp:165-244) for one camera: min-fusion of
 * orig - Gaussian projection (TracerShakeStrategy::gaussIntensity, Shake.cpp:901-916)
 * over each object's window; clamp != 0 is the output_ipr clamp at 0.
 * uv: n_obj x 2 centres on this camera; otf5: n_obj x 5 (a, b, c, cos, sin). */
void oo_residual(double* res, const double* orig, int H, int W, int64_t n_obj, const double* uv,
                 const double* o5, double r_px, int clamp) {
  int64_t i;
  for (i = 0; i < (int64_t)H * W; ++i) res[i] = orig[i];
  for (i = 0; i < n_obj; ++i) {
    int R[4], r, c;
    if (!roi_bound(H, W, uv[2 * i], uv[2 * i + 1], r_px, r_px, R)) continue;
    for (r = R[0]; r < R[1]; ++r)
      for (c = R[2]; c < R[3]; ++c) {
        const double* o = o5 + 5 * i;
        const double dx = c - uv[2 * i], dy = r - uv[2 * i + 1];
        const double xx = dx * o[3] + dy * o[4];
        const double yy = -dx * o[4] + dy * o[3];
        double p = o[0] * exp(-(o[1] * xx * xx + o[2] * yy * yy));
        double* rr;
        double cand;
        p = p > 0.0 ? p : 0.0;
        if (p == 0.0) continue;
        rr = &res[(int64_t)r * W + c];
        cand = orig[(int64_t)r * W + c] - p;
        if (cand < *rr) *rr = cand;
        if (clamp && *rr < 0) *rr = 0.0;
      }
  }
}
