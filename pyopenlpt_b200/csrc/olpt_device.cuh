// Device-side data layout and FP64 geometry for the OpenLPT hot path on sm_100a.
//
// Bit-exactness contract: every function here evaluates the same IEEE-754
// double operations, in the same order, as the reference C++ code it cites.
// The library is compiled with --fmad=false so that no multiply-add is
// contracted (the reference builds in ISO C++20 mode, -ffp-contract=off, on an
// x86-64 baseline without FMA).  Division and sqrt are IEEE-rounded on both
// sides.  Transcendentals (acos, sin, exp, pow) are not bit-identical between
// glibc and CUDA; where they feed a decision the caller documents it.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define OLPT_MAX_CAM 8
#define OLPT_MAX_POLY 32

namespace olpt {

enum CamType : int { CAM_PINHOLE = 0, CAM_POLYNOMIAL = 1 };

// One camera, flattened.  Matches the parameter set of Camera::loadParameters
// (src/srcMath/Camera.cpp:19-158).
struct CamDev {
  int type;
  int n_row, n_col;
  int is_active;
  // pinhole
  double fx, fy, cx, cy;  // cam_mtx(0,0), (1,1), (0,2), (1,2)
  int is_distorted, n_dist;
  double dist[12];
  double R[9], T[3], Rinv[9], Tinv[3];
  // polynomial
  int ref_plane;  // 1 = REF_X, 2 = REF_Y, 3 = REF_Z
  int n_coeff;
  int pow3;       // every exponent (of the model and its derivatives) is 0, 1, 2 or 3
  double plane[2];
  double ucoef[OLPT_MAX_POLY * 4];
  double vcoef[OLPT_MAX_POLY * 4];
  double ducoef[2 * OLPT_MAX_POLY * 4];
  double dvcoef[2 * OLPT_MAX_POLY * 4];
};

struct Line3 {
  double p[3];
  double u[3];
};

// ---------------------------------------------------------------- pinhole
// Camera::distort (Camera.cpp:913-966), returns pixel coordinates.
__device__ __forceinline__ void cam_distort(const CamDev& c, double x, double y, double& pu,
                                            double& pv) {
  double xd, yd;
  if (c.is_distorted) {
    const double* k = c.dist;
    double r2 = x * x + y * y;
    double r4 = r2 * r2;
    double r6 = r4 * r2;
    double a1 = 2 * x * y;
    double a2 = r2 + 2 * x * x;
    double a3 = r2 + 2 * y * y;
    double cdist = 1 + k[0] * r2 + k[1] * r4;
    if (c.n_dist > 4) cdist += k[4] * r6;
    double icdist2 = 1.0;
    if (c.n_dist > 5) icdist2 = 1.0 / (1 + k[5] * r2 + k[6] * r4 + k[7] * r6);
    xd = x * cdist * icdist2 + k[2] * a1 + k[3] * a2;
    yd = y * cdist * icdist2 + k[2] * a3 + k[3] * a1;
    if (c.n_dist > 8) {
      xd += k[8] * r2 + k[9] * r4;
      yd += k[10] * r2 + k[11] * r4;
    }
  } else {
    xd = x;
    yd = y;
  }
  pu = xd * c.fx + c.cx;
  pv = yd * c.fy + c.cy;
}

// Camera::worldToUndistImg + distort (Camera.cpp:648-690, 913-966).
__device__ __forceinline__ void pinhole_project(const CamDev& c, double X, double Y, double Z,
                                                double& u, double& v) {
  // Matrix<double>::operator* accumulates from 0 in column order (Matrix.hpp:392-406),
  // then operator+ adds T elementwise.
  double t0 = c.R[0] * X + c.R[1] * Y + c.R[2] * Z;
  double t1 = c.R[3] * X + c.R[4] * Y + c.R[5] * Z;
  double t2 = c.R[6] * X + c.R[7] * Y + c.R[8] * Z;
  t0 = t0 + c.T[0];
  t1 = t1 + c.T[1];
  t2 = t2 + c.T[2];
  double x = (t2 != 0.0) ? (t0 / t2) : t0;
  double y = (t2 != 0.0) ? (t1 / t2) : t1;
  cam_distort(c, x, y, u, v);
}

// Camera::undistort (Camera.cpp:1018-1094).
__device__ __forceinline__ void pinhole_undistort(const CamDev& c, double u, double v, double& ox,
                                                  double& oy) {
  double x = (u - c.cx) / c.fx;
  double y = (v - c.cy) / c.fy;
  ox = x;
  oy = y;
  if (!c.is_distorted) return;
  const double* k = c.dist;
  const double x0 = x, y0 = y;
  double err = 1.7976931348623157e308;
  int iter = 0;
  while (err > 1e-5 && iter < 50) {
    double r2 = x * x + y * y;
    double a1 = 2 * x * y;
    double a2 = r2 + 2 * x * x;
    double a3 = r2 + 2 * y * y;
    double icdist;
    if (c.n_dist == 4)
      icdist = 1 / (1 + (k[1] * r2 + k[0]) * r2);
    else if (c.n_dist == 5)
      icdist = 1 / (1 + ((k[4] * r2 + k[1]) * r2 + k[0]) * r2);
    else
      icdist = (1 + ((k[7] * r2 + k[6]) * r2 + k[5]) * r2) /
               (1 + ((k[4] * r2 + k[1]) * r2 + k[0]) * r2);
    if (icdist < 0) {
      ox = (u - c.cx) / c.fx;
      oy = (v - c.cy) / c.fy;
      break;
    }
    double dX = k[2] * a1 + k[3] * a2;
    double dY = k[2] * a3 + k[3] * a1;
    if (c.n_dist > 8) {
      dX += k[8] * r2 + k[9] * r2 * r2;
      dY += k[10] * r2 + k[11] * r2 * r2;
    }
    x = (x0 - dX) * icdist;
    y = (y0 - dY) * icdist;
    ox = x;
    oy = y;
    double pu, pv;
    cam_distort(c, x, y, pu, pv);
    double du = pu - u, dv = pv - v;
    err = sqrt(du * du + dv * dv);
    iter++;
  }
}

// myMATH::createUnitVector (myMATH.cpp:217-223) + Matrix::norm (Matrix.hpp:255-261).
__device__ __forceinline__ void unit_vector3(const double a[3], const double b[3], double o[3]) {
  double d0 = b[0] - a[0], d1 = b[1] - a[1], d2 = b[2] - a[2];
  double n = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  o[0] = d0 / n;
  o[1] = d1 / n;
  o[2] = d2 / n;
}

// Camera::pinholeLine (Camera.cpp:1096-1108).
__device__ __forceinline__ void pinhole_line(const CamDev& c, double x, double y, Line3& L) {
  double p[3];
  p[0] = c.Rinv[0] * x + c.Rinv[1] * y + c.Rinv[2] * 1.0;
  p[1] = c.Rinv[3] * x + c.Rinv[4] * y + c.Rinv[5] * 1.0;
  p[2] = c.Rinv[6] * x + c.Rinv[7] * y + c.Rinv[8] * 1.0;
  p[0] = p[0] + c.Tinv[0];
  p[1] = p[1] + c.Tinv[1];
  p[2] = p[2] + c.Tinv[2];
  L.p[0] = c.Tinv[0];
  L.p[1] = c.Tinv[1];
  L.p[2] = c.Tinv[2];
  unit_vector3(c.Tinv, p, L.u);
}

// ---------------------------------------------------------------- polynomial
// Integer powers are evaluated in double-double and rounded once, which gives
// the correctly rounded x^n (what glibc's pow returns in practice); other
// exponents use CUDA pow.
__device__ __forceinline__ double poly_pow(double x, double e) {
  if (e == 0.0) return 1.0;
  if (e == 1.0) return x;
  double r = rint(e);
  if (r == e && e > 0 && e <= 16) {
    int n = (int)e;
    double hi = x, lo = 0.0;
    for (int i = 1; i < n; ++i) {
      double p = hi * x;
      double pe = fma(hi, x, -p);
      double q = lo * x;
      double s = p + q;
      double se = (p - s) + q;
      hi = s;
      lo = se + pe;
      double t = hi + lo;
      lo = lo - (t - hi);
      hi = t;
    }
    return hi + lo;
  }
  return pow(x, e);
}

// The powers 0..3 of a point's coordinates, each the value poly_pow returns, so that
// a model whose exponents are all 0..3 (pow3) multiplies table entries instead of
// evaluating one power per term: the same factors in the same order.
__device__ __forceinline__ void poly_powers(const double P[3], double pw[3][4]) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    pw[j][0] = 1.0;
    pw[j][1] = P[j];
    pw[j][2] = poly_pow(P[j], 2.0);
    pw[j][3] = poly_pow(P[j], 3.0);
  }
}

// Camera::polyProject (Camera.cpp:969-990).
__device__ __forceinline__ void poly_project(const CamDev& c, double X, double Y, double Z,
                                             double& u, double& v) {
  const double P[3] = {X, Y, Z};
  double su = 0, sv = 0;
  if (c.pow3) {
    double pw[3][4];
    poly_powers(P, pw);
    for (int i = 0; i < c.n_coeff; ++i) {
      double uv = c.ucoef[4 * i];
      double vv = c.vcoef[4 * i];
#pragma unroll
      for (int j = 1; j < 4; ++j) {
        uv *= pw[j - 1][(int)c.ucoef[4 * i + j]];
        vv *= pw[j - 1][(int)c.vcoef[4 * i + j]];
      }
      su += uv;
      sv += vv;
    }
  } else {
    for (int i = 0; i < c.n_coeff; ++i) {
      double uv = c.ucoef[4 * i];
      double vv = c.vcoef[4 * i];
      for (int j = 1; j < 4; ++j) {
        uv *= poly_pow(P[j - 1], c.ucoef[4 * i + j]);
        vv *= poly_pow(P[j - 1], c.vcoef[4 * i + j]);
      }
      su += uv;
      sv += vv;
    }
  }
  u = su;
  v = sv;
}

// Camera::polyImgToWorld (Camera.cpp:1174-1283) with a deterministic start
// point (0.5, 0.5, 0.5) in place of the reference's rand() draw.
__device__ __forceinline__ void poly_img_to_world(const CamDev& c, double pu, double pv,
                                                  double plane, double P[3]) {
  P[0] = 0.5;
  P[1] = 0.5;
  P[2] = 0.5;
  P[c.ref_plane - 1] = plane;
  double err = 1.7976931348623157e308;
  int iter = 0;
  const int n = c.n_coeff;
  while (err > 1e-5 && iter < 50) {
    double j00 = 0, j01 = 0, j10 = 0, j11 = 0;
    double pw[3][4];
    if (c.pow3) poly_powers(P, pw);
    for (int i = 0; i < n; ++i) {
      double dudx = c.ducoef[4 * i], dudy = c.ducoef[4 * (i + n)];
      double dvdx = c.dvcoef[4 * i], dvdy = c.dvcoef[4 * (i + n)];
      for (int j = 1; j < 4; ++j) {
        if (c.pow3) {
          dudx *= pw[j - 1][(int)c.ducoef[4 * i + j]];
          dudy *= pw[j - 1][(int)c.ducoef[4 * (i + n) + j]];
          dvdx *= pw[j - 1][(int)c.dvcoef[4 * i + j]];
          dvdy *= pw[j - 1][(int)c.dvcoef[4 * (i + n) + j]];
        } else {
          dudx *= poly_pow(P[j - 1], c.ducoef[4 * i + j]);
          dudy *= poly_pow(P[j - 1], c.ducoef[4 * (i + n) + j]);
          dvdx *= poly_pow(P[j - 1], c.dvcoef[4 * i + j]);
          dvdy *= poly_pow(P[j - 1], c.dvcoef[4 * (i + n) + j]);
        }
      }
      j00 += dudx;
      j01 += dudy;
      j10 += dvdx;
      j11 += dvdy;
    }
    // myMATH::internal::detInverse, n == 2 (myMATH.h:227-250)
    double det = j00 * j11 - j01 * j10;
    if (fabs(det) < 1e-8) det = 1e-8;
    double i00 = j11 / det, i01 = -j01 / det, i10 = -j10 / det, i11 = j00 / det;
    double tu, tv;
    poly_project(c, P[0], P[1], P[2], tu, tv);
    double du = pu - tu, dv = pv - tv;
    double dx = i00 * du + i01 * dv;
    double dy = i10 * du + i11 * dv;
    if (c.ref_plane == 1) {
      P[1] += dx;
      P[2] += dy;
    } else if (c.ref_plane == 2) {
      P[0] += dx;
      P[2] += dy;
    } else {
      P[0] += dx;
      P[1] += dy;
    }
    err = sqrt(du * du + dv * dv);
    iter++;
  }
}

// ---------------------------------------------------------------- dispatch
// Camera::project (Camera.cpp:648-677).
__device__ __forceinline__ void cam_project(const CamDev& c, double X, double Y, double Z,
                                            double& u, double& v) {
  if (c.type == CAM_PINHOLE)
    pinhole_project(c, X, Y, Z, u, v);
  else
    poly_project(c, X, Y, Z, u, v);
}

// Camera::lineOfSight (Camera.cpp:996-1016; polyLineOfSight 1285-1294).
__device__ __forceinline__ void cam_los(const CamDev& c, double pu, double pv, Line3& L) {
  if (c.type == CAM_PINHOLE) {
    double x, y;
    pinhole_undistort(c, pu, pv, x, y);
    pinhole_line(c, x, y, L);
  } else {
    double P1[3], P2[3];
    poly_img_to_world(c, pu, pv, c.plane[0], P1);
    poly_img_to_world(c, pu, pv, c.plane[1], P2);
    L.p[0] = P1[0];
    L.p[1] = P1[1];
    L.p[2] = P1[2];
    unit_vector3(P1, P2, L.u);
  }
}

// StereoMatch::makeLine2DFromLOS3D (StereoMatch.cpp:1055-1068): image line of a
// 3D line of sight on camera c.  out = {pt.x, pt.y, unit.x, unit.y}.
__device__ __forceinline__ void los_to_line2d(const CamDev& c, const Line3& L, double out[4]) {
  double ax, ay, bx, by;
  cam_project(c, L.p[0], L.p[1], L.p[2], ax, ay);
  cam_project(c, L.p[0] + L.u[0], L.p[1] + L.u[1], L.p[2] + L.u[2], bx, by);
  double dx = bx - ax, dy = by - ay;
  double n = sqrt(dx * dx + dy * dy);
  out[0] = ax;
  out[1] = ay;
  out[2] = dx / n;
  out[3] = dy / n;
}

// ---------------------------------------------------------------- triangulation
// myMATH::internal::gaussForward/gaussBackward (myMATH.h:183-289) for n = 3,
// returning inverse(A) (gaussInverse, myMATH.h:291-301).
__device__ __forceinline__ void gauss_inverse3(const double A[9], double R[9]) {
  // Rows move physically instead of through an index permutation (same operations on
  // the same values, so the same result), which keeps every array in registers.
  double r[3][3], mr[3];
  int perm[3];
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    r[x][0] = A[3 * x];
    r[x][1] = A[3 * x + 1];
    r[x][2] = A[3 * x + 2];
    double m = r[x][0];
    if (r[x][1] > m) m = r[x][1];
    if (r[x][2] > m) m = r[x][2];
    mr[x] = m;
    perm[x] = x;
  }
#pragma unroll
  for (int y = 0; y < 2; ++y) {
    double maxp = 0;
    int t = 0;
#pragma unroll
    for (int x = y; x < 3; ++x) {
      const double piv = fabs(r[x][y] / mr[x]);
      if (piv > maxp) {
        maxp = piv;
        t = x;
      }
    }
    // swap positions y and t (t may be below y when no pivot is positive)
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      if (x == y || x != t) continue;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double tmp = r[x][k];
        r[x][k] = r[y][k];
        r[y][k] = tmp;
      }
      const double tm = mr[x];
      mr[x] = mr[y];
      mr[y] = tm;
      const int tp = perm[x];
      perm[x] = perm[y];
      perm[y] = tp;
    }
#pragma unroll
    for (int x = y + 1; x < 3; ++x) {
      const double m = r[x][y] / r[y][y];
      r[x][y] = m;
#pragma unroll
      for (int it = y + 1; it < 3; ++it) r[x][it] -= m * r[y][it];
    }
  }
  double pb[3][3];
#pragma unroll
  for (int x = 0; x < 3; ++x)
#pragma unroll
    for (int k = 0; k < 3; ++k) pb[x][k] = perm[x] == k ? 1.0 : 0.0;
#pragma unroll
  for (int it = 0; it < 3; ++it) {
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int x = y + 1; x < 3; ++x) pb[x][it] -= r[x][y] * pb[y][it];
    R[3 * 2 + it] = pb[2][it] / r[2][2];
#pragma unroll
    for (int x = 1; x > -1; --x) {
      double z = pb[x][it];
#pragma unroll
      for (int y = x + 1; y < 3; ++y) z -= r[x][y] * R[3 * y + it];
      R[3 * x + it] = z / r[x][x];
    }
  }
}

// myMATH::triangulation (myMATH.cpp:357-419).  Lines are given by pointers so
// callers can pass them in any (build or camera) order.  Returns false where the
// reference throws (h < -1e-8).
template <int MAXK>
__device__ __forceinline__ bool triangulate(const Line3* const* L, int n, double X[3],
                                            double& err) {
  double M[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double b[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i) {
    const double nx = L[i]->u[0], ny = L[i]->u[1], nz = L[i]->u[2];
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
    const double* p = L[i]->p;
    for (int r = 0; r < 3; ++r) {
      double s = t[3 * r] * p[0] + t[3 * r + 1] * p[1] + t[3 * r + 2] * p[2];
      b[r] = b[r] + s;
    }
    for (int q = 0; q < 9; ++q) M[q] = M[q] + t[q];
  }
  double Mi[9];
  gauss_inverse3(M, Mi);
  for (int r = 0; r < 3; ++r) X[r] = Mi[3 * r] * b[0] + Mi[3 * r + 1] * b[1] + Mi[3 * r + 2] * b[2];
  double e = 0.0;
  for (int i = 0; i < n; ++i) {
    double d0 = X[0] - L[i]->p[0], d1 = X[1] - L[i]->p[1], d2 = X[2] - L[i]->p[2];
    double nrm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    double dt = d0 * L[i]->u[0] + d1 * L[i]->u[1] + d2 * L[i]->u[2];
    double h = nrm * nrm - dt * dt;
    if (h < 0.0 && h >= -1e-8) {
      h = 0.0;
    } else if (h < -1e-8) {
      return false;
    } else {
      h = sqrt(h);
    }
    e += h * h;
  }
  err = sqrt(e / n);
  return true;
}

}  // namespace olpt
