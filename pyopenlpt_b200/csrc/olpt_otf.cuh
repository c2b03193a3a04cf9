// OTF table lookup on the device: OTF::getOTFParam (src/srcSTB/OTF.cpp:273-338)
// with myMATH::linspace grid nodes (myMATH.cpp:9-33) and myMATH::triLinearInterp
// (myMATH.cpp:131-214), evaluated in FP64 in the reference's operation order.
#pragma once
#include "olpt_device.cuh"

namespace olpt {

struct OtfView {
  int nx, ny, nz, n_grid, n_cam;
  double bmin[3], bmax[3], d[3];
  const double* table;  // [4][n_cam][n_grid]
  // every alpha entry is +0.0: the interpolated angle is then +0.0 and its cosine and
  // sine are exactly 1 and +0 (the reference's values), so they are not evaluated
  int alpha_zero;
};

__device__ __forceinline__ double otf_lerp8(const double* v, double xd, double yd, double zd) {
  // v: c000, c100, c101, c001, c010, c110, c111, c011 (OTF.cpp:312-317 order)
  double c00 = v[0] * (1 - xd) + v[1] * xd;
  double c01 = v[3] * (1 - xd) + v[2] * xd;
  double c10 = v[4] * (1 - xd) + v[5] * xd;
  double c11 = v[7] * (1 - xd) + v[6] * xd;
  double c0 = c00 * (1 - yd) + c10 * yd;
  double c1 = c01 * (1 - yd) + c11 * yd;
  return c0 * (1 - zd) + c1 * zd;
}

// out: a, b, c, cos(alpha), sin(alpha)
__device__ __forceinline__ void otf_param(const OtfView& o, int cam, double X, double Y, double Z,
                                          double out[5]) {
  const double P[3] = {X, Y, Z};
  const int n[3] = {o.nx, o.ny, o.nz};
  double p[3], lo[3], hi[3];
  int id[3];
  for (int k = 0; k < 3; ++k) {
    p[k] = fmin(fmax(P[k], o.bmin[k]), o.bmax[k]);
    int i = (int)floor((p[k] - o.bmin[k]) / o.d[k]);
    i = i < 0 ? 0 : i;
    i = i > n[k] - 2 ? n[k] - 2 : i;
    id[k] = i;
    const double delta = (o.bmax[k] - o.bmin[k]) / (n[k] - 1);
    lo[k] = o.bmin[k] + delta * i;
    hi[k] = o.bmin[k] + delta * (i + 1);
  }
  double t[3];
  for (int k = 0; k < 3; ++k) {
    double v = (p[k] - lo[k]) / (hi[k] - lo[k]);
    t[k] = fmax(0.0, fmin(1.0, v));
  }
  const int nyz = o.ny * o.nz;
  const int x0 = id[0], y0 = id[1], z0 = id[2];
  const int g[8] = {x0 * nyz + y0 * o.nz + z0,             x0 * nyz + nyz + y0 * o.nz + z0,
                    x0 * nyz + nyz + y0 * o.nz + z0 + 1,   x0 * nyz + y0 * o.nz + z0 + 1,
                    x0 * nyz + (y0 + 1) * o.nz + z0,       x0 * nyz + nyz + (y0 + 1) * o.nz + z0,
                    x0 * nyz + nyz + (y0 + 1) * o.nz + z0 + 1, x0 * nyz + (y0 + 1) * o.nz + z0 + 1};
  double res[4];
  const int nq = o.alpha_zero ? 3 : 4;
  for (int q = 0; q < nq; ++q) {
    const double* tab = o.table + ((size_t)q * o.n_cam + cam) * o.n_grid;
    double v[8];
    for (int k = 0; k < 8; ++k) v[k] = tab[g[k]];
    res[q] = otf_lerp8(v, t[0], t[1], t[2]);
  }
  out[0] = res[0];
  out[1] = res[1];
  out[2] = res[2];
  if (o.alpha_zero) {
    out[3] = 1.0;
    out[4] = 0.0;
  } else {
    out[3] = cos(res[3]);
    out[4] = sin(res[3]);
  }
}

}  // namespace olpt
