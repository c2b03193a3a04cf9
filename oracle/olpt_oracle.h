/*
 * Test infrastructure only -- the CPU oracle's C restatement of the reference
 * (OpenLPT) hot-path arithmetic.  Plain C99 in FP64, compiled without FMA
 * contraction (oracle/Makefile), each function citing the reference lines it
 * restates.  Checked against the reference's golden vectors and against the
 * reference compiled from source (tests/test_oracle.py).  The product never
 * links it.
 */
#ifndef OLPT_ORACLE_H
#define OLPT_ORACLE_H
#include <stdint.h>

typedef struct {
  double fx, fy, cx, cy;
  int n_dist;       /* coefficients given */
  double dist[12];
  double R[9], T[3], Rinv[9], Tinv[3];
} oo_pinhole;

typedef struct {
  int n_coeff;
  int ref_plane; /* 1 = X, 2 = Y, 3 = Z */
  double plane[2];
  const double* u; /* n_coeff x 4 */
  const double* v;
} oo_poly;

int64_t oo_find_peaks(const double* img, int H, int W, double min_int, double* out_xy,
                      int64_t cap);
void oo_pinhole_project(const oo_pinhole* c, const double xyz[3], double uv[2]);
void oo_pinhole_world_to_undist(const oo_pinhole* c, const double xyz[3], double xy[2]);
void oo_pinhole_distort(const oo_pinhole* c, const double xy[2], double uv[2]);
void oo_pinhole_undistort(const oo_pinhole* c, const double uv[2], double xy[2]);
void oo_pinhole_los(const oo_pinhole* c, const double uv[2], double line6[6]);
void oo_poly_project(const oo_poly* c, const double xyz[3], double uv[2]);
int oo_triangulate(const double* lines6, int k, double out4[4]);
void oo_otf_param(int nx, int ny, int nz, const double bound[6], const double* table, int n_cam,
                  int cam, const double xyz[3], double out5[5]);
void oo_residual(double* res, const double* orig, int H, int W, int64_t n_obj,
                 const double* uv, const double* otf5, double r_px, int clamp);

#endif
