// Device helpers of the shake shared with the learned proposal's feature kernel:
// ROI bounds (Shake::calROIBound), the Gaussian projection (gaussIntensity) and
// pixel loads of any image type.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/olpt.h"
#include "olpt_shake.h"

namespace olpt {

struct Rect {
  int rmin, rmax, cmin, cmax;  // [min, max)
};

// Shake::calROIBound (Shake.cpp:246-277)
__host__ __device__ __forceinline__ Rect roi_bound(int H, int W, double cx, double cy, double dx,
                                                   double dy) {
  Rect e{1, 0, 1, 0};
  if (H <= 0 || W <= 0 || dx <= 0.0 || dy <= 0.0 || cx <= 0 || cy <= 0 || cx >= W || cy >= H)
    return e;
  const int width = (int)round(2.0 * dx);
  const int height = (int)round(2.0 * dy);
  int cmin = (int)round(cx - (width - 1) / 2.0);
  int rmin = (int)round(cy - (height - 1) / 2.0);
  int cmax = cmin + width;
  int rmax = rmin + height;
  rmin = rmin > 0 ? rmin : 0;
  cmin = cmin > 0 ? cmin : 0;
  rmax = rmax < H ? rmax : H;
  cmax = cmax < W ? cmax : W;
  if (rmax < rmin || cmax < cmin) return e;
  return Rect{rmin, rmax, cmin, cmax};
}

__device__ __forceinline__ bool rect_empty(const Rect& r) {
  return r.rmax < r.rmin || r.cmax < r.cmin;
}

// TracerShakeStrategy::gaussIntensity (Shake.cpp:901-916)
template <typename Real>
__device__ __forceinline__ Real gauss(int col, int row, double u, double v, const Real* o) {
  const Real dx = (Real)((double)col - u);
  const Real dy = (Real)((double)row - v);
  const Real xx = dx * o[3] + dy * o[4];
  const Real yy = -dx * o[4] + dy * o[3];
  const Real val = o[0] * exp(-(o[1] * xx * xx + o[2] * yy * yy));
  return val > (Real)0 ? val : (Real)0;
}

template <typename T>
__device__ __forceinline__ double load_px(const unsigned char* base, int64_t pitch, int r, int c) {
  return (double)reinterpret_cast<const T*>(base + (int64_t)r * pitch)[c];
}

__device__ __forceinline__ double load_any(const PlaneView& p, int r, int c) {
  switch (p.dtype) {
    case OLPT_U8: return load_px<uint8_t>(p.p, p.pitch, r, c);
    case OLPT_U16: return load_px<uint16_t>(p.p, p.pitch, r, c);
    case OLPT_F32: return load_px<float>(p.p, p.pitch, r, c);
    default: return load_px<double>(p.p, p.pitch, r, c);
  }
}

}  // namespace olpt
