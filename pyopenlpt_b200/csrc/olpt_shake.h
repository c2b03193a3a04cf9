// Shake: parameter block, kernel views and device workspace (shake.cu).
#pragma once
#include <cstddef>
#include <cstdint>

#include "olpt_otf.cuh"

namespace olpt {

struct ShakeParams {
  double shake_width;
  double shakewidth_min;
  int n_shake_loop;
  double thred_ghost;
  int ratio_augimg;
  double radius_obj;
  double tol_3d_mm;
  int precision;  // 0 = FP32 residual / OTF / line-search sums, 1 = FP64
};

struct PlaneView {
  unsigned char* p;
  int64_t pitch;  // bytes
  int H, W;
  int dtype;
};

struct ShakeView {
  int n_cam;
  const CamDev* cams;
  OtfView otf;
  double r_px, ratio;
  int roi_area;          // augmented ROI pixels (side^2)
  int win_w, win_h;      // projection window
  int exact_sums;        // FP64 path: row-major sequential sums
  int tile_base[OLPT_MAX_CAM];
  int n_tiles;
  PlaneView orig[OLPT_MAX_CAM];  // current images (u8/u16/f32/f64)
  PlaneView res[OLPT_MAX_CAM];   // residual planes (Real)
  size_t smem_per_warp, off_dd, off_otf, off_uv;
};

}  // namespace olpt
