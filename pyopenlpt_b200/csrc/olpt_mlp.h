// Learned proposal: the MLP that maps per-camera residual patches of a candidate
// to a 3D correction and a ghost logit (mlp.cu), and its device state.
//
// Input (per candidate, for a rig of C cameras): for each camera an 11 x 11 patch of
// the augmented residual max(0, residual + own projection) around the rounded
// projection, divided by the candidate's OTF amplitude on that camera (row-major,
// camera-major: C x 121); then the 2 C sub-pixel offsets (u - round(u), v - round(v));
// then a constant 1.  Stored bf16, zero-padded to MlpDims::in_pad columns.
// Layers: in -> 256 -> 256 -> 256 (GELU) -> 4 (dx, dy, dz in units of out_scale_mm,
// ghost logit).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace olpt {

constexpr int kMlpPatch = 11, kMlpArea = kMlpPatch * kMlpPatch;
constexpr int kMlpHid = 256, kMlpOut = 4;
constexpr int kMlpMaxCams = 8;

// Network geometry for a rig of `cams` cameras (2..8): input cams * 121 patch values +
// 2 * cams sub-pixel offsets + 1, zero-padded to a multiple of 64 (the GEMM's K slice);
// flat f32 parameter layout (row-major weights, [out][in]): W1, b1, W2, b2, W3, b3, W4, b4.
// For 4 cameras: 493 inputs (512 padded), 259,076 parameters.
struct MlpDims {
  int cams = 0, in = 0, in_pad = 0;
  int64_t off_w1 = 0, off_b1 = 0, off_w2 = 0, off_b2 = 0, off_w3 = 0, off_b3 = 0, off_w4 = 0,
          off_b4 = 0, params = 0;
};
inline MlpDims mlp_dims(int cams) {
  MlpDims d;
  d.cams = cams;
  d.in = cams * kMlpArea + 2 * cams + 1;
  d.in_pad = (d.in + 63) / 64 * 64;
  d.off_w1 = 0;
  d.off_b1 = d.off_w1 + (int64_t)kMlpHid * d.in;
  d.off_w2 = d.off_b1 + kMlpHid;
  d.off_b2 = d.off_w2 + (int64_t)kMlpHid * kMlpHid;
  d.off_w3 = d.off_b2 + kMlpHid;
  d.off_b3 = d.off_w3 + (int64_t)kMlpHid * kMlpHid;
  d.off_w4 = d.off_b3 + kMlpHid;
  d.off_b4 = d.off_w4 + (int64_t)kMlpOut * kMlpHid;
  d.params = d.off_b4 + kMlpOut;
  return d;
}

// Learned-shake settings (olpt_learned_params).
struct LearnedParams {
  int enable = 0;
  double out_scale_mm = 0.05;     // network output unit for dx, dy, dz
  double ghost_logit = 2.0;       // candidates above are dropped before shaking
  int refine_loops = 1;           // plain shake iterations after the correction
  double refine_width_mm = 0.02;  // their first shake width
  double fallback_residual = 0;   // per-object residue (normalised by a^2) above which
                                  // the object reruns the full plain shake
};

}  // namespace olpt
