// Learned proposal: the MLP that maps per-camera residual patches of a candidate
// to a 3D correction and a ghost logit (mlp.cu), and its device state.
//
// Input (kIn = 493 per candidate): for each of 4 cameras an 11 x 11 patch of the
// augmented residual max(0, residual + own projection) around the rounded
// projection, divided by the candidate's OTF amplitude on that camera (row-major,
// camera-major: 4 x 121); then the 8 sub-pixel offsets (u - round(u), v - round(v))
// per camera; then a constant 1.  Stored bf16, zero-padded to kInPad columns.
// Layers: kIn -> 256 -> 256 -> 256 (GELU) -> 4 (dx, dy, dz in units of out_scale_mm,
// ghost logit).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace olpt {

constexpr int kMlpCams = 4, kMlpPatch = 11;
constexpr int kMlpIn = kMlpCams * kMlpPatch * kMlpPatch + 2 * kMlpCams + 1;  // 493
constexpr int kMlpInPad = 512, kMlpHid = 256, kMlpOut = 4;

// flat f32 parameter layout (row-major weights, [out][in])
constexpr int64_t kOffW1 = 0;
constexpr int64_t kOffB1 = kOffW1 + (int64_t)kMlpHid * kMlpIn;
constexpr int64_t kOffW2 = kOffB1 + kMlpHid;
constexpr int64_t kOffB2 = kOffW2 + (int64_t)kMlpHid * kMlpHid;
constexpr int64_t kOffW3 = kOffB2 + kMlpHid;
constexpr int64_t kOffB3 = kOffW3 + (int64_t)kMlpHid * kMlpHid;
constexpr int64_t kOffW4 = kOffB3 + kMlpHid;
constexpr int64_t kOffB4 = kOffW4 + (int64_t)kMlpOut * kMlpHid;
constexpr int64_t kMlpParams = kOffB4 + kMlpOut;  // 259,076

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
