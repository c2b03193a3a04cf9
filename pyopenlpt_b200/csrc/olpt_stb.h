// Shake-the-Box state: parameters, host-side track containers (the reference's
// four std::deque<Track>, inc/libSTB/STB.h:60-66) and the device views used by
// the per-frame kernels in stb.cu.
#pragma once
#include <deque>
#include <string>
#include <vector>

#include "olpt_device.cuh"

namespace olpt {

struct IprParams;

// STBParam + PFParam + the axis limit and frame range of BasicSetting
// (inc/libSTB/Config.h:17-69, 170-180).
struct StbParams {
  int frame_start = 0, frame_end = 0;
  int n_initial_frames = 4;
  double radius_search_obj = 0.0;    // mm
  double radius_search_track = 0.0;  // mm
  double limit[6] = {0, 0, 0, 0, 0, 0};  // x_min, x_max, y_min, y_max, z_min, z_max
  int pf_n[3] = {2, 2, 2};
  double pf_r = 0.0;
  int pf_nbin[3] = {11, 11, 11};
  int pf_smooth = 1;
  double pf_sigma[3] = {1.0, 1.0, 1.0};
  std::string output_path;  // empty: no files written
};

// One track: points in frame order (Track::_obj3d_list centres, _t_list).
struct TrackH {
  std::vector<double> xyz;  // 3 per point
  std::vector<int> t;
  size_t size() const { return t.size(); }
};

struct StbView {
  int n_cam;
  const CamDev* cams;
  double limit[6];
};

// Predictive-field grid (PredField::setGrid, src/srcSTB/PredField.cpp:153-176).
struct PfView {
  int nx, ny, nz;
  double lo[3], hi[3], d[3];
  int nbin[3], nbin_tot;
  double m[3], c[3];
  double r;
};

}  // namespace olpt
