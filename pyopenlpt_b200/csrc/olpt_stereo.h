// Stereo matching: host-side types shared by the device driver (stereo.cu) and the
// host-side candidate ordering / greedy prune (stereo_host.cpp).
#pragma once
#include <cstdint>
#include <vector>

namespace olpt {

struct SmParams {
  int match_cam_count;
  int idmap_cell_px;
  double tol_2d_px;
  double tol_3d_mm;
  double limit[6];
};

// Candidate set after checkMatch, sorted by ids (StereoMatch.cpp:153-156), and the
// prune selection (StereoMatch.cpp:631-980).
// After the device prune the arrays stay on the device (the context's prune
// workspace) until a caller asks for them (on_device; stereo_result_to_host).
struct StereoResult {
  int n_cam = 0;
  int ref_cam = -1;
  int64_t M = 0;               // candidates
  bool on_device = false;      // ids / e / X / selected not yet downloaded
  std::vector<int> ids;        // M x n_cam, -1 = camera unused
  std::vector<double> e;       // e_check
  std::vector<double> X;       // M x 3, triangulated position (camera order)
  std::vector<char> selected;  // M
};

void sort_candidates(StereoResult& r);
void prune_candidates(StereoResult& r, const std::vector<int>& det_counts,
                      const std::vector<int>& active);
// The greedy of pruneMatch over candidates in greedy order: g_pts G x n global point
// indices (g_cnt used), their percentile and e_check; sel[i] = 1 for kept ones.
void greedy_select(int64_t G, int n, const int* g_pts, const uint8_t* g_cnt, const double* g_pct,
                   const double* g_e, int64_t total_points, char* sel);

}  // namespace olpt
