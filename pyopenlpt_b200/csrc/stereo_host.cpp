// Host half of stereo matching: canonical candidate order and the greedy prune.
//
// StereoMatch::pruneMatch (src/srcSTB/StereoMatch.cpp:631-980) is an
// order-dependent greedy whose comparators use a relative tolerance and are not a
// strict weak ordering; the ranks it produces depend on the exact merge sequence of
// libstdc++'s std::stable_sort.  It is a short serial pass over an already small
// candidate list, so it runs here, with the same std::stable_sort over the same
// comparators, which keeps the selection identical to the reference's.  All
// numerical work (detection, lines of sight, strip search, triangulation) stays on
// the device.
#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <utility>
#include <vector>

#include "olpt_stereo.h"

namespace olpt {

void sort_candidates(StereoResult& r) {
  const int n = r.n_cam;
  const size_t M = r.e.size();
  std::vector<size_t> ord(M);
  std::iota(ord.begin(), ord.end(), 0);
  const int* ids = r.ids.data();
  std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
    return std::lexicographical_compare(ids + a * n, ids + a * n + n, ids + b * n, ids + b * n + n);
  });
  std::vector<int> ids2(r.ids.size());
  std::vector<double> e2(M), X2(3 * M);
  for (size_t i = 0; i < M; ++i) {
    const size_t j = ord[i];
    std::copy(ids + j * n, ids + j * n + n, ids2.begin() + i * n);
    e2[i] = r.e[j];
    X2[3 * i] = r.X[3 * j];
    X2[3 * i + 1] = r.X[3 * j + 1];
    X2[3 * i + 2] = r.X[3 * j + 2];
  }
  r.ids.swap(ids2);
  r.e.swap(e2);
  r.X.swap(X2);
}

void prune_candidates(StereoResult& r, const std::vector<int>& det_counts,
                      const std::vector<int>& active) {
  const size_t M = r.e.size();
  const int n_cams = r.n_cam;
  r.selected.assign(M, 0);
  if (M == 0) return;
  const double rtol = 1e-9, atol = 1e-12;
  auto eq_eps = [&](double a, double b) {
    const double s = std::max(std::fabs(a), std::fabs(b));
    return std::fabs(a - b) <= (s * rtol + atol);
  };
  const double swap_pct_margin = 1e-12, swap_err_margin = 1e-12;
  const std::vector<double>& e_checks = r.e;

  std::vector<size_t> cam_offsets(n_cams + 1, 0);
  for (int c = 0; c < n_cams; ++c) cam_offsets[c + 1] = cam_offsets[c] + det_counts[c];
  const size_t total_points = cam_offsets.back();

  // Step 1: flat 2D point indices per candidate
  std::vector<std::vector<size_t>> flats(M);
  for (size_t j = 0; j < M; ++j) {
    auto& lf = flats[j];
    for (int c = 0; c < n_cams; ++c) {
      if (!active[c]) continue;
      const int pid = r.ids[j * n_cams + c];
      if (pid < 0 || pid >= det_counts[c]) continue;
      lf.push_back(cam_offsets[c] + (size_t)pid);
    }
  }
  // Step 2: reverse index
  std::vector<std::vector<int>> p2c(total_points);
  for (size_t j = 0; j < M; ++j)
    for (size_t f : flats[j]) p2c[f].push_back((int)j);
  // Step 3: percentile scores
  std::vector<double> pct_sum(M, 0.0);
  std::vector<int> pct_count(M, 0);
  for (size_t f = 0; f < total_points; ++f) {
    const auto& idxs = p2c[f];
    if (idxs.empty()) continue;
    std::vector<std::pair<double, int>> pool;
    pool.reserve(idxs.size());
    for (int j : idxs)
      if (std::isfinite(e_checks[j])) pool.emplace_back(e_checks[j], j);
    const int n = (int)pool.size();
    if (n == 0) continue;
    if (n == 1) {
      pct_sum[pool[0].second] += 0.0;
      pct_count[pool[0].second] += 1;
      continue;
    }
    std::stable_sort(pool.begin(), pool.end(), [&](const auto& A, const auto& B) {
      if (!eq_eps(A.first, B.first)) return A.first < B.first;
      return A.second < B.second;
    });
    int k = 0;
    while (k < n) {
      int k0 = k, k1 = k + 1;
      while (k1 < n && eq_eps(pool[k1].first, pool[k0].first)) ++k1;
      const double avg_rank = 0.5 * (double)(k0 + (k1 - 1));
      const double denom = (double)(n - 1);
      const double pct = (denom > 0.0) ? (avg_rank / denom) : 0.0;
      for (int t = k0; t < k1; ++t) {
        pct_sum[pool[t].second] += pct;
        pct_count[pool[t].second] += 1;
      }
      k = k1;
    }
  }
  std::vector<double> pct_score(M, std::numeric_limits<double>::infinity());
  for (size_t j = 0; j < M; ++j)
    if (pct_count[j] > 0) pct_score[j] = pct_sum[j] / (double)pct_count[j];
  // Step 4: order by (pct, e_check, index)
  std::vector<int> order(M);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int aj, int bj) {
    const double pa = pct_score[aj], pb = pct_score[bj];
    const bool af = std::isfinite(pa), bf = std::isfinite(pb);
    if (af && bf) {
      if (!eq_eps(pa, pb)) return pa < pb;
    } else if (af) {
      return true;
    } else if (bf) {
      return false;
    }
    const double ea = e_checks[aj], eb = e_checks[bj];
    const bool aef = std::isfinite(ea), bef = std::isfinite(eb);
    if (aef && bef) {
      if (!eq_eps(ea, eb)) return ea < eb;
    } else if (aef) {
      return true;
    } else if (bef) {
      return false;
    }
    return aj < bj;
  });
  // Step 5: greedy exclusive ownership with local replacement
  std::vector<int> owner(total_points, -1);
  std::vector<char>& selected = r.selected;
  auto place = [&](int cand) {
    for (size_t f : flats[cand]) owner[f] = cand;
    selected[cand] = 1;
  };
  auto clear_owner_of = [&](int cand) {
    for (size_t f : flats[cand])
      if (owner[f] == cand) owner[f] = -1;
    selected[cand] = 0;
  };
  for (int j : order) {
    if (!std::isfinite(pct_score[j]) || !std::isfinite(e_checks[j])) continue;
    const auto& fl = flats[j];
    if (fl.empty()) continue;
    bool conflict = false;
    for (size_t f : fl)
      if (owner[f] != -1) {
        conflict = true;
        break;
      }
    if (!conflict) {
      place(j);
      continue;
    }
    std::vector<int> S;
    for (size_t f : fl) {
      const int o = owner[f];
      if (o == -1) continue;
      if (std::find(S.begin(), S.end(), o) == S.end()) S.push_back(o);
    }
    if (S.empty()) {
      place(j);
      continue;
    }
    double avg_pct = 0.0, avg_err = 0.0;
    int cnt = 0;
    for (int o : S) {
      const double po = pct_score[o], eo = e_checks[o];
      if (!std::isfinite(po) || !std::isfinite(eo)) continue;
      avg_pct += po;
      avg_err += eo;
      ++cnt;
    }
    if (cnt == 0) continue;
    avg_pct /= (double)cnt;
    avg_err /= (double)cnt;
    const double pj = pct_score[j], ej = e_checks[j];
    const bool better_pct = (!eq_eps(pj, avg_pct)) && ((pj + swap_pct_margin) < avg_pct);
    const bool tie_better = eq_eps(pj, avg_pct) && (!eq_eps(ej, avg_err)) &&
                            ((ej + swap_err_margin) < avg_err);
    if (better_pct || tie_better) {
      for (int o : S) clear_owner_of(o);
      place(j);
    }
  }
}

}  // namespace olpt
