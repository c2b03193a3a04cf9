// Host half of stereo matching: canonical candidate order and the greedy prune.
//
// StereoMatch::pruneMatch (src/srcSTB/StereoMatch.cpp:631-980) is an
// order-dependent greedy whose comparators use a relative tolerance and are not a
// strict weak ordering; the ranks it produces depend on the exact merge sequence of
// libstdc++'s std::stable_sort.  It therefore runs here, calling the same
// std::stable_sort with the same comparators, which keeps the selection identical
// to the reference's.  The data layout is flat (CSR point -> candidate lists), and
// the per-point percentile pass runs on all host threads: every point writes its own
// slots, and each candidate then sums its slots in ascending point order -- the
// order in which the reference accumulates pct_sum -- so the floating-point sums are
// unchanged.  All numerical geometry (detection, lines of sight, strip search,
// triangulation) stays on the device.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
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
  const int* ids = r.ids.data();
  // ids are compared lexicographically (camera 0 first, -1 < any id); with
  // 21 bits per camera the key of up to 6 cameras fits in 128 bits.
  int max_id = 0;
  for (size_t q = 0; q < r.ids.size(); ++q) max_id = std::max(max_id, ids[q]);
  if (n <= 6 && max_id < (1 << 21) - 2) {
    std::vector<std::pair<unsigned __int128, uint32_t>> key(M);
    for (size_t j = 0; j < M; ++j) {
      unsigned __int128 k = 0;
      for (int c = 0; c < n; ++c) k = (k << 21) | (unsigned __int128)(ids[j * n + c] + 1);
      key[j] = {k, (uint32_t)j};
    }
    std::sort(key.begin(), key.end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t i = 0; i < M; ++i) ord[i] = key[i].second;
  } else {
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
      return std::lexicographical_compare(ids + a * n, ids + a * n + n, ids + b * n,
                                          ids + b * n + n);
    });
  }
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

  // Step 1: flat 2D point indices per candidate (ascending: camera order)
  std::vector<int> foff(M + 1, 0);
  std::vector<int64_t> flat;
  flat.reserve(M * n_cams);
  for (size_t j = 0; j < M; ++j) {
    for (int c = 0; c < n_cams; ++c) {
      if (!active[c]) continue;
      const int pid = r.ids[j * n_cams + c];
      if (pid < 0 || pid >= det_counts[c]) continue;
      flat.push_back((int64_t)(cam_offsets[c] + (size_t)pid));
    }
    foff[j + 1] = (int)flat.size();
  }
  // Step 2: point -> candidates (ascending j), with the slot of the point in the candidate
  std::vector<int> poff(total_points + 1, 0);
  for (int64_t f : flat) ++poff[f + 1];
  for (size_t f = 0; f < total_points; ++f) poff[f + 1] += poff[f];
  std::vector<int> pc_j(flat.size()), pc_slot(flat.size());
  {
    std::vector<int> cur(poff.begin(), poff.end() - 1);
    for (size_t j = 0; j < M; ++j)
      for (int q = foff[j]; q < foff[j + 1]; ++q) {
        const int64_t f = flat[q];
        pc_j[cur[f]] = (int)j;
        pc_slot[cur[f]] = q;
        ++cur[f];
      }
  }
  // Step 3: percentile of every (point, candidate) pair, written to the candidate's slot
  std::vector<double> slot_pct(flat.size(), 0.0);
  std::vector<char> slot_used(flat.size(), 0);
#pragma omp parallel
  {
    std::vector<std::pair<double, int>> pool;
    std::vector<int> pool_slot;
#pragma omp for schedule(dynamic, 256)
    for (int64_t f = 0; f < (int64_t)total_points; ++f) {
      const int b = poff[f], e = poff[f + 1];
      if (b == e) continue;
      pool.clear();
      for (int q = b; q < e; ++q) {
        const int j = pc_j[q];
        const double ej = e_checks[j];
        if (std::isfinite(ej)) pool.emplace_back(ej, j);
      }
      const int n = (int)pool.size();
      if (n == 0) continue;
      auto slot_of = [&](int j) {
        for (int q = b; q < e; ++q)
          if (pc_j[q] == j) return pc_slot[q];
        return -1;
      };
      if (n == 1) {
        const int s = slot_of(pool[0].second);
        slot_pct[s] = 0.0;
        slot_used[s] = 1;
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
          const int s = slot_of(pool[t].second);
          slot_pct[s] = pct;
          slot_used[s] = 1;
        }
        k = k1;
      }
    }
  }
  // per candidate: sum over its points in ascending point order (the reference's order)
  std::vector<double> pct_score(M, std::numeric_limits<double>::infinity());
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)M; ++j) {
    double sum = 0.0;
    int cnt = 0;
    for (int q = foff[j]; q < foff[j + 1]; ++q)
      if (slot_used[q]) {
        sum += slot_pct[q];
        ++cnt;
      }
    if (cnt > 0) pct_score[j] = sum / (double)cnt;
  }
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
    for (int q = foff[cand]; q < foff[cand + 1]; ++q) owner[flat[q]] = cand;
    selected[cand] = 1;
  };
  auto clear_owner_of = [&](int cand) {
    for (int q = foff[cand]; q < foff[cand + 1]; ++q)
      if (owner[flat[q]] == cand) owner[flat[q]] = -1;
    selected[cand] = 0;
  };
  std::vector<int> S;
  for (int j : order) {
    if (!std::isfinite(pct_score[j]) || !std::isfinite(e_checks[j])) continue;
    if (foff[j] == foff[j + 1]) continue;
    bool conflict = false;
    for (int q = foff[j]; q < foff[j + 1]; ++q)
      if (owner[flat[q]] != -1) {
        conflict = true;
        break;
      }
    if (!conflict) {
      place(j);
      continue;
    }
    S.clear();
    for (int q = foff[j]; q < foff[j + 1]; ++q) {
      const int o = owner[flat[q]];
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
