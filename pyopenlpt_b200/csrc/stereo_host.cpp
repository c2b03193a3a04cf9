// Host half of stereo matching: canonical candidate order and the greedy prune.
//
// StereoMatch::pruneMatch (src/srcSTB/StereoMatch.cpp:631-980) is an
// order-dependent greedy whose comparators use a relative tolerance; such a
// comparator is not a strict weak ordering in general, and then the ranks depend on
// the exact merge sequence of libstdc++'s std::stable_sort.  The reference's result
// is kept bit-for-bit as follows:
//  * per 2D point, the candidate pools are small: they are sorted with the same
//    std::stable_sort and comparator as the reference, from the same input order;
//  * the global order of the candidates by (percentile, e_check, index) is only
//    needed for the candidates the greedy can take (finite percentile and e_check).
//    The values are grouped into tolerance classes (runs of neighbours within the
//    tolerance in sorted order).  When every class is within the tolerance end to
//    end, the tolerance relation is an equivalence on the data, the comparator is a
//    strict weak ordering made total by the index, and stable_sort's output is the
//    unique sorted order by (class, class, index): that order is produced here by
//    parallel sorts.  Otherwise the reference's std::stable_sort runs as is.
// Point -> candidate lists are built in parallel; every per-point pool is put into
// ascending candidate order, the order in which the reference appends to it, and
// each candidate sums its per-point percentiles in ascending point order, as the
// reference accumulates pct_sum.  All numerical geometry (detection, lines of sight,
// strip search, triangulation) stays on the device.
#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <utility>
#include <vector>

#include "olpt_stereo.h"

namespace olpt {
namespace {

// Sorts by a strict total order on all host threads (libstdc++ parallel mode).
template <class It, class Cmp>
void par_sort(It b, It e, Cmp cmp) {
  __gnu_parallel::sort(b, e, cmp);
}

}  // namespace

void sort_candidates(StereoResult& r) {
  const int n = r.n_cam;
  const size_t M = r.e.size();
  const int* ids = r.ids.data();
  // ids are compared lexicographically (camera 0 first, -1 < any id); with
  // 21 bits per camera the key of up to 6 cameras fits in 128 bits.  Candidate id
  // sets are unique, so the order is total.
  int max_id = 0;
  for (size_t q = 0; q < r.ids.size(); ++q) max_id = std::max(max_id, ids[q]);
  std::vector<int> ord(M);
  if (n <= 6 && max_id < (1 << 21) - 2) {
    std::vector<std::pair<unsigned __int128, int>> key(M);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < (int64_t)M; ++j) {
      unsigned __int128 k = 0;
      for (int c = 0; c < n; ++c) k = (k << 21) | (unsigned __int128)(ids[j * n + c] + 1);
      key[j] = {k, (int)j};
    }
    par_sort(key.begin(), key.end(), [](const auto& a, const auto& b) {
      return a.first < b.first || (a.first == b.first && a.second < b.second);
    });
    for (size_t i = 0; i < M; ++i) ord[i] = key[i].second;
  } else {
    std::iota(ord.begin(), ord.end(), 0);
    par_sort(ord.begin(), ord.end(), [&](int a, int b) {
      const bool lt = std::lexicographical_compare(ids + (size_t)a * n, ids + (size_t)a * n + n,
                                                   ids + (size_t)b * n, ids + (size_t)b * n + n);
      const bool gt = std::lexicographical_compare(ids + (size_t)b * n, ids + (size_t)b * n + n,
                                                   ids + (size_t)a * n, ids + (size_t)a * n + n);
      return lt || (!gt && a < b);
    });
  }
  std::vector<int> ids2(r.ids.size());
  std::vector<double> e2(M), X2(3 * M);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)M; ++i) {
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

// StereoMatch::pruneMatch step 5 (StereoMatch.cpp:880-975): greedy exclusive
// ownership of 2D points with local replacement, over G candidates already in greedy
// order (all with finite percentile and e_check).  Per point the owner's position and
// its (percentile, e_check) are cached, so the loop reads the candidates in order and
// touches other candidates only to release them.
void greedy_select(int64_t G, int n, const int* g_pts, const uint8_t* g_cnt, const double* g_pct,
                   const double* g_e, int64_t total_points, char* sel) {
  const double rtol = 1e-9, atol = 1e-12;
  auto eq_eps = [&](double a, double b) {
    const double s = std::max(std::fabs(a), std::fabs(b));
    return std::fabs(a - b) <= (s * rtol + atol);
  };
  const double swap_pct_margin = 1e-12, swap_err_margin = 1e-12;
  struct Own {
    int o;
    double pct, e;
  };
  std::vector<Own> owner(total_points, Own{-1, 0.0, 0.0});
  auto place = [&](int64_t i) {
    for (int k = 0; k < g_cnt[i]; ++k) owner[g_pts[i * n + k]] = Own{(int)i, g_pct[i], g_e[i]};
    sel[i] = 1;
  };
  auto clear_owner_of = [&](int o) {
    for (int k = 0; k < g_cnt[o]; ++k) {
      Own& w = owner[g_pts[(int64_t)o * n + k]];
      if (w.o == o) w.o = -1;
    }
    sel[o] = 0;
  };
  std::vector<int> S_buf(std::max(n, 1));
  int* S = S_buf.data();
  constexpr int64_t kAhead = 16;  // owner entries of later candidates are prefetched
  for (int64_t i = 0; i < G; ++i) {
    if (i + kAhead < G)
      for (int k = 0; k < g_cnt[i + kAhead]; ++k)
        __builtin_prefetch(&owner[g_pts[(i + kAhead) * n + k]]);
    const int cnt_i = g_cnt[i];
    if (cnt_i == 0) continue;
    const int* P = &g_pts[i * n];
    int ns = 0;
    double avg_pct = 0.0, avg_err = 0.0;
    for (int k = 0; k < cnt_i; ++k) {
      const Own& w = owner[P[k]];
      if (w.o == -1) continue;
      bool seen = false;
      for (int t = 0; t < ns; ++t) seen |= (S[t] == w.o);
      if (!seen) {
        S[ns++] = w.o;
        avg_pct += w.pct;  // owners are always finite in both
        avg_err += w.e;
      }
    }
    if (ns == 0) {
      place(i);
      continue;
    }
    avg_pct /= (double)ns;
    avg_err /= (double)ns;
    const double pj = g_pct[i], ej = g_e[i];
    const bool better_pct = (!eq_eps(pj, avg_pct)) && ((pj + swap_pct_margin) < avg_pct);
    const bool tie_better = eq_eps(pj, avg_pct) && (!eq_eps(ej, avg_err)) &&
                            ((ej + swap_err_margin) < avg_err);
    if (better_pct || tie_better) {
      for (int t = 0; t < ns; ++t) clear_owner_of(S[t]);
      place(i);
    }
  }
}

void prune_candidates(StereoResult& r, const std::vector<int>& det_counts,
                      const std::vector<int>& active) {
  const size_t M = r.e.size();
  const int n = r.n_cam;
  r.selected.assign(M, 0);
  if (M == 0) return;
  const double rtol = 1e-9, atol = 1e-12;
  auto eq_eps = [&](double a, double b) {
    const double s = std::max(std::fabs(a), std::fabs(b));
    return std::fabs(a - b) <= (s * rtol + atol);
  };
  const std::vector<double>& e_checks = r.e;

  std::vector<int64_t> cam_offsets(n + 1, 0);
  for (int c = 0; c < n; ++c) cam_offsets[c + 1] = cam_offsets[c] + det_counts[c];
  const int64_t total_points = cam_offsets.back();

  // Step 1: the candidate's 2D points (global point index, ascending = camera order),
  // fixed width n; slot j*n+k
  std::vector<int> fl(M * n, -1);
  std::vector<uint8_t> fcnt(M);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)M; ++j) {
    int k = 0;
    for (int c = 0; c < n; ++c) {
      if (!active[c]) continue;
      const int pid = r.ids[j * n + c];
      if (pid < 0 || pid >= det_counts[c]) continue;
      fl[j * n + k++] = (int)(cam_offsets[c] + pid);
    }
    fcnt[j] = (uint8_t)k;
  }
  // Step 2: point -> (candidate, slot) lists
  std::vector<std::atomic<int>> pcount(total_points + 1);
  for (auto& a : pcount) a.store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)M; ++j)
    for (int k = 0; k < fcnt[j]; ++k) pcount[fl[j * n + k] + 1].fetch_add(1, std::memory_order_relaxed);
  std::vector<int> poff(total_points + 1, 0);
  for (int64_t f = 0; f < total_points; ++f) poff[f + 1] = poff[f] + pcount[f + 1].load();
  for (int64_t f = 0; f < total_points; ++f) pcount[f].store(poff[f], std::memory_order_relaxed);
  std::vector<int> pc_slot(poff[total_points]);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)M; ++j)
    for (int k = 0; k < fcnt[j]; ++k) {
      const int pos = pcount[fl[j * n + k]].fetch_add(1, std::memory_order_relaxed);
      pc_slot[pos] = (int)(j * n + k);
    }
  // Step 3: percentile of every (point, candidate) pair, written to the slot
  std::vector<double> slot_pct(M * n, 0.0);
  std::vector<char> slot_used(M * n, 0);
#pragma omp parallel
  {
    struct Item {
      double e;
      int j, slot;
    };
    std::vector<Item> pool;
#pragma omp for schedule(dynamic, 256)
    for (int64_t f = 0; f < total_points; ++f) {
      const int b = poff[f], e = poff[f + 1];
      if (b == e) continue;
      // the reference appends candidates to the point's pool in ascending j
      std::sort(pc_slot.begin() + b, pc_slot.begin() + e);
      pool.clear();
      for (int q = b; q < e; ++q) {
        const int slot = pc_slot[q];
        const int j = slot / n;
        const double ej = e_checks[j];
        if (std::isfinite(ej)) pool.push_back({ej, j, slot});
      }
      const int np = (int)pool.size();
      if (np == 0) continue;
      if (np == 1) {
        slot_pct[pool[0].slot] = 0.0;
        slot_used[pool[0].slot] = 1;
        continue;
      }
      std::stable_sort(pool.begin(), pool.end(), [&](const Item& A, const Item& B) {
        if (!eq_eps(A.e, B.e)) return A.e < B.e;
        return A.j < B.j;
      });
      int k = 0;
      while (k < np) {
        int k0 = k, k1 = k + 1;
        while (k1 < np && eq_eps(pool[k1].e, pool[k0].e)) ++k1;
        const double avg_rank = 0.5 * (double)(k0 + (k1 - 1));
        const double denom = (double)(np - 1);
        const double pct = (denom > 0.0) ? (avg_rank / denom) : 0.0;
        for (int t = k0; t < k1; ++t) {
          slot_pct[pool[t].slot] = pct;
          slot_used[pool[t].slot] = 1;
        }
        k = k1;
      }
    }
  }
  // per candidate: sum over its points in ascending point order
  std::vector<double> pct_score(M, std::numeric_limits<double>::infinity());
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)M; ++j) {
    double sum = 0.0;
    int cnt = 0;
    for (int k = 0; k < fcnt[j]; ++k)
      if (slot_used[j * n + k]) {
        sum += slot_pct[j * n + k];
        ++cnt;
      }
    if (cnt > 0) pct_score[j] = sum / (double)cnt;
  }

  // Step 4: the greedy order of the candidates it can take, by (pct, e_check, index)
  std::vector<int> order;
  {
    // tolerance classes of the finite values; false when a class is wider than the
    // tolerance end to end
    auto classes = [&](const std::vector<int>& items, const std::vector<double>& val,
                       std::vector<int>& cls) -> int {
      std::vector<std::pair<double, int>> v(items.size());
      for (size_t i = 0; i < items.size(); ++i) v[i] = {val[items[i]], items[i]};
      par_sort(v.begin(), v.end(), [](const auto& a, const auto& b) {
        return a.first < b.first || (a.first == b.first && a.second < b.second);
      });
      int c = -1;
      double first = 0.0, prev = 0.0;
      for (size_t i = 0; i < v.size(); ++i) {
        const double x = v[i].first;
        if (i == 0 || !eq_eps(prev, x)) {
          ++c;
          first = x;
        } else if (!eq_eps(first, x)) {
          return -1;
        }
        cls[v[i].second] = c;
        prev = x;
      }
      return c + 1;
    };
    std::vector<int> fin_pct;  // finite percentile (the comparator's consistent part)
    for (size_t j = 0; j < M; ++j)
      if (std::isfinite(pct_score[j])) fin_pct.push_back((int)j);
    std::vector<int> fin_both;
    for (int j : fin_pct)
      if (std::isfinite(e_checks[j])) fin_both.push_back(j);
    std::vector<int> pcls(M, 0), ecls(M, 0);
    const int n_pc = classes(fin_pct, pct_score, pcls);
    const int n_ec = n_pc < 0 ? -1 : classes(fin_both, e_checks, ecls);
    if (n_pc >= 0 && n_ec >= 0) {
      std::vector<std::pair<uint64_t, int>> key(fin_both.size());
      for (size_t i = 0; i < fin_both.size(); ++i) {
        const int j = fin_both[i];
        key[i] = {((uint64_t)pcls[j] << 32) | (uint64_t)ecls[j], j};
      }
      par_sort(key.begin(), key.end(), [](const auto& a, const auto& b) {
        return a.first < b.first || (a.first == b.first && a.second < b.second);
      });
      order.resize(key.size());
      for (size_t i = 0; i < key.size(); ++i) order[i] = key[i].second;
    } else {
      // the reference's sort, verbatim in its comparator
      std::vector<int> all(M);
      std::iota(all.begin(), all.end(), 0);
      std::stable_sort(all.begin(), all.end(), [&](int aj, int bj) {
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
      for (int j : all)
        if (std::isfinite(pct_score[j]) && std::isfinite(e_checks[j])) order.push_back(j);
    }
  }

  // Step 5: greedy exclusive ownership with local replacement, over the candidates
  // gathered in greedy order (owner holds the position in that order)
  const int64_t G = (int64_t)order.size();
  std::vector<int> g_pts((size_t)G * n);
  std::vector<uint8_t> g_cnt(G);
  std::vector<double> g_pct(G), g_e(G);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < G; ++i) {
    const int j = order[i];
    g_cnt[i] = fcnt[j];
    for (int k = 0; k < n; ++k) g_pts[i * n + k] = fl[(size_t)j * n + k];
    g_pct[i] = pct_score[j];
    g_e[i] = e_checks[j];
  }
  std::vector<char> sel(G, 0);
  greedy_select(G, n, g_pts.data(), g_cnt.data(), g_pct.data(), g_e.data(), total_points,
                sel.data());
  for (int64_t i = 0; i < G; ++i)
    if (sel[i]) r.selected[order[i]] = 1;
}

}  // namespace olpt
