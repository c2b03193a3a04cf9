// Device half of the candidate ordering and of StereoMatch::pruneMatch
// (src/srcSTB/StereoMatch.cpp:153-156, 631-980).
//
// The candidates of checkMatch stay on the device:
//  1. sort by ids (lexicographic, camera 0 first; -1 < any id) with a stable LSD
//     radix sort of packed 64-bit keys;
//  2. every candidate's 2D points (global point index per active camera, camera
//     order) and the point -> candidate lists (CSR, ascending candidate);
//  3. per 2D point (one warp): the percentile of every candidate in the point's pool.
//     The reference stable-sorts the pool with a tolerance comparator (rtol 1e-9,
//     atol 1e-12) and averages ranks over runs of tolerance-equal e_check.  When the
//     runs are tolerance-equal end to end (checked here), the comparator is a strict
//     weak ordering on the pool, the runs are the tolerance classes, and every rank
//     follows from the class boundaries of the exactly sorted pool;
//  4. per candidate: the mean percentile over its points, summed in point order;
//  5. the greedy order by (percentile, e_check, index) of the candidates the greedy
//     can take: tolerance classes of the percentiles, then of e_check inside every
//     percentile class (computed and checked the same way over the sorted values),
//     and a radix sort by class;
//  6. the greedy: parallel rounds of the in-order greedy independent set, checked
//     against the replacement rule (greedy_device); the sequential loop on the host
//     when a replacement would fire.
// Whenever a check fails (a tolerance class wider than the tolerance, a key wider
// than 64 bits) the caller falls back to the host implementation, which keeps the
// reference's std::stable_sort.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "olpt_ctx.cuh"
#include "olpt_prune.h"
#include "olpt_scan.cuh"

namespace olpt {
namespace {

inline int nblk(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------- radix sort
constexpr int kRsThreads = 256;
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsThreads * kRsItems;

__global__ void __launch_bounds__(kRsThreads) rs_hist_kernel(const uint64_t* key, int n, int shift,
                                                             int* hist, int n_blocks) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int tile = blockIdx.x * kRsTile;
#pragma unroll
  for (int k = 0; k < kRsItems; ++k) {
    const int i = tile + k * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(int)((key[i] >> shift) & 255u)], 1);
  }
  __syncthreads();
  hist[threadIdx.x * n_blocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one 8-bit digit: items of a tile are ranked in index order
// (round k holds items k*256 .. k*256+255 of the tile, warps in order, lanes in order).
__global__ void __launch_bounds__(kRsThreads) rs_scatter_kernel(const uint64_t* key, const int* val,
                                                                int n, int shift, const int* offs,
                                                                int n_blocks, uint64_t* key_out,
                                                                int* val_out) {
  __shared__ int base[256];
  __shared__ int whist[kRsThreads / 32][256];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  base[threadIdx.x] = offs[threadIdx.x * n_blocks + blockIdx.x];
  const int tile = blockIdx.x * kRsTile;
  for (int k = 0; k < kRsItems; ++k) {
    for (int q = threadIdx.x; q < (kRsThreads / 32) * 256; q += kRsThreads) (&whist[0][0])[q] = 0;
    __syncthreads();
    const int i = tile + k * kRsThreads + threadIdx.x;
    const bool ok = i < n;
    const uint64_t kk = ok ? key[i] : 0ull;
    const int vv = ok ? val[i] : 0;
    const int d = ok ? (int)((kk >> shift) & 255u) : 256 + lane;  // invalid: unique per lane
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (ok && lane == __ffs(peers) - 1) whist[w][d] = __popc(peers);
    __syncthreads();
    {
      const int dd = threadIdx.x;
      int run = base[dd];
      for (int ww = 0; ww < kRsThreads / 32; ++ww) {
        const int t = whist[ww][dd];
        whist[ww][dd] = run;
        run += t;
      }
      base[dd] = run;
    }
    __syncthreads();
    if (ok) {
      const int pos = whist[w][d] + rank;
      key_out[pos] = kk;
      val_out[pos] = vv;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- candidates
__device__ __forceinline__ bool eq_eps(double a, double b) {
  const double s = fmax(fabs(a), fabs(b));
  return fabs(a - b) <= (s * 1e-9 + 1e-12);
}

__global__ void id_keys_kernel(const int* ids, int M, int n, int bits, uint64_t* key, int* val) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  uint64_t k = 0;
  for (int c = 0; c < n; ++c) k = (k << bits) | (uint64_t)(uint32_t)(ids[(int64_t)j * n + c] + 1);
  key[j] = k;
  val[j] = j;
}

// Word w of the candidates' id keys, for a lexicographic sort in several 64-bit
// passes: the ids of cameras [w * per, (w + 1) * per) of candidate perm[i] (i when perm
// is null), packed most significant first; val[i] = the candidate.
__global__ void word_keys_kernel(const int* ids, int M, int n, int bits, int per, int w,
                                 const int* perm, uint64_t* key, int* val) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const int j = perm ? perm[i] : i;
  const int c1 = min(n, (w + 1) * per);
  uint64_t k = 0;
  for (int c = w * per; c < c1; ++c)
    k = (k << bits) | (uint64_t)(uint32_t)(ids[(int64_t)j * n + c] + 1);
  key[i] = k;
  val[i] = j;
}

__global__ void gather_cand_kernel(const int* perm, int M, int n, const int* ids, const double* e,
                                   const double* X, int* ids_s, double* e_s, double* X_s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const int j = perm[i];
  for (int c = 0; c < n; ++c) ids_s[(int64_t)i * n + c] = ids[(int64_t)j * n + c];
  e_s[i] = e[j];
  for (int d = 0; d < 3; ++d) X_s[3 * (int64_t)i + d] = X[3 * (int64_t)j + d];
}

// The candidate's 2D points (global index, camera order) in slots j*n .. j*n+n-1.
__global__ void flat_kernel(const int* ids, int M, int n, PruneView pv, int* fl, int* key,
                            uint8_t* fcnt) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  int k = 0;
  for (int c = 0; c < n; ++c) {
    const int pid = ids[(int64_t)j * n + c];
    if (!pv.active[c] || pid < 0 || pid >= pv.count[c]) continue;
    const int f = pv.offset[c] + pid;
    fl[(int64_t)j * n + k] = f;
    key[(int64_t)j * n + k] = f;
    ++k;
  }
  for (int q = k; q < n; ++q) {
    fl[(int64_t)j * n + q] = -1;
    key[(int64_t)j * n + q] = -1;
  }
  fcnt[j] = (uint8_t)k;
}

// Per 2D point, one warp: percentile of each candidate of the point's pool.  Pools
// of up to kPoolMax candidates live in shared memory, larger ones in the global
// scratch (indexed by their position in the point -> candidate list).
constexpr int kPctWarps = 4;
constexpr int kPoolMax = 512;
struct PoolSmem {
  double e[kPoolMax];
  int j[kPoolMax];
  int slot[kPoolMax];
  int ord[kPoolMax];
  int cls[kPoolMax];
  int start[kPoolMax];
};
struct PoolScratch {  // global, one entry per (point, candidate) pair
  double* e;
  int *j, *slot, *ord, *cls, *start;
};

__global__ void __launch_bounds__(kPctWarps * 32) pct_kernel(const int* pstart, const int* items,
                                                             int n_points, int n, const double* e,
                                                             PoolScratch gs, double* slot_pct,
                                                             uint8_t* slot_used, int* flag) {
  extern __shared__ __align__(16) unsigned char pool_raw[];
  PoolSmem& S = reinterpret_cast<PoolSmem*>(pool_raw)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int f = blockIdx.x * kPctWarps + (threadIdx.x >> 5);
  if (f >= n_points) return;
  const int b = pstart[f], end = pstart[f + 1];
  const unsigned lt = (1u << lane) - 1u;
  int np = 0;
  for (int base = b; base < end; base += 32) {
    const int q = base + lane;
    const bool fin = q < end && isfinite(e[items[q] / n]);
    np += __popc(__ballot_sync(0xffffffffu, fin));
  }
  if (np == 0) return;
  const bool big = np > kPoolMax;
  double* pe = big ? gs.e + b : S.e;
  int* pj = big ? gs.j + b : S.j;
  int* pslot = big ? gs.slot + b : S.slot;
  int* pord = big ? gs.ord + b : S.ord;
  int* pcls = big ? gs.cls + b : S.cls;
  int* pstart2 = big ? gs.start + b : S.start;
  int cnt = 0;
  for (int base = b; base < end; base += 32) {
    const int q = base + lane;
    const bool valid = q < end;
    const int slot = valid ? items[q] : 0;
    const int j = slot / n;
    const double ev = valid ? e[j] : 0.0;
    const bool fin = valid && isfinite(ev);
    const unsigned m = __ballot_sync(0xffffffffu, fin);
    const int pos = cnt + __popc(m & lt);
    if (fin) {
      pe[pos] = ev;
      pj[pos] = j;
      pslot[pos] = slot;
    }
    cnt += __popc(m);
  }
  __syncwarp();
  if (np == 1) {
    if (lane == 0) {
      slot_pct[pslot[0]] = 0.0;
      slot_used[pslot[0]] = 1;
    }
    return;
  }
  // exact order by (e, j)
  for (int i = lane; i < np; i += 32) {
    const double ei = pe[i];
    const int ji = pj[i];
    int r = 0;
    for (int k = 0; k < np; ++k) r += (pe[k] < ei || (pe[k] == ei && pj[k] < ji)) ? 1 : 0;
    pord[r] = i;
  }
  __syncwarp();
  // tolerance classes over the sorted values
  int run = -1;
  for (int p0 = 0; p0 < np; p0 += 32) {
    const int p = p0 + lane;
    const bool valid = p < np;
    const bool newc = valid && (p == 0 || !eq_eps(pe[pord[p - 1]], pe[pord[p]]));
    const unsigned m = __ballot_sync(0xffffffffu, newc);
    const int cid = run + __popc(m & (lt | (1u << lane)));
    if (valid) pcls[p] = cid;
    if (newc) pstart2[cid] = p;
    run += __popc(m);
  }
  __syncwarp();
  const int n_cls = run + 1;
  bool bad = false;
  for (int p = lane; p < np; p += 32) {
    const int c = pcls[p];
    const int s0 = pstart2[c];
    const int s1 = (c + 1 < n_cls) ? pstart2[c + 1] - 1 : np - 1;
    if (!eq_eps(pe[pord[s0]], pe[pord[p]])) bad = true;
    const double avg_rank = 0.5 * (double)(s0 + s1);
    const double pct = avg_rank / (double)(np - 1);
    const int slot = pslot[pord[p]];
    slot_pct[slot] = pct;
    slot_used[slot] = 1;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flag, 2);
}

__global__ void pct_score_kernel(const uint8_t* fcnt, int M, int n, const double* slot_pct,
                                 const uint8_t* slot_used, double* pct_score) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  double sum = 0.0;
  int cnt = 0;
  for (int k = 0; k < fcnt[j]; ++k) {
    const int64_t s = (int64_t)j * n + k;
    if (slot_used[s]) {
      sum += slot_pct[s];
      ++cnt;
    }
  }
  pct_score[j] = cnt > 0 ? sum / (double)cnt : __longlong_as_double(0x7ff0000000000000LL);
}

// flags for the two candidate sets: finite percentile; finite percentile and e_check
__global__ void finite_flags_kernel(const double* pct, const double* e, int M, int* f_pct,
                                    int* f_both) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const bool a = isfinite(pct[j]);
  f_pct[j] = a ? 1 : 0;
  f_both[j] = (a && isfinite(e[j])) ? 1 : 0;
}

__device__ __forceinline__ uint64_t ordered_bits(double v) {
  if (v == 0.0) v = 0.0;
  const uint64_t b = (uint64_t)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | (1ull << 63));
}

// compacted list (ascending index) with value keys
__global__ void compact_keys_kernel(const int* flag, const int* pos, int M, const double* val,
                                    uint64_t* key, int* idx) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M || !flag[j]) return;
  key[pos[j]] = ordered_bits(val[j]);
  idx[pos[j]] = j;
}

// A class starts where the value leaves the tolerance of its predecessor, or where
// the group (the percentile class, when given) changes.
__global__ void newclass_kernel(const int* idx, int m, const double* val, const int* grp,
                                int* newc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const bool split = p == 0 || (grp && grp[idx[p - 1]] != grp[idx[p]]) ||
                     !eq_eps(val[idx[p - 1]], val[idx[p]]);
  newc[p] = split ? 1 : 0;
}

__global__ void group_keys_kernel(const int* idx, int m, const int* grp, uint64_t* key) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  key[p] = (uint64_t)grp[idx[p]];
}

__global__ void class_start_kernel(const int* newc, const int* excl, int m, int* start) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m || !newc[p]) return;
  start[excl[p]] = p;
}

// class of every candidate; flag when a class is not tolerance-equal end to end
__global__ void class_assign_kernel(const int* idx, const int* newc, const int* excl, int m,
                                    const int* start, const double* val, int* cls, int* flag,
                                    int bad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const int c = excl[p] + newc[p] - 1;
  if (!eq_eps(val[idx[start[c]]], val[idx[p]])) atomicOr(flag, bad);
  cls[idx[p]] = c;
}

// The (percentile class, e_check) order has the members of an e_check class sorted by
// e_check value, then index; the greedy wants them by index.  Only classes whose members
// differ in value need it: mark them, then sort each such class by index.
__global__ void class_mixed_kernel(const int* idx, const int* newc, const int* excl, int m,
                                   const double* val, int* mixed) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < 1 || p >= m || newc[p]) return;
  if (val[idx[p - 1]] != val[idx[p]]) mixed[excl[p] + newc[p] - 1] = 1;
}

__global__ void class_index_sort_kernel(int* idx, const int* start, int n_cls, int m,
                                        const int* mixed) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cls || !mixed[c]) return;
  const int b = start[c], e = c + 1 < n_cls ? start[c + 1] : m;
  for (int i = b + 1; i < e; ++i) {
    const int v = idx[i];
    int j = i - 1;
    while (j >= b && idx[j] > v) {
      idx[j + 1] = idx[j];
      --j;
    }
    idx[j + 1] = v;
  }
}

__global__ void gather_greedy_kernel(const int* order, int G, int n, const int* fl,
                                     const uint8_t* fcnt, const double* pct, const double* e,
                                     int* g_pts, uint8_t* g_cnt, double* g_pct, double* g_e) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G) return;
  const int j = order[i];
  for (int k = 0; k < n; ++k) g_pts[(int64_t)i * n + k] = fl[(int64_t)j * n + k];
  g_cnt[i] = fcnt[j];
  g_pct[i] = pct[j];
  g_e[i] = e[j];
}

// ---------------------------------------------------------------- greedy
// The greedy of pruneMatch over candidates in greedy order.  Without replacements it
// is the in-order greedy independent set (a candidate is taken iff no earlier taken
// candidate shares one of its points), which these rounds compute in parallel: a
// candidate is taken once it is the earliest candidate not yet rejected on every one
// of its points, and rejected once an earlier taken candidate shares a point.  Then
// every rejected candidate evaluates the replacement rule against its owners (the
// taken candidates before it on its points) exactly as the sequential loop would; if
// any would replace, the caller runs the sequential loop instead.
constexpr uint8_t kUndecided = 0, kTaken = 1, kRejected = 2, kSkipped = 3;

// candidates without a point are passed over by the loop (neither kept nor owners)
__global__ void greedy_init_kernel(const uint8_t* g_cnt, int G, uint8_t* state) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < G) state[i] = g_cnt[i] == 0 ? kSkipped : kUndecided;
}

__global__ void greedy_keys_kernel(const int* g_pts, const uint8_t* g_cnt, int G, int n,
                                   int* key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G) return;
  for (int k = 0; k < n; ++k) key[(int64_t)i * n + k] = k < g_cnt[i] ? g_pts[(int64_t)i * n + k] : -1;
}

// first[f]: position in the point's list of its earliest candidate not rejected
__global__ void greedy_advance_kernel(const int* pstart, const int* items, int n_points, int n,
                                      const uint8_t* state, int* first) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_points) return;
  int q = first[f];
  const int end = pstart[f + 1];
  while (q < end && state[items[q] / n] == kRejected) ++q;
  first[f] = q;
}

__global__ void greedy_decide_kernel(const int* g_pts, const uint8_t* g_cnt, int G, int n,
                                     const int* pstart, const int* items, const int* first,
                                     uint8_t* state, int* undecided) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G || state[i] != kUndecided) return;
  bool all_first = true, blocked = false;
  for (int k = 0; k < g_cnt[i]; ++k) {
    const int f = g_pts[(int64_t)i * n + k];
    const int q = first[f];
    const int p = q < pstart[f + 1] ? items[q] / n : i;
    if (p != i) {
      all_first = false;
      if (state[p] == kTaken) blocked = true;
    }
  }
  if (blocked)
    state[i] = kRejected;
  else if (all_first)
    state[i] = kTaken;
  else
    atomicAdd(undecided, 1);
}

__global__ void greedy_owner_kernel(const int* g_pts, const uint8_t* g_cnt, int G, int n,
                                    const uint8_t* state, int* owner) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G || state[i] != kTaken) return;
  for (int k = 0; k < g_cnt[i]; ++k) owner[g_pts[(int64_t)i * n + k]] = i;
}

// StereoMatch::pruneMatch replacement rule (StereoMatch.cpp:930-975) for a rejected
// candidate against the owners of its points, averaged in point order.
__global__ void greedy_check_kernel(const int* g_pts, const uint8_t* g_cnt, int G, int n,
                                    const uint8_t* state, const int* owner, const double* g_pct,
                                    const double* g_e, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G || state[i] != kRejected) return;
  int S[OLPT_MAX_CAM];
  int ns = 0;
  double avg_pct = 0.0, avg_err = 0.0;
  for (int k = 0; k < g_cnt[i]; ++k) {
    const int o = owner[g_pts[(int64_t)i * n + k]];
    if (o < 0 || o >= i) continue;
    bool seen = false;
    for (int t = 0; t < ns; ++t) seen |= (S[t] == o);
    if (seen) continue;
    S[ns++] = o;
    avg_pct += g_pct[o];
    avg_err += g_e[o];
  }
  if (ns == 0) {  // cannot happen for a rejected candidate
    atomicOr(flag, 1);
    return;
  }
  avg_pct /= (double)ns;
  avg_err /= (double)ns;
  const double pj = g_pct[i], ej = g_e[i];
  const bool better_pct = (!eq_eps(pj, avg_pct)) && ((pj + 1e-12) < avg_pct);
  const bool tie_better = eq_eps(pj, avg_pct) && (!eq_eps(ej, avg_err)) && ((ej + 1e-12) < avg_err);
  if (better_pct || tie_better) atomicOr(flag, 1);
}

__global__ void greedy_select_kernel(const int* order, const uint8_t* state, int G, uint8_t* sel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G) return;
  sel[order[i]] = state[i] == kTaken ? 1 : 0;
}

int bit_width(uint64_t x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

}  // namespace

// Stable LSD radix sort of (key, val) pairs on the low `bits` bits; result in
// (key, val), scratch in (key2, val2).
// Short lists: one CTA sorts (masked key, original position) pairs bitonically in
// shared memory -- the same stable order as the radix passes, without their launches.
constexpr int kSmallSort = 2048;

__global__ void __launch_bounds__(1024) small_sort_kernel(const uint64_t* key, const int* val,
                                                          int n, uint64_t mask, uint64_t* key_out,
                                                          int* val_out) {
  __shared__ uint64_t k[kSmallSort];
  __shared__ int p[kSmallSort];
  int N = 1;
  while (N < n) N <<= 1;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    if (i < n) {
      k[i] = key[i] & mask;
      p[i] = i;
    } else {
      k[i] = ~0ull;
      p[i] = 0x7fffffff;
    }
  }
  __syncthreads();
  for (int size = 2; size <= N; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool asc = (i & size) == 0;
          const bool gt = k[i] > k[j] || (k[i] == k[j] && p[i] > p[j]);
          if (gt == asc) {
            const uint64_t tk = k[i];
            k[i] = k[j];
            k[j] = tk;
            const int tp = p[i];
            p[i] = p[j];
            p[j] = tp;
          }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    key_out[i] = key[p[i]];
    val_out[i] = val[p[i]];
  }
}

void radix_sort_device(DevBuf& key, DevBuf& val, DevBuf& key2, DevBuf& val2, DevBuf& hist,
                       DevBuf& scan_tmp, int n, int bits, cudaStream_t s) {
  if (n <= 1 || bits <= 0) return;
  if (n <= kSmallSort) {
    key2.ensure((size_t)(n + 1) * sizeof(uint64_t), s);
    val2.ensure((size_t)(n + 1) * sizeof(int), s);
    // the radix passes order by the key bits below the first multiple of 8 >= bits
    const int used = ((bits + 7) / 8) * 8;
    const uint64_t m = used >= 64 ? ~0ull : ((1ull << used) - 1ull);
    small_sort_kernel<<<OLPT_G(1), 1024, 0, s>>>(key.as<uint64_t>(), val.as<int>(), n, m,
                                                key2.as<uint64_t>(), val2.as<int>());
    OLPT_CUDA(cudaGetLastError());
    std::swap(key, key2);
    std::swap(val, val2);
    return;
  }
  const int n_blocks = (n + kRsTile - 1) / kRsTile;
  key2.ensure((size_t)(n + 1) * sizeof(uint64_t), s);
  val2.ensure((size_t)(n + 1) * sizeof(int), s);
  hist.ensure((size_t)(2 * 256 * n_blocks + 2) * sizeof(int), s);
  int* h = hist.as<int>();
  int* offs = h + 256 * n_blocks + 1;
  for (int shift = 0; shift < bits; shift += 8) {
    rs_hist_kernel<<<OLPT_G(n_blocks), kRsThreads, 0, s>>>(key.as<uint64_t>(), n, shift, h,
                                                         n_blocks);
    exclusive_scan(h, 256 * n_blocks, offs, scan_tmp, s);
    rs_scatter_kernel<<<OLPT_G(n_blocks), kRsThreads, 0, s>>>(
        key.as<uint64_t>(), val.as<int>(), n, shift, offs, n_blocks, key2.as<uint64_t>(),
        val2.as<int>());
    std::swap(key, key2);
    std::swap(val, val2);
  }
  OLPT_CUDA(cudaGetLastError());
}

// Sort the device candidates (ids, e, X) by ids into the `_s` buffers.  The ids of all
// cameras form one lexicographic key; when it does not fit in 64 bits it is split into
// words sorted least significant first, each pass stable, so the order is the same.
bool sort_candidates_device(PruneWork& W, const int* ids, const double* e, const double* X, int M,
                            int n, int max_id, cudaStream_t s) {
  const int bits = bit_width((uint64_t)(max_id + 1));
  if (bits > 32) return false;
  W.key.ensure((size_t)(M + 1) * sizeof(uint64_t), s);
  W.val.ensure((size_t)(M + 1) * sizeof(int), s);
  W.key2.ensure((size_t)(M + 1) * sizeof(uint64_t), s);
  W.val2.ensure((size_t)(M + 1) * sizeof(int), s);
  W.ids_s.ensure((size_t)(M + 1) * n * sizeof(int), s);
  W.e_s.ensure((size_t)(M + 1) * sizeof(double), s);
  W.X_s.ensure((size_t)(M + 1) * 3 * sizeof(double), s);
  if (M == 0) return true;
  if (bits * n <= 64) {
    id_keys_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(ids, M, n, bits, W.key.as<uint64_t>(),
                                                  W.val.as<int>());
    radix_sort_device(W.key, W.val, W.key2, W.val2, W.hist, W.scan_tmp, M, bits * n, s);
  } else {
    const int per = 64 / bits;
    const int words = (n + per - 1) / per;
    for (int w = words - 1; w >= 0; --w) {
      const bool first = w == words - 1;
      word_keys_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(
          ids, M, n, bits, per, w, first ? nullptr : W.val.as<int>(), W.key2.as<uint64_t>(),
          W.val2.as<int>());
      std::swap(W.key, W.key2);
      std::swap(W.val, W.val2);
      const int in_word = std::min(n, (w + 1) * per) - w * per;
      radix_sort_device(W.key, W.val, W.key2, W.val2, W.hist, W.scan_tmp, M, bits * in_word, s);
    }
  }
  gather_cand_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(W.val.as<int>(), M, n, ids, e, X,
                                                    W.ids_s.as<int>(), W.e_s.as<double>(),
                                                    W.X_s.as<double>());
  OLPT_CUDA(cudaGetLastError());
  return true;
}

// Steps 2-5 on the sorted candidates (W.ids_s, W.e_s); on success the greedy input
// is in W.g_* (G entries, in greedy order, with W.order mapping to candidates).
// Returns false when the host must run the reference comparator sorts.
bool prune_order_device(PruneWork& W, const PruneView& pv, int M, int n, int64_t total_points,
                        int* G_out, cudaStream_t s) {
  *G_out = 0;
  if (M == 0) return true;
  const size_t slots = (size_t)M * n;
  W.fl.ensure((slots + 1) * sizeof(int), s);
  W.slot_key.ensure((slots + 1) * sizeof(int), s);
  W.fcnt.ensure(M + 16, s);
  W.slot_pct.ensure((slots + 1) * sizeof(double), s);
  W.slot_used.ensure(slots + 16, s);
  W.pct.ensure((size_t)(M + 1) * sizeof(double), s);
  W.flag.ensure(sizeof(int), s);
  OLPT_CUDA(cudaMemsetAsync(W.flag.p, 0, sizeof(int), s));
  OLPT_CUDA(cudaMemsetAsync(W.slot_used.p, 0, slots, s));
  flat_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(W.ids_s.as<int>(), M, n, pv, W.fl.as<int>(),
                                             W.slot_key.as<int>(), W.fcnt.as<uint8_t>());
  W.points.build(W.slot_key.as<int>(), (int)slots, (int)total_points, s, true);
  const size_t smem = kPctWarps * sizeof(PoolSmem);
  OLPT_CUDA(cudaFuncSetAttribute(pct_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  W.pool_e.ensure((slots + 1) * sizeof(double), s);
  W.pool_i.ensure((slots + 1) * 5 * sizeof(int), s);
  PoolScratch gs;
  gs.e = W.pool_e.as<double>();
  gs.j = W.pool_i.as<int>();
  gs.slot = gs.j + slots;
  gs.ord = gs.slot + slots;
  gs.cls = gs.ord + slots;
  gs.start = gs.cls + slots;
  if (total_points > 0)
    pct_kernel<<<OLPT_G(nblk(total_points, kPctWarps)), kPctWarps * 32, smem, s>>>(
        W.points.start.as<int>(), W.points.items.as<int>(), (int)total_points, n,
        W.e_s.as<double>(), gs, W.slot_pct.as<double>(), W.slot_used.as<uint8_t>(),
        W.flag.as<int>());
  pct_score_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(W.fcnt.as<uint8_t>(), M, n,
                                                  W.slot_pct.as<double>(),
                                                  W.slot_used.as<uint8_t>(), W.pct.as<double>());
  // the two candidate sets and their tolerance classes
  W.f_pct.ensure((size_t)(M + 1) * sizeof(int), s);
  W.f_both.ensure((size_t)(M + 1) * sizeof(int), s);
  W.pos_pct.ensure((size_t)(M + 1) * sizeof(int), s);
  W.pos_both.ensure((size_t)(M + 1) * sizeof(int), s);
  finite_flags_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(W.pct.as<double>(), W.e_s.as<double>(), M,
                                                     W.f_pct.as<int>(), W.f_both.as<int>());
  exclusive_scan(W.f_pct.as<int>(), M, W.pos_pct.as<int>(), W.scan_tmp, s);
  exclusive_scan(W.f_both.as<int>(), M, W.pos_both.as<int>(), W.scan_tmp, s);
  int cnt[2];
  OLPT_CUDA(cudaMemcpyAsync(&cnt[0], W.pos_pct.as<int>() + M, sizeof(int), cudaMemcpyDeviceToHost,
                            s));
  OLPT_CUDA(cudaMemcpyAsync(&cnt[1], W.pos_both.as<int>() + M, sizeof(int),
                            cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  const int m_pct = cnt[0], m_both = cnt[1];
  W.pcls.ensure((size_t)(M + 1) * sizeof(int), s);
  W.ecls.ensure((size_t)(M + 1) * sizeof(int), s);
  W.newc.ensure((size_t)(M + 1) * sizeof(int), s);
  W.excl.ensure((size_t)(M + 2) * sizeof(int), s);
  W.cstart.ensure((size_t)(M + 1) * sizeof(int), s);
  W.key.ensure((size_t)(M + 1) * sizeof(uint64_t), s);
  W.val.ensure((size_t)(M + 1) * sizeof(int), s);
  // tolerance classes: class ids follow the sorted order; a class start is recorded
  // and every member is checked against it
  auto classes = [&](int m, const double* val, const int* grp, int* cls, int bad) {
    newclass_kernel<<<OLPT_G(nblk(m)), 256, 0, s>>>(W.val.as<int>(), m, val, grp,
                                                   W.newc.as<int>());
    exclusive_scan(W.newc.as<int>(), m, W.excl.as<int>(), W.scan_tmp, s);
    class_start_kernel<<<OLPT_G(nblk(m)), 256, 0, s>>>(W.newc.as<int>(), W.excl.as<int>(), m,
                                                      W.cstart.as<int>());
    class_assign_kernel<<<OLPT_G(nblk(m)), 256, 0, s>>>(W.val.as<int>(), W.newc.as<int>(),
                                                       W.excl.as<int>(), m, W.cstart.as<int>(),
                                                       val, cls, W.flag.as<int>(), bad);
    int k = 0;
    OLPT_CUDA(cudaMemcpyAsync(&k, W.excl.as<int>() + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    return k;
  };
  // percentile classes over all candidates with a finite percentile
  int n_pcls = 0;
  if (m_pct > 0) {
    compact_keys_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(W.f_pct.as<int>(), W.pos_pct.as<int>(),
                                                       M, W.pct.as<double>(),
                                                       W.key.as<uint64_t>(), W.val.as<int>());
    radix_sort_device(W.key, W.val, W.key2, W.val2, W.hist, W.scan_tmp, m_pct, 64, s);
    n_pcls = classes(m_pct, W.pct.as<double>(), nullptr, W.pcls.as<int>(), 4);
  }
  // e_check classes inside every percentile class (the reference compares e_check
  // only between candidates of equal percentile), over the candidates the greedy
  // takes: sorted by (percentile class, e_check, index)
  int n_ecls = 0;
  if (m_both > 0) {
    compact_keys_kernel<<<OLPT_G(nblk(M)), 256, 0, s>>>(W.f_both.as<int>(),
                                                       W.pos_both.as<int>(), M,
                                                       W.e_s.as<double>(), W.key.as<uint64_t>(),
                                                       W.val.as<int>());
    radix_sort_device(W.key, W.val, W.key2, W.val2, W.hist, W.scan_tmp, m_both, 64, s);
    group_keys_kernel<<<OLPT_G(nblk(m_both)), 256, 0, s>>>(W.val.as<int>(), m_both,
                                                          W.pcls.as<int>(), W.key.as<uint64_t>());
    radix_sort_device(W.key, W.val, W.key2, W.val2, W.hist, W.scan_tmp, m_both,
                      bit_width((uint64_t)n_pcls), s);
    n_ecls = classes(m_both, W.e_s.as<double>(), W.pcls.as<int>(), W.ecls.as<int>(), 8);
  }
  int flag = 0;
  OLPT_CUDA(cudaMemcpyAsync(&flag, W.flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  if (flag) return false;
  const int G = m_both;
  *G_out = G;
  if (G == 0) return true;
  // greedy order: e_check class ids already increase with the percentile class, so
  // (class, index) is (percentile class, e_check class, index).  W.val holds the
  // candidates in (percentile class, e_check, index) order from the class pass; only
  // the classes whose members differ in e_check need their members re-sorted by index.
  W.mixed.ensure((size_t)(n_ecls + 1) * sizeof(int), s);
  OLPT_CUDA(cudaMemsetAsync(W.mixed.p, 0, (size_t)(n_ecls + 1) * sizeof(int), s));
  class_mixed_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(W.val.as<int>(), W.newc.as<int>(),
                                                    W.excl.as<int>(), G, W.e_s.as<double>(),
                                                    W.mixed.as<int>());
  class_index_sort_kernel<<<OLPT_G(nblk(n_ecls)), 256, 0, s>>>(
      W.val.as<int>(), W.cstart.as<int>(), n_ecls, G, W.mixed.as<int>());
  W.g_pts.ensure((size_t)(G + 1) * n * sizeof(int), s);
  W.g_cnt.ensure(G + 16, s);
  W.g_pct.ensure((size_t)(G + 1) * sizeof(double), s);
  W.g_e.ensure((size_t)(G + 1) * sizeof(double), s);
  gather_greedy_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(
      W.val.as<int>(), G, n, W.fl.as<int>(), W.fcnt.as<uint8_t>(), W.pct.as<double>(),
      W.e_s.as<double>(), W.g_pts.as<int>(), W.g_cnt.as<uint8_t>(), W.g_pct.as<double>(),
      W.g_e.as<double>());
  OLPT_CUDA(cudaGetLastError());
  return true;
}

// The greedy on the device (see greedy_*_kernel); sel[j] = 1 for kept candidates
// (M entries, candidate order).  False when a replacement would have happened, in
// which case the caller runs the sequential greedy.
bool greedy_device(PruneWork& W, int M, int G, int n, int64_t total_points, uint8_t* sel,
                   cudaStream_t s) {
  if (M > 0) OLPT_CUDA(cudaMemsetAsync(sel, 0, (size_t)M, s));
  if (G == 0) return true;
  const size_t slots = (size_t)G * n;
  W.gkey.ensure((slots + 1) * sizeof(int), s);
  W.gstate.ensure(G + 16, s);
  W.gfirst.ensure((size_t)(total_points + 1) * sizeof(int), s);
  W.gowner.ensure((size_t)(total_points + 1) * sizeof(int), s);
  W.flag.ensure(2 * sizeof(int), s);
  const int* pts = W.g_pts.as<int>();
  const uint8_t* cnt = W.g_cnt.as<uint8_t>();
  uint8_t* state = W.gstate.as<uint8_t>();
  greedy_keys_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(pts, cnt, G, n, W.gkey.as<int>());
  W.gpoints.build(W.gkey.as<int>(), (int)slots, (int)total_points, s, true);
  greedy_init_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(cnt, G, state);
  OLPT_CUDA(cudaMemcpyAsync(W.gfirst.p, W.gpoints.start.p, (size_t)total_points * sizeof(int),
                            cudaMemcpyDeviceToDevice, s));
  int* und = W.flag.as<int>() + 1;
  // every round decides at least the earliest undecided candidate; a few rounds are
  // queued per look at the count
  constexpr int kRoundsPerSync = 4;
  for (int64_t round = 0;; round += kRoundsPerSync) {
    for (int r = 0; r < kRoundsPerSync; ++r) {
      OLPT_CUDA(cudaMemsetAsync(und, 0, sizeof(int), s));
      if (total_points > 0)
        greedy_advance_kernel<<<OLPT_G(nblk(total_points)), 256, 0, s>>>(
            W.gpoints.start.as<int>(), W.gpoints.items.as<int>(), (int)total_points, n, state,
            W.gfirst.as<int>());
      greedy_decide_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(pts, cnt, G, n,
                                                          W.gpoints.start.as<int>(),
                                                          W.gpoints.items.as<int>(),
                                                          W.gfirst.as<int>(), state, und);
    }
    OLPT_CUDA(cudaGetLastError());
    int left = 0;
    OLPT_CUDA(cudaMemcpyAsync(&left, und, sizeof(int), cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    if (left == 0) break;
    OLPT_REQUIRE(round <= (int64_t)G, OLPT_ERR_INTERNAL, "device greedy did not converge");
  }
  OLPT_CUDA(cudaMemsetAsync(W.gowner.p, 0xff, (size_t)total_points * sizeof(int), s));
  OLPT_CUDA(cudaMemsetAsync(W.flag.p, 0, sizeof(int), s));
  greedy_owner_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(pts, cnt, G, n, state, W.gowner.as<int>());
  greedy_check_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(pts, cnt, G, n, state, W.gowner.as<int>(),
                                                     W.g_pct.as<double>(), W.g_e.as<double>(),
                                                     W.flag.as<int>());
  greedy_select_kernel<<<OLPT_G(nblk(G)), 256, 0, s>>>(W.val.as<int>(), state, G, sel);
  OLPT_CUDA(cudaGetLastError());
  int flag = 0;
  OLPT_CUDA(cudaMemcpyAsync(&flag, W.flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  return flag == 0;
}

}  // namespace olpt
