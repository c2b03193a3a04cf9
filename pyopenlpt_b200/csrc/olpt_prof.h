// Optional per-kernel timing: when enabled, launches of the named kernel classes are
// bracketed by CUDA events recorded on the context's stream (no extra
// synchronisation); olpt_profile_read sums the durations after a sync.  The
// algorithmic bytes of every timed launch are accumulated alongside.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <vector>

namespace olpt {

enum ProfKernel : int {
  PROF_PEAKS = 0,     // detection, count + emit passes
  PROF_STEREO = 1,    // stereo level expansion (all levels)
  PROF_RESIDUAL = 2,  // tile-owned residual image
  PROF_SHAKE = 3,     // warp-per-particle shake
  PROF_PF = 4,        // predictive-field nodes (STB initial phase)
  PROF_N = 5
};

// Host wall-clock phases (ids PROF_N + phase in olpt_profile_read).
enum ProfPhase : int {
  PH_DETECT = 0,   // detection incl. count read-back
  PH_STEREO = 1,   // whole stereo match (device + host)
  PH_PRUNE = 2,    // candidate sort + prune + greedy (device and host)
  PH_SHAKE = 3,    // whole shake (all iterations + flags)
  PH_OUTPUT = 4,   // compaction of kept objects + final residual
  PH_TRACK = 5,    // STB track bookkeeping, prediction, linking and pruning
  PH_GREEDY_HOST = 6,  // sequential greedy, run when the device greedy meets a replacement
  // parts of PH_TRACK
  PH_TR_PREDICT = 7,   // packing, prediction kernel, range check
  PH_TR_EXTEND = 8,    // extension of the long tracks by their shaken predictions
  PH_TR_LINK = 9,      // new objects: repeat removal, short-track linking, new tracks
  PH_TR_PRUNE = 10,    // linear-fit pruning of the long tracks
  PH_N = 11
};

struct Prof {
  bool on = false;
  double phase_ms[PH_N] = {};
  long long phase_n[PH_N] = {};
  struct Rec {
    cudaEvent_t a, b;
    double bytes;
  };
  std::vector<Rec> open[PROF_N];
  std::vector<cudaEvent_t> pool;

  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  // begin/end bracket one launch (or one group of launches) on stream s
  int begin(int k, cudaStream_t s) {
    if (!on) return -1;
    Rec r{get(), get(), 0.0};
    cudaEventRecord(r.a, s);
    open[k].push_back(r);
    return (int)open[k].size() - 1;
  }
  void end(int k, int id, cudaStream_t s, double bytes) {
    if (id < 0) return;
    open[k][id].bytes = bytes;
    cudaEventRecord(open[k][id].b, s);
  }
  // sum of durations (ms), launches and bytes; recycles the events
  void read(int k, double& ms, long long& n, double& bytes) {
    ms = 0;
    n = 0;
    bytes = 0;
    for (auto& r : open[k]) {
      float t = 0;
      cudaEventSynchronize(r.b);
      cudaEventElapsedTime(&t, r.a, r.b);
      ms += t;
      bytes += r.bytes;
      ++n;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    open[k].clear();
  }
  void add_phase(int p, double ms) {
    if (!on) return;
    phase_ms[p] += ms;
    phase_n[p] += 1;
  }
  void read_phase(int p, double& ms, long long& n) {
    ms = phase_ms[p];
    n = phase_n[p];
    phase_ms[p] = 0;
    phase_n[p] = 0;
  }
  void release() {
    for (auto& v : open)
      for (auto& r : v) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
      }
    for (auto e : pool) cudaEventDestroy(e);
    pool.clear();
  }
};

// Scope timer for a host phase (wall clock, includes the stream waits it contains).
struct PhaseTimer {
  Prof& p;
  int id;
  std::chrono::steady_clock::time_point t0;
  PhaseTimer(Prof& pr, int i) : p(pr), id(i), t0(std::chrono::steady_clock::now()) {}
  ~PhaseTimer() {
    p.add_phase(id, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                        .count());
  }
};

}  // namespace olpt
