// Shake-the-Box state: parameters, host-side track containers (the reference's
// four std::deque<Track>, inc/libSTB/STB.h:60-66, here TrackList) and the device views used by
// the per-frame kernels in stb.cu.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
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

// Growable array of a trivially copyable T whose first N elements live inline, so a
// short track costs no heap allocation (tens of thousands of short tracks are created
// and dropped per frame).  Only the operations the track code uses.
template <class T, int N>
class SmallVec {
 public:
  SmallVec() = default;
  ~SmallVec() { release(); }
  SmallVec(const SmallVec& o) { append(o.begin(), o.end()); }
  SmallVec(SmallVec&& o) noexcept { take(o); }
  SmallVec& operator=(const SmallVec& o) {
    if (this != &o) {
      n_ = 0;
      append(o.begin(), o.end());
    }
    return *this;
  }
  SmallVec& operator=(SmallVec&& o) noexcept {
    if (this != &o) {
      release();
      take(o);
    }
    return *this;
  }
  size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  T* begin() { return data(); }
  T* end() { return data() + n_; }
  const T* begin() const { return data(); }
  const T* end() const { return data() + n_; }
  T& operator[](size_t i) { return data()[i]; }
  const T& operator[](size_t i) const { return data()[i]; }
  void push_back(const T& v) {
    if (n_ == cap_) grow(n_ + 1);
    data()[n_++] = v;
  }
  // append only: pos must be end()
  void insert(const T* pos, const T* first, const T* last) {
    (void)pos;
    append(first, last);
  }
  void assign(const T* first, const T* last) {
    n_ = 0;
    append(first, last);
  }
  void clear() { n_ = 0; }

 private:
  T* heap_ = nullptr;
  uint32_t n_ = 0, cap_ = N;
  T buf_[N];
  T* data() { return heap_ ? heap_ : buf_; }
  const T* data() const { return heap_ ? heap_ : buf_; }
  void append(const T* first, const T* last) {
    const size_t k = (size_t)(last - first);
    if (n_ + k > cap_) grow(n_ + k);
    std::memcpy(data() + n_, first, k * sizeof(T));
    n_ += (uint32_t)k;
  }
  void grow(size_t need) {
    size_t cap = cap_ * 2;
    while (cap < need) cap *= 2;
    T* p = static_cast<T*>(std::malloc(cap * sizeof(T)));
    if (!p) throw std::bad_alloc();
    std::memcpy(p, data(), n_ * sizeof(T));
    std::free(heap_);
    heap_ = p;
    cap_ = (uint32_t)cap;
  }
  void release() {
    std::free(heap_);
    heap_ = nullptr;
    n_ = 0;
    cap_ = N;
  }
  void take(SmallVec& o) {
    n_ = o.n_;
    cap_ = o.cap_;
    if (o.heap_) {
      heap_ = o.heap_;
      o.heap_ = nullptr;
    } else {
      heap_ = nullptr;
      std::memcpy(buf_, o.buf_, n_ * sizeof(T));
    }
    o.n_ = 0;
    o.cap_ = N;
  }
};

// One track: points in frame order (Track::_obj3d_list centres, _t_list); up to four
// points inline.
struct TrackH {
  SmallVec<double, 12> xyz;  // 3 per point
  SmallVec<int, 4> t;
  size_t size() const { return t.size(); }
};

// A track list in list order (the reference's std::deque<Track>; only appends,
// indexing and whole-list replacement are needed).
using TrackList = std::vector<TrackH>;

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
