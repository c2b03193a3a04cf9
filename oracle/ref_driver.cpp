// Test infrastructure only (oracle build): a small C ABI over the REFERENCE
// OpenLPT classes so that Python tests and bench.py's CPU legs can drive the
// reference's own code on in-memory data through ctypes.
//
// Every entry point forwards to the reference implementation:
//   ObjectFinder2D::findObject2D      src/srcObject/ObjectFinder.cpp:6-111
//   StereoMatch (build/check/prune/triangulate)  src/srcSTB/StereoMatch.cpp:65-1050
//   Shake::runShake / calResidualImage           src/srcSTB/Shake.cpp:36-244
//   IPR::runIPR                                   src/srcSTB/IPR.cpp:195-305
//   STB::processFrame                             src/srcSTB/STB.cpp:40-89
// The staged stereo-match entry mirrors StereoMatch::match() (StereoMatch.cpp:65-178)
// so that the pre-prune candidate set can be compared as well.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "Camera.h"
#include "Config.h"
#include "IPR.h"
#include "ObjectFinder.h"
#include "STB.h"
#include "Shake.h"
#include "StereoMatch.h"

struct DebugAccess_StereoMatch {
  static void build(const StereoMatch& m, std::vector<int>& id,
                    std::vector<std::vector<int>>& out) {
    m.buildMatch(id, out);
  }
  static bool check(const StereoMatch& m, const std::vector<int>& ids, double& e) {
    return m.checkMatch(ids, e);
  }
  static std::vector<std::vector<int>> prune(const StereoMatch& m,
                                             const std::vector<std::vector<int>>& c,
                                             const std::vector<double>& e) {
    return m.pruneMatch(c, e);
  }
  static std::vector<std::unique_ptr<Object3D>> tri(const StereoMatch& m,
                                                    const std::vector<std::vector<int>>& s) {
    return m.triangulateMatch(s);
  }
};

struct DebugAccess_Shake {
  static const std::vector<double>& scores(const Shake& s) { return s._score_list; }
};

extern "C" {

// Flat parameter block (all fields of TracerConfig used on the hot path).
typedef struct {
  int n_cam;
  int min_obj_int;
  double radius_obj;
  double shake_width;
  int n_shake_loop;
  double thred_ghost;
  double shakewidth_min;
  int ratio_augimg;
  int match_cam_count;
  int idmap_cell_px;
  double tol_2d_px;
  double tol_3d_mm;
  double limit[6];
  int n_cam_reduced;
  int n_loop_ipr;
  int n_loop_ipr_reduced;
  int n_obj2d_process_max;
  double radius_search_obj;
  int n_initial_frames;
  double radius_search_track;
  int pf_nx, pf_ny, pf_nz;
  double pf_r;
  int otf_nx, otf_ny, otf_nz;
  double otf_bound[6];
  const double* otf_abca;  // [4][n_cam][n_grid] : a, b, c, alpha
} oref_cfg_t;

}  // extern "C"

namespace {

struct Result {
  std::map<std::string, std::vector<double>> arrays;
  std::string error;
};

thread_local std::string g_last_error;

std::vector<Image> make_images(int n_cam, const double* const* imgs, const int* H, const int* W) {
  std::vector<Image> out;
  out.reserve(n_cam);
  for (int c = 0; c < n_cam; ++c) {
    Image im(H[c], W[c], 0.0);
    std::memcpy(&im(0, 0), imgs[c], sizeof(double) * (size_t)H[c] * W[c]);
    out.push_back(im);
  }
  return out;
}

void put_objects(Result* r, const std::vector<std::unique_ptr<Object3D>>& objs, int n_cam) {
  auto& xyz = r->arrays["xyz"];
  auto& uv = r->arrays["uv"];
  xyz.reserve(objs.size() * 3);
  uv.reserve(objs.size() * n_cam * 2);
  for (auto const& o : objs) {
    for (int i = 0; i < 3; ++i) xyz.push_back(o->_pt_center[i]);
    for (int c = 0; c < n_cam; ++c) {
      if (c < (int)o->_obj2d_list.size() && o->_obj2d_list[c]) {
        uv.push_back(o->_obj2d_list[c]->_pt_center[0]);
        uv.push_back(o->_obj2d_list[c]->_pt_center[1]);
      } else {
        uv.push_back(std::numeric_limits<double>::quiet_NaN());
        uv.push_back(std::numeric_limits<double>::quiet_NaN());
      }
    }
  }
}

}  // namespace

extern "C" {

const char* oref_last_error() { return g_last_error.c_str(); }
void oref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_num_procs()); }
// Seeds the C library's rand(), which Camera::polyImgToWorld draws its Newton start
// point from (src/srcMath/Camera.cpp:1176-1180).
void oref_srand(unsigned seed) { srand(seed); }
int oref_max_threads() { return omp_get_max_threads(); }

// ---------------------------------------------------------------- results
void oref_res_free(void* h) { delete static_cast<Result*>(h); }
long long oref_res_len(void* h, const char* name) {
  auto* r = static_cast<Result*>(h);
  auto it = r->arrays.find(name);
  return it == r->arrays.end() ? -1 : (long long)it->second.size();
}
int oref_res_copy(void* h, const char* name, double* out) {
  auto* r = static_cast<Result*>(h);
  auto it = r->arrays.find(name);
  if (it == r->arrays.end()) return -1;
  if (!it->second.empty()) std::memcpy(out, it->second.data(), sizeof(double) * it->second.size());
  return 0;
}

// ---------------------------------------------------------------- cameras
void* oref_cams_new(int n, const char* const* paths) {
  try {
    auto* v = new std::vector<Camera>();
    v->reserve(n);
    for (int i = 0; i < n; ++i) v->emplace_back(std::string(paths[i]));
    return v;
  } catch (std::exception const& e) {
    g_last_error = e.what();
  } catch (...) {
    g_last_error = "camera load failed";
  }
  return nullptr;
}
void oref_cams_free(void* h) { delete static_cast<std::vector<Camera>*>(h); }
void oref_cams_set_active(void* h, const int* active) {
  auto& cams = *static_cast<std::vector<Camera>*>(h);
  for (size_t i = 0; i < cams.size(); ++i) cams[i]._is_active = active[i] != 0;
}
int oref_project(void* h, int cam, long long n, const double* xyz, double* uv) {
  auto& cams = *static_cast<std::vector<Camera>*>(h);
  try {
    for (long long i = 0; i < n; ++i) {
      Pt2D p = cams[cam].project(Pt3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
      uv[2 * i] = p[0];
      uv[2 * i + 1] = p[1];
    }
  } catch (...) {
    return -1;
  }
  return 0;
}
int oref_los(void* h, int cam, long long n, const double* uv, double* line6) {
  auto& cams = *static_cast<std::vector<Camera>*>(h);
  try {
    for (long long i = 0; i < n; ++i) {
      Line3D L = cams[cam].lineOfSight(Pt2D(uv[2 * i], uv[2 * i + 1]));
      for (int k = 0; k < 3; ++k) {
        line6[6 * i + k] = L.pt[k];
        line6[6 * i + 3 + k] = L.unit_vector[k];
      }
    }
  } catch (...) {
    return -1;
  }
  return 0;
}
// lines: k x (pt xyz, unit xyz); out: xyz, err.  Returns -1 if the reference throws.
int oref_triangulate(int k, const double* lines6, double* out4) {
  std::vector<Line3D> los(k);
  for (int i = 0; i < k; ++i) {
    los[i].pt = Pt3D(lines6[6 * i], lines6[6 * i + 1], lines6[6 * i + 2]);
    los[i].unit_vector = Pt3D(lines6[6 * i + 3], lines6[6 * i + 4], lines6[6 * i + 5]);
  }
  try {
    Pt3D X;
    double err = 0;
    myMATH::triangulation(X, err, los);
    out4[0] = X[0];
    out4[1] = X[1];
    out4[2] = X[2];
    out4[3] = err;
  } catch (...) {
    return -1;
  }
  return 0;
}

// ---------------------------------------------------------------- config
void* oref_cfg_new(const oref_cfg_t* p, void* cams_h) {
  auto& cams = *static_cast<std::vector<Camera>*>(cams_h);
  auto* cfg = new TracerConfig();
  cfg->_min_obj_int = p->min_obj_int;
  cfg->_radius_obj = p->radius_obj;
  cfg->_shake_param._shake_width = p->shake_width;
  cfg->_shake_param._n_shake_loop = p->n_shake_loop;
  cfg->_shake_param._thred_ghost = p->thred_ghost;
  cfg->_shake_param._shakewidth_min = p->shakewidth_min;
  cfg->_shake_param._ratio_augimg = p->ratio_augimg;
  cfg->_sm_param.match_cam_count = p->match_cam_count;
  cfg->_sm_param.idmap_cell_px = p->idmap_cell_px;
  cfg->_sm_param.tol_2d_px = p->tol_2d_px;
  cfg->_sm_param.tol_3d_mm = p->tol_3d_mm;
  AxisLimit lim(p->limit[0], p->limit[1], p->limit[2], p->limit[3], p->limit[4], p->limit[5]);
  cfg->_sm_param.limit = lim;
  cfg->_ipr_param.n_cam_reduced = p->n_cam_reduced;
  cfg->_ipr_param.n_loop_ipr = p->n_loop_ipr;
  cfg->_ipr_param.n_loop_ipr_reduced = p->n_loop_ipr_reduced;
  cfg->_ipr_param.n_obj2d_process_max = p->n_obj2d_process_max;
  cfg->_stb_param._radius_search_obj = p->radius_search_obj;
  cfg->_stb_param._n_initial_frames = p->n_initial_frames;
  cfg->_stb_param._radius_search_track = p->radius_search_track;
  cfg->_pf_param.limit = lim;
  cfg->_pf_param.nx = p->pf_nx;
  cfg->_pf_param.ny = p->pf_ny;
  cfg->_pf_param.nz = p->pf_nz;
  cfg->_pf_param.r = p->pf_r;
  AxisLimit ob(p->otf_bound[0], p->otf_bound[1], p->otf_bound[2], p->otf_bound[3],
               p->otf_bound[4], p->otf_bound[5]);
  cfg->_otf.loadParam(p->n_cam, p->otf_nx, p->otf_ny, p->otf_nz, ob, cams);
  const int ng = cfg->_otf._param.n_grid;
  Matrix<double>* planes[4] = {&cfg->_otf._param.a, &cfg->_otf._param.b, &cfg->_otf._param.c,
                               &cfg->_otf._param.alpha};
  for (int q = 0; q < 4; ++q)
    for (int c = 0; c < p->n_cam; ++c)
      for (int g = 0; g < ng; ++g) (*planes[q])(c, g) = p->otf_abca[((size_t)q * p->n_cam + c) * ng + g];
  return cfg;
}
void oref_cfg_free(void* h) { delete static_cast<TracerConfig*>(h); }

// ---------------------------------------------------------------- stages
void* oref_find_peaks(void* cfg_h, const double* img, int H, int W) {
  auto& cfg = *static_cast<TracerConfig*>(cfg_h);
  Image im(H, W, 0.0);
  std::memcpy(&im(0, 0), img, sizeof(double) * (size_t)H * W);
  ObjectFinder2D f;
  auto objs = f.findObject2D(im, cfg);
  auto* r = new Result();
  auto& xy = r->arrays["xy"];
  xy.reserve(objs.size() * 2);
  for (auto const& o : objs) {
    xy.push_back(o->_pt_center[0]);
    xy.push_back(o->_pt_center[1]);
  }
  return r;
}

// Staged StereoMatch::match(): candidates (sorted by ids), prune selection, and
// the final objects, each selected match triangulated on its own so that the
// surviving ones can be identified.
void* oref_stereo(void* cams_h, void* cfg_h, int n_cam, const long long* counts,
                  const double* const* xy) {
  auto& cams = *static_cast<std::vector<Camera>*>(cams_h);
  auto& cfg = *static_cast<TracerConfig*>(cfg_h);
  auto* r = new Result();
  try {
    std::vector<std::vector<std::unique_ptr<Object2D>>> o2d(n_cam);
    for (int c = 0; c < n_cam; ++c) {
      for (long long i = 0; i < counts[c]; ++i) {
        auto t = std::make_unique<Tracer2D>();
        t->_r_px = cfg._radius_obj;
        t->_pt_center[0] = xy[c][2 * i];
        t->_pt_center[1] = xy[c][2 * i + 1];
        o2d[c].push_back(std::move(t));
      }
    }
    StereoMatch sm(cams, o2d, cfg);
    int ref_cam = -1;
    size_t best = std::numeric_limits<size_t>::max();
    for (int i = 0; i < n_cam; ++i) {
      if (!cams[i]._is_active) continue;
      if (o2d[i].size() < best) {
        best = o2d[i].size();
        ref_cam = i;
      }
    }
    struct MS {
      std::vector<int> ids;
      double e;
    };
    const int T = std::max(1, omp_get_max_threads());
    std::vector<std::vector<MS>> buckets(T);
    const long long n_ref = (long long)o2d[ref_cam].size();
#pragma omp parallel num_threads(T)
    {
      auto& bucket = buckets[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 32)
      for (long long id_ref = 0; id_ref < n_ref; ++id_ref) {
        std::vector<int> mc(n_cam, -1);
        mc[ref_cam] = (int)id_ref;
        std::vector<std::vector<int>> bc;
        DebugAccess_StereoMatch::build(sm, mc, bc);
        for (auto& cand : bc) {
          double e = std::numeric_limits<double>::quiet_NaN();
          if (!DebugAccess_StereoMatch::check(sm, cand, e)) continue;
          bucket.push_back(MS{std::move(cand), e});
        }
      }
    }
    std::vector<MS> all;
    for (auto& b : buckets)
      for (auto& m : b) all.push_back(std::move(m));
    std::sort(all.begin(), all.end(), [](const MS& a, const MS& b) { return a.ids < b.ids; });
    std::vector<std::vector<int>> cands;
    std::vector<double> es;
    auto& rc = r->arrays["cand"];
    auto& re = r->arrays["e_check"];
    for (auto& m : all) {
      for (int v : m.ids) rc.push_back(v);
      re.push_back(m.e);
      cands.push_back(m.ids);
      es.push_back(m.e);
    }
    auto sel = DebugAccess_StereoMatch::prune(sm, cands, es);
    auto& rs = r->arrays["sel"];
    auto& rk = r->arrays["kept"];
    std::vector<std::unique_ptr<Object3D>> objs;
    for (auto& s : sel) {
      for (int v : s) rs.push_back(v);
      auto one = DebugAccess_StereoMatch::tri(sm, std::vector<std::vector<int>>{s});
      rk.push_back(one.empty() ? 0.0 : 1.0);
      for (auto& o : one) objs.push_back(std::move(o));
    }
    put_objects(r, objs, n_cam);
    r->arrays["ref_cam"] = {(double)ref_cam};
  } catch (std::exception const& e) {
    g_last_error = e.what();
    delete r;
    return nullptr;
  }
  return r;
}

// Shake::runShake on tracers placed at xyz (radius radius_obj); returns the
// shaken positions, flags, per-object scores and final projections.
void* oref_shake(void* cams_h, void* cfg_h, long long n_obj, const double* xyz, int n_cam,
                 const double* const* imgs, const int* H, const int* W) {
  auto& cams = *static_cast<std::vector<Camera>*>(cams_h);
  auto& cfg = *static_cast<TracerConfig*>(cfg_h);
  auto* r = new Result();
  try {
    std::vector<std::unique_ptr<Object3D>> objs;
    objs.reserve(n_obj);
    for (long long i = 0; i < n_obj; ++i) {
      CreateArgs a;
      a._pt_center = Pt3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
      objs.push_back(cfg.creatObject3D(std::move(a)));
    }
    auto images = make_images(n_cam, imgs, H, W);
    Shake sh(cams, cfg);
    auto flags = sh.runShake(objs, images);
    auto& rf = r->arrays["flags"];
    for (auto f : flags) rf.push_back((double)(int)f);
    r->arrays["score"] = DebugAccess_Shake::scores(sh);
    put_objects(r, objs, n_cam);
  } catch (std::exception const& e) {
    g_last_error = e.what();
    delete r;
    return nullptr;
  }
  return r;
}

// Shake::calResidualImage (output_ipr = true) for tracers at xyz with flags
// (flags may be null).  Arrays "img0", "img1", ...
void* oref_residual(void* cams_h, void* cfg_h, long long n_obj, const double* xyz,
                    const int* flags, int n_cam, const double* const* imgs, const int* H,
                    const int* W) {
  auto& cams = *static_cast<std::vector<Camera>*>(cams_h);
  auto& cfg = *static_cast<TracerConfig*>(cfg_h);
  auto* r = new Result();
  try {
    std::vector<std::unique_ptr<Object3D>> objs;
    for (long long i = 0; i < n_obj; ++i) {
      CreateArgs a;
      a._pt_center = Pt3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
      auto o = cfg.creatObject3D(std::move(a));
      o->projectObject2D(cams);
      objs.push_back(std::move(o));
    }
    std::vector<ObjFlag> fl;
    if (flags)
      for (long long i = 0; i < n_obj; ++i) fl.push_back((ObjFlag)flags[i]);
    auto images = make_images(n_cam, imgs, H, W);
    Shake sh(cams, cfg);
    auto res = sh.calResidualImage(objs, images, flags ? &fl : nullptr);
    for (int c = 0; c < n_cam; ++c) {
      auto& v = r->arrays["img" + std::to_string(c)];
      v.assign(&res[c](0, 0), &res[c](0, 0) + (size_t)H[c] * W[c]);
    }
  } catch (std::exception const& e) {
    g_last_error = e.what();
    delete r;
    return nullptr;
  }
  return r;
}

// IPR::runIPR on in-memory images.
void* oref_ipr(void* cams_h, void* cfg_h, int n_cam, const double* const* imgs, const int* H,
               const int* W) {
  auto& cams = *static_cast<std::vector<Camera>*>(cams_h);
  auto& cfg = *static_cast<TracerConfig*>(cfg_h);
  auto* r = new Result();
  try {
    auto images = make_images(n_cam, imgs, H, W);
    IPR ipr(cams);
    auto objs = ipr.runIPR(cfg, images);
    put_objects(r, objs, n_cam);
  } catch (std::exception const& e) {
    g_last_error = e.what();
    delete r;
    return nullptr;
  }
  return r;
}

}  // extern "C"

extern "C" {
// OTF::estimateUniformOTFFromImage (OTF.cpp:17-144) of camera `cam` on n_img in-memory
// images of that camera; out: a, b, c, alpha of grid node 0.  Returns 1 when the
// reference skipped the estimation (an image without detections), -1 on a throw.
int oref_otf_estimate(void* cfg_h, int cam, int n_img, const double* const* imgs, const int* H,
                      const int* W, double* out4) {
  auto& cfg = *static_cast<TracerConfig*>(cfg_h);
  try {
    auto images = make_images(n_img, imgs, H, W);
    const double before = cfg._otf._param.a(cam, 0);
    cfg._otf._param.a(cam, 0) = std::nan("");
    cfg._otf.estimateUniformOTFFromImage(cam, cfg, images);
    const bool skipped = std::isnan(cfg._otf._param.a(cam, 0));
    if (skipped) cfg._otf._param.a(cam, 0) = before;
    out4[0] = cfg._otf._param.a(cam, 0);
    out4[1] = cfg._otf._param.b(cam, 0);
    out4[2] = cfg._otf._param.c(cam, 0);
    out4[3] = cfg._otf._param.alpha(cam, 0);
    return skipped ? 1 : 0;
  } catch (std::exception const& e) {
    g_last_error = e.what();
    return -1;
  }
}

// OTF::getOTFParam (OTF.cpp:273-338) of the config's OTF for n points.
int oref_otf_param(void* cfg_h, int cam, long long n, const double* xyz, double* out5) {
  auto& cfg = *static_cast<TracerConfig*>(cfg_h);
  for (long long i = 0; i < n; ++i) {
    auto r = cfg._otf.getOTFParam(cam, Pt3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
    for (int k = 0; k < 5; ++k) out5[5 * i + k] = r[k];
  }
  return 0;
}
}  // extern "C"

// ---------------------------------------------------------------- STB
// STB::processFrame (src/srcSTB/STB.cpp:40-89) on in-memory frames.  The STB is
// built from reference-format config files (BasicSetting::readConfig and the
// STB constructor, which estimates an OTF from the first frames); the OTF is then
// replaced by the scene's exact table (when one is given) so that the device run
// sees the same one.
struct DebugAccess_STB {
  static ObjectConfig& cfg(STB& s) { return *s._obj_config; }
};

namespace {
struct RefStb {
  BasicSetting bs;
  std::unique_ptr<STB> stb;
};

void put_tracks(Result* r, const char* name, const std::deque<Track>& tracks) {
  auto& v = r->arrays[name];
  for (size_t i = 0; i < tracks.size(); ++i) {
    const Track& tr = tracks[i];
    for (size_t k = 0; k < tr._obj3d_list.size(); ++k) {
      v.push_back((double)i);
      v.push_back((double)tr._t_list[k]);
      for (int d = 0; d < 3; ++d) v.push_back(tr._obj3d_list[k]->_pt_center[d]);
    }
  }
}
}  // namespace

extern "C" {

void* oref_stb_new(const char* main_cfg, const char* otf_file) {
  try {
    auto* r = new RefStb();
    if (!r->bs.readConfig(main_cfg)) {
      g_last_error = "BasicSetting::readConfig failed";
      delete r;
      return nullptr;
    }
    r->stb = std::make_unique<STB>(r->bs, "Tracer", r->bs._object_config_paths.at(0));
    auto& tc = static_cast<TracerConfig&>(DebugAccess_STB::cfg(*r->stb));
    if (otf_file && *otf_file) tc._otf.loadParam(std::string(otf_file));
    return r;
  } catch (std::exception const& e) {
    g_last_error = e.what();
  } catch (...) {
    g_last_error = "STB construction failed";
  }
  return nullptr;
}

void oref_stb_free(void* h) { delete static_cast<RefStb*>(h); }

// SMParam::match_cam_count after the config is read (the tracer config file has no
// line for it; readCommonConfig caps the default of 4 at n_cam, Config.cpp:222-224).
void oref_stb_set_match_cam_count(void* h, int n) {
  auto* r = static_cast<RefStb*>(h);
  DebugAccess_STB::cfg(*r->stb)._sm_param.match_cam_count = n;
}

// The tracer config's OTF table [4][n_cam][n_grid] (a, b, c, alpha); returns n_grid.
int oref_stb_otf(void* h, double* out) {
  auto* r = static_cast<RefStb*>(h);
  auto& tc = static_cast<TracerConfig&>(DebugAccess_STB::cfg(*r->stb));
  const OTFParam& p = tc._otf._param;
  const int n_cam = p.n_cam, n_grid = p.n_grid;
  if (out) {
    const Matrix<double>* m[4] = {&p.a, &p.b, &p.c, &p.alpha};
    for (int q = 0; q < 4; ++q)
      for (int c = 0; c < n_cam; ++c)
        for (int g = 0; g < n_grid; ++g) out[((size_t)q * n_cam + c) * n_grid + g] = (*m[q])(c, g);
  }
  return n_grid;
}

int oref_stb_frame(void* h, int frame, int n_cam, const double* const* imgs, const int* H,
                   const int* W) {
  auto* r = static_cast<RefStb*>(h);
  try {
    auto images = make_images(n_cam, imgs, H, W);
    r->stb->processFrame(frame, images);
  } catch (std::exception const& e) {
    g_last_error = e.what();
    return -1;
  } catch (...) {
    g_last_error = "processFrame failed";
    return -1;
  }
  return 0;
}

// tracks of the four lists: rows of (track index, frame, x, y, z)
void* oref_stb_tracks(void* h) {
  auto* r = static_cast<RefStb*>(h);
  auto* res = new Result();
  put_tracks(res, "long_active", r->stb->_long_track_active);
  put_tracks(res, "short_active", r->stb->_short_track_active);
  put_tracks(res, "long_inactive", r->stb->_long_track_inactive);
  put_tracks(res, "exit", r->stb->_exit_track);
  return res;
}

}  // extern "C"
