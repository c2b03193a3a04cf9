// Host-side context shared by all translation units of libolpt_cuda.so.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/olpt.h"
#include "olpt_device.cuh"
#include "olpt_mlp.h"
#include "olpt_prof.h"
#include "olpt_shake.h"
#include "olpt_stb.h"
#include "olpt_stereo.h"
#include "olpt_trackio.h"

namespace olpt {

// Number of kernel launches issued by this library (every launch site wraps its
// grid expression in OLPT_G, which is evaluated exactly once per launch).
extern std::atomic<long long> g_launches;
#define OLPT_G(grid) (::olpt::g_launches.fetch_add(1, std::memory_order_relaxed), (grid))

struct CudaError {
  cudaError_t code;
  std::string where;
};
struct ApiError {
  olpt_status_t code;
  std::string msg;
};

#define OLPT_CUDA(call)                                                             \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess) throw ::olpt::CudaError{_e, std::string(#call) + " @ " + \
                                                       __FILE__ + ":" + std::to_string(__LINE__)}; \
  } while (0)

#define OLPT_REQUIRE(cond, code, msg) \
  do {                                \
    if (!(cond)) throw ::olpt::ApiError{(code), (msg)}; \
  } while (0)

// Grow-only device buffer (stream-ordered allocation).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t need, cudaStream_t s) {
    if (need <= bytes) return;
    if (p) OLPT_CUDA(cudaFreeAsync(p, s));
    size_t nb = need + need / 4 + 256;
    OLPT_CUDA(cudaMallocAsync(&p, nb, s));
    bytes = nb;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
  void release(cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    bytes = 0;
  }
};

// Pinned host staging buffer.
struct HostBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t need) {
    if (need <= bytes) return;
    if (p) cudaFreeHost(p);
    size_t nb = need + need / 4 + 256;
    OLPT_CUDA(cudaMallocHost(&p, nb));
    bytes = nb;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
};

// One camera image plane in HBM (row pitch padded to 16 bytes for vector loads).
struct ImagePlane {
  DevBuf buf;
  int dtype = OLPT_U8;
  int H = 0, W = 0;
  int64_t pitch = 0;  // bytes
};

struct OtfDev {
  int nx = 2, ny = 2, nz = 2, n_grid = 8;
  double bmin[3], bmax[3];
  double d[3];  // grid spacing
  double* table = nullptr;  // [4][n_cam][n_grid] a,b,c,alpha (device)
  int alpha_zero = 0;       // every alpha entry is +0.0 (cos = 1, sin = +0 exactly)
};

// Per-camera 2D detection list (SoA, FP64 like the reference's Pt2D).
struct Dets {
  DevBuf x, y, rc;          // rc: packed (row<<16 | col) is not enough for 2048+; store int2
  int64_t cap = 0;
};

// CSR (start[n_buckets + 1], items[n]) from per-item bucket keys (key < 0: dropped);
// built by count -> exclusive scan -> scatter -> per-bucket ascending order (scan.cu).
struct Csr {
  DevBuf start, items, cursor, tmp;
  // sort_buckets: ascending item order inside each bucket (only where order matters)
  void build(const int* key, int n, int n_buckets, cudaStream_t s, bool sort_buckets = false);
  void release(cudaStream_t s) {
    start.release(s);
    items.release(s);
    cursor.release(s);
    tmp.release(s);
  }
};

// Device workspace of the shake (grown on demand).
struct ShakeWork {
  DevBuf otfp;      // n x n_cam x 5 OTF parameters at the object centres
  DevBuf pair_key;  // n x n_cam tile keys
  Csr bins;         // (object, camera) pairs per image tile
  DevBuf rep, hkey, has_nb, nb_pos, nb_list, scan_tmp, gpart;
  Csr hash;         // 3D hash grid of object centres
  void release(cudaStream_t s) {
    nb_pos.release(s);
    nb_list.release(s);
    scan_tmp.release(s);
    otfp.release(s);
    pair_key.release(s);
    bins.release(s);
    rep.release(s);
    hkey.release(s);
    has_nb.release(s);
    gpart.release(s);
    hash.release(s);
  }
};

// Device workspace of stereo matching (grown on demand, reused across frames).
struct StereoWork {
  DevBuf cell_start[OLPT_MAX_CAM], cell_cursor[OLPT_MAX_CAM], cell_items[OLPT_MAX_CAM];
  DevBuf cell_of[OLPT_MAX_CAM], los[OLPT_MAX_CAM];
  DevBuf l2d[OLPT_MAX_CAM * OLPT_MAX_CAM];
  DevBuf cxy[OLPT_MAX_CAM], cbp[OLPT_MAX_CAM * OLPT_MAX_CAM];
  DevBuf l2d_ptrs, cbp_ptrs, active_d, counters, scan_tmp;
  DevBuf path_a, path_b, term, pairs;
  DevBuf cand_ids, cand_e, cand_x;
  // near-tolerance decision log: records (olpt_near_record) and a 64-bit counter of
  // every near-tolerance test seen since the last reset (records beyond near_cap are
  // counted, not stored)
  DevBuf near_rec, near_count;
  double near_band = 0.0;
  int64_t near_cap = 0;
  void release(cudaStream_t s) {
    near_rec.release(s);
    near_count.release(s);
    for (int c = 0; c < OLPT_MAX_CAM; ++c) {
      cell_start[c].release(s);
      cell_cursor[c].release(s);
      cell_items[c].release(s);
      cell_of[c].release(s);
      los[c].release(s);
    }
    for (auto& b : l2d) b.release(s);
    for (auto& b : cxy) b.release(s);
    for (auto& b : cbp) b.release(s);
    l2d_ptrs.release(s);
    cbp_ptrs.release(s);
    active_d.release(s);
    counters.release(s);
    path_a.release(s);
    path_b.release(s);
    term.release(s);
    pairs.release(s);
    cand_ids.release(s);
    cand_e.release(s);
    cand_x.release(s);
  }
};

// Per camera: active flag, detection count and offset of its first detection in the
// global point numbering of the prune.
struct PruneView {
  int active[OLPT_MAX_CAM];
  int count[OLPT_MAX_CAM];
  int offset[OLPT_MAX_CAM];
};

// Device workspace of the candidate sort and prune (prune.cu).
struct PruneWork {
  DevBuf key, val, key2, val2, hist, scan_tmp;
  DevBuf ids_s, e_s, X_s;
  DevBuf fl, slot_key, fcnt, slot_pct, slot_used, pct, flag;
  DevBuf f_pct, f_both, pos_pct, pos_both, pcls, ecls, newc, excl, cstart;
  DevBuf g_pts, g_cnt, g_pct, g_e, pool_e, pool_i;
  DevBuf gkey, gstate, gfirst, gowner, sel, spos, scnt, mixed;
  Csr points, gpoints;
  HostBuf pin;  // pinned staging of the greedy's input
  void release(cudaStream_t s) {
    for (DevBuf* b : {&key, &val, &key2, &val2, &hist, &scan_tmp, &ids_s, &e_s, &X_s, &fl,
                      &slot_key, &fcnt, &slot_pct, &slot_used, &pct, &flag, &f_pct, &f_both,
                      &pos_pct, &pos_both, &pcls, &ecls, &newc, &excl, &cstart, &g_pts, &g_cnt,
                      &g_pct, &g_e, &pool_e, &pool_i, &gkey, &gstate, &gfirst, &gowner, &sel, &spos, &scnt, &mixed})
      b->release(s);
    points.release(s);
    gpoints.release(s);
  }
};

// 3D objects resident on the device (SoA).
struct Objects {
  DevBuf xyz;    // n x 3 double
  DevBuf uv;     // n x n_cam x 2 double: current 2D projections
  DevBuf flags;  // n uint8 (ObjFlag bits)
  DevBuf score;  // n double
  int64_t n = 0;
  void ensure(int64_t cap, int n_cam, cudaStream_t s) {
    xyz.ensure((cap + 1) * 3 * sizeof(double), s);
    uv.ensure((cap + 1) * n_cam * 2 * sizeof(double), s);
    flags.ensure(cap + 16, s);
    score.ensure((cap + 1) * sizeof(double), s);
  }
  void release(cudaStream_t s) {
    xyz.release(s);
    uv.release(s);
    flags.release(s);
    score.release(s);
  }
};

// IPR knobs (IPRParam + tracer threshold, inc/libSTB/Config.h:37-44, 190-195).
struct IprParams {
  double min_obj_int;
  SmParams sm;
  ShakeParams shake;
  int n_cam_reduced, n_loop_ipr, n_loop_ipr_reduced;
  int64_t n_obj2d_process_max;
};

// IPR workspace and the accumulated output objects of the last run.
struct IprWork {
  DevBuf perm, tx, ty, trc, keep, pos, scan_tmp;
  DevBuf out_xyz, out_uv;
  int64_t n_out = 0, cap_out = 0;
  void release(cudaStream_t s) {
    perm.release(s);
    tx.release(s);
    ty.release(s);
    trc.release(s);
    keep.release(s);
    pos.release(s);
    scan_tmp.release(s);
    out_xyz.release(s);
    out_uv.release(s);
    n_out = cap_out = 0;
  }
};

void stereo_match_device(olpt_ctx* ctx, const SmParams& prm, StereoResult& res);
bool prune_select_device(olpt_ctx* ctx, const PruneView& pv, int M, int n_cam,
                         int64_t total_points, char* selected);
// Download a device-resident stereo result (no-op for a host one).
void stereo_result_to_host(olpt_ctx* ctx, StereoResult& r);
// The kept matches become the context's 3D objects (triangulateMatch order); returns
// their number.
int64_t stereo_objects(olpt_ctx* ctx, const StereoResult& r);
void ipr_device(olpt_ctx* ctx, const IprParams& p);
OtfView otf_view(olpt_ctx* ctx);
void shake_device(olpt_ctx* ctx, const ShakeParams& sp);
void residual_device(olpt_ctx* ctx, const ShakeParams& sp, bool use_flags, bool make_current);

// Track files (trackio.cu): device buffers of the row formatter and the writer thread.
// async: the frame loop's track files are written while later frames run (flush_files
// waits for them); otherwise every save returns after its file is written.
constexpr int64_t kMaxRowsPerPass = 1 << 20;
struct TrackIoWork {
  DevBuf ints, xyz, uv, len, off, bad, bytes, tmp;
  bool async = false;
  FileWriter writer;
  void release(cudaStream_t s) {
    for (DevBuf* x : {&ints, &xyz, &uv, &len, &off, &bad, &bytes, &tmp}) x->release(s);
  }
};
// rows of n_int ints, then n1 + n2 doubles from two arrays (device), "%.6f" numbers,
// comma separated, one per line; n <= kMaxRowsPerPass; appended to out
void format_rows_device(olpt_ctx* ctx, const int* ints, int n_int, const double* d1, int n1,
                        const double* d2, int n2, int64_t n, std::string& out);
// bytes -> file on the writer thread (waits for it unless the context writes async)
void write_file(olpt_ctx* ctx, const std::string& file, std::string&& bytes);
// waits for every posted file; throws the first write error
void flush_files(olpt_ctx* ctx);
// OTF estimation from the context's planes (otf_est.cu); false: an image without detections
bool otf_estimate_device(olpt_ctx* ctx, double min_int, double r_pt, int max_det, double abc[3],
                         int64_t* n_samples);

// Device workspace of the STB frame loop (grown on demand, reused across frames).
struct StbWork {
  DevBuf a, b, c, d, ia, link, flag, field, field2, kern, k1, k2;
  Csr g1, g2;
  void release(cudaStream_t s) {
    for (DevBuf* x : {&a, &b, &c, &d, &ia, &link, &flag, &field, &field2, &kern, &k1, &k2})
      x->release(s);
    g1.release(s);
    g2.release(s);
  }
};

// STB state (STB members, inc/libSTB/STB.h:58-70): the four track lists and the
// initial-phase IPR results.
struct StbState {
  StbParams p;
  IprParams ipr;
  bool configured = false;
  TrackList short_active, long_active, long_inactive, exited;
  // capacity kept for the frame loop's temporary lists: one spare per role, so that the
  // long-track and short-track buffers each circulate between their list and its spare
  TrackList spare_long, spare_short;
  std::vector<std::vector<double>> ipr_xyz;   // initial phase, per frame
  std::vector<std::vector<char>> ipr_tracked;
  std::vector<double> linfit_kernel;          // 2 x n_pts
  int64_t last_new = 0, last_extended = 0;
  std::vector<double> last_xyz;               // particles of the last frame
  ImagePlane frame_img[OLPT_MAX_CAM];         // the frame's images as processFrame leaves them
  StbWork w;
};

// Device state of the learned proposal (mlp.cu): f32 master parameters, Adam moments
// and gradients (flat, MlpDims::params), bf16 weight copies for the GEMMs (row-major and
// transposed), and the activations of one batch.
struct MlpWork {
  bool ready = false;
  MlpDims dims = mlp_dims(4);  // network geometry (set from the camera count at init)
  int adam_t = 0;
  LearnedParams lp;
  int64_t n_learned = 0, n_fallback = 0;  // objects through the learned shake / its fallback
  int64_t cap = 0;  // batch capacity of the activation buffers
  DevBuf master, grad, am, av, wb1, wb2, wb3, wt2, wt3;
  DevBuf x, xt, xin, tgt, z1, z2, z3, h1, h2, h3, h1t, h2t, o, dout;
  DevBuf dz1f, dz2f, dz3f, dz2b, dz3b, dz1t, dz2t, dz3t, part, hpart, loss, err;
  // learned shake: keep[i] = 1 for the input objects the network did not drop (the
  // objects left are the kept ones in input order), pos = their exclusive scan; fb =
  // fallback counter
  DevBuf keep, pos, start_xyz, act, nres, ds_x, ds_t, loss_hist, fb;
  void release(cudaStream_t s) {
    for (DevBuf* b : {&master, &grad, &am, &av, &wb1, &wb2, &wb3, &wt2, &wt3, &x, &xt, &xin, &tgt,
                      &z1, &z2, &z3, &h1, &h2, &h3, &h1t, &h2t, &o, &dout, &dz1f, &dz2f, &dz3f,
                      &dz2b, &dz3b, &dz1t, &dz2t, &dz3t, &part, &hpart, &loss, &err, &keep, &pos,
                      &start_xyz, &act, &nres, &ds_x, &ds_t, &loss_hist, &fb})
      b->release(s);
    ready = false;
    cap = 0;
  }
};

// mlp.cu
// the network geometry of the context's camera count, unless a network is set
void mlp_sync_dims(olpt_ctx* ctx);
void mlp_init(olpt_ctx* ctx, uint64_t seed);
void mlp_set_params(olpt_ctx* ctx, const float* host);
void mlp_get_params(olpt_ctx* ctx, float* host);
// features of the context's objects against residual planes computed with all of
// them (FP32 or FP64 planes per sp.precision); x: n x dims.in_pad bf16 (device),
// f32 (optional, device): n x dims.in
void mlp_features_device(olpt_ctx* ctx, const ShakeParams& sp, __nv_bfloat16* x, float* f32);
// f32 rows of dims.in (device) -> bf16 rows of dims.in_pad
void mlp_input_device(olpt_ctx* ctx, const float* x_f32, int64_t n, __nv_bfloat16* x);
void gelu_inplace_device(float* p, int64_t n, cudaStream_t s);
// residual planes of the current images with every object projected (the first step
// of a shake iteration)
void residual_all_device(olpt_ctx* ctx, const ShakeParams& sp);
// o (device, n x 4) = network(x)
void mlp_infer_device(olpt_ctx* ctx, const __nv_bfloat16* x, int64_t n, float* o);
// one training batch: loss (mean), gradients into MlpWork::grad, Adam update when lr > 0
double mlp_train_device(olpt_ctx* ctx, const float* x_f32, const float* tgt, int64_t n, double lr,
                        double ghost_weight, bool update);
// steps Adam steps on uniform mini-batches of a device-resident dataset (cosine
// learning-rate decay to 5%); losses (host, optional) per step
void mlp_train_many(olpt_ctx* ctx, const float* x, const float* t, int64_t n, int batch, int steps,
                    double lr, double ghost_weight, uint64_t seed, float* losses);
// the learned shake: features -> network -> correction and ghost pruning -> short
// plain refinement -> full plain shake for objects whose residue stays high
void learned_shake_device(olpt_ctx* ctx, const ShakeParams& sp);

void stb_configure(olpt_ctx* ctx, const StbParams& p, const IprParams& ipr);
void stb_process_frame(olpt_ctx* ctx, int frame);
TrackList& stb_list(olpt_ctx* ctx, int which);
void stb_save_tracks(olpt_ctx* ctx, int which, const std::string& path);
void stb_load_tracks(olpt_ctx* ctx, int which, const std::string& path);

}  // namespace olpt

struct olpt_ctx {
  int device = 0;
  // launch shapes chosen by olpt_autotune_ipr (they never change results)
  olpt_tuning tune{4, 256, 64};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  int n_cam = 0;
  std::vector<olpt::CamDev> cams_h;
  olpt::DevBuf cams_d;

  olpt::OtfDev otf;
  olpt::DevBuf otf_table;

  olpt::ImagePlane img[OLPT_MAX_CAM];  // current working image per camera

  // detections
  olpt::Dets dets[OLPT_MAX_CAM];
  // int64 words: [OLPT_MAX_CAM] detection counts, then the staged detector's error
  // word, band ticket and per-band look-back states
  olpt::DevBuf det_counts;
  std::vector<int64_t> det_counts_h;
  struct DetMap {  // TMA descriptor of one camera plane, re-encoded when the plane changes
    const void* p = nullptr;
    int dtype = -1, H = 0, W = 0, box_w = 0, box_h = 0;
    int64_t pitch = 0;
    CUtensorMap map;
  } det_map[OLPT_MAX_CAM];
  olpt::DevBuf band_counts, band_offsets;
  olpt::DevBuf lut_u8, lut_u16;  // log(max(v, 1e-4)) of every integer level
  // failure-detection test hook of the next staged detection launch (-1 = off)
  int test_hold_ticket = -1;
  unsigned long long test_wait_limit_ns = 0;

  // stereo matching
  olpt::StereoWork sm;
  olpt::StereoResult sm_result;
  olpt::PruneWork prune;

  // 3D objects (stereo output / shake input and output)
  olpt::Objects obj;

  // shake: residual planes (FP32 or FP64) and workspace
  olpt::ImagePlane resid[OLPT_MAX_CAM];
  olpt::ShakeWork shk;

  // IPR workspace and output
  olpt::IprWork ipr;

  // Shake-the-Box frame loop
  olpt::StbState stb;
  olpt::TrackIoWork tio;

  // learned proposal
  olpt::MlpWork mlp;

  // optional per-kernel event timing
  olpt::Prof prof;

  // scratch
  olpt::DevBuf scratch;
  olpt::HostBuf pinned;
};
