/*
 * olpt.h -- C ABI of the B200-native OpenLPT hot path (libolpt_cuda.so).
 *
 * Plain C types only: no exceptions cross this boundary, every entry returns an
 * olpt_status_t and olpt_last_error(ctx) holds the message of the last failure.
 * A context owns one CUDA stream and all device-resident state of one camera
 * rig (cameras, OTF table, current images, 2D detections, 3D objects).  Calls on
 * one context are stream-ordered; entry points that return host data
 * synchronise the context's stream before returning.  One context per host
 * thread; a context must not be used from two threads at once.
 *
 * Each entry cites the reference (OpenLPT) interface it replaces.
 */
#ifndef OLPT_H
#define OLPT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum olpt_status {
  OLPT_OK = 0,
  OLPT_ERR_INVALID_ARG = 1,
  OLPT_ERR_OOM = 2,
  OLPT_ERR_CUDA = 3,
  OLPT_ERR_TIMEOUT = 4,
  OLPT_ERR_UNSUPPORTED = 5,
  OLPT_ERR_INTERNAL = 6
} olpt_status_t;

typedef enum olpt_dtype { OLPT_U8 = 0, OLPT_U16 = 1, OLPT_F32 = 2, OLPT_F64 = 3 } olpt_dtype_t;

typedef struct olpt_ctx olpt_ctx;

/* Camera parameters, as read by Camera::loadParameters (src/srcMath/Camera.cpp:19-158).
 * type 0 = PINHOLE, 1 = POLYNOMIAL.  Polynomial coefficient tables are
 * n_coeff x 4 row-major (coeff, x_power, y_power, z_power). */
typedef struct olpt_camera_desc {
  int type;
  int n_row, n_col;
  int is_active;
  double cam_mtx[9];
  int n_dist;
  double dist[12];
  double r_mtx[9], t_vec[3], r_inv[9], t_inv[3];
  int ref_plane; /* 1 = REF_X, 2 = REF_Y, 3 = REF_Z */
  double plane[2];
  int n_coeff;
  const double* u_coeffs;
  const double* v_coeffs;
} olpt_camera_desc;

/* ------------------------------------------------------------------ context */
/* (no reference counterpart: the reference is host-only) */
olpt_status_t olpt_ctx_create(olpt_ctx** out, int device);
void olpt_ctx_destroy(olpt_ctx* ctx);
const char* olpt_last_error(const olpt_ctx* ctx);
/* Synchronise the context's stream. */
olpt_status_t olpt_sync(olpt_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that record their own events. */
olpt_status_t olpt_stream(olpt_ctx* ctx, void** stream);
/* Per-kernel event timing (no reference counterpart; the reference prints clock()
 * CPU time per stage).  kernel: 0 = detection, 1 = stereo level expansion,
 * 2 = residual image, 3 = shake, 4 = predictive field (device time from CUDA
 * events); 5..11 = host wall-clock phases (detection, stereo matching, candidate
 * sort + prune + greedy, shake, output compaction + residual, STB track work outside
 * the IPR and the shake of predictions, the sequential greedy run when the device
 * greedy meets a replacement).  read returns the summed duration,
 * the number of timed launches/phases and their algorithmic bytes since the last
 * read. */
olpt_status_t olpt_profile(olpt_ctx* ctx, int enable);
/* Total number of kernel launches issued by this library in this process. */
int64_t olpt_launch_count(void);
olpt_status_t olpt_profile_read(olpt_ctx* ctx, int kernel, double* total_ms, int64_t* launches,
                                double* bytes);

/* ------------------------------------------------------------------ cameras */
/* Replaces std::vector<Camera> set-up (Camera::loadParameters, Camera.cpp:19-158;
 * polynomial derivative tables as Camera::updatePolyDuDv, Camera.cpp:340-393). */
olpt_status_t olpt_cameras_upload(olpt_ctx* ctx, const olpt_camera_desc* cams, int n_cam);
/* Replaces toggling Camera::_is_active (inc/libMath/Camera.h:83; CameraUtil::setActiveSubset). */
olpt_status_t olpt_cameras_set_active(olpt_ctx* ctx, const int* active);
/* Camera::project (Camera.cpp:648-677) for n world points; host arrays n x 3 -> n x 2. */
olpt_status_t olpt_camera_project(olpt_ctx* ctx, int cam, int64_t n, const double* xyz,
                                  double* uv);
/* Camera::lineOfSight (Camera.cpp:996-1016) for n image points; out n x 6 (pt, unit). */
olpt_status_t olpt_camera_los(olpt_ctx* ctx, int cam, int64_t n, const double* uv,
                              double* line6);
/* myMATH::triangulation (src/srcMath/myMATH.cpp:357-419) for n_sets independent sets
 * of k lines (n_sets x k x 6); out n_sets x 4 (x, y, z, err), ok[i] = 0 where the
 * reference throws (negative squared distance). */
olpt_status_t olpt_triangulate(olpt_ctx* ctx, int64_t n_sets, int k, const double* lines6,
                               double* out4, int* ok);

/* ------------------------------------------------------------------ OTF */
/* OTF::loadParam(file) contents (src/srcSTB/OTF.cpp:195-243): grid sizes, boundary
 * (xmin,xmax,ymin,ymax,zmin,zmax) and a table [4][n_cam][nx*ny*nz] of a, b, c, alpha. */
olpt_status_t olpt_otf_upload(olpt_ctx* ctx, int nx, int ny, int nz, const double* bound6,
                              const double* abca);
/* OTF::getOTFParam (OTF.cpp:273-338) for n points on one camera; out n x 5
 * (a, b, c, cos alpha, sin alpha). */
olpt_status_t olpt_otf_param(olpt_ctx* ctx, int cam, int64_t n, const double* xyz, double* out5);

/* ------------------------------------------------------------------ images */
/* Load the current image of every camera (replaces building std::vector<Image>,
 * inc/libMath/Matrix.h:171, from ImageIO::loadImg).  imgs[c] points to H[c] x W[c]
 * elements of `dtype` with row pitch pitch_bytes[c] (0 = dense).  on_device != 0
 * means the pointers are device pointers (zero host traffic). */
olpt_status_t olpt_images_upload(olpt_ctx* ctx, int n_cam, olpt_dtype_t dtype,
                                 const void* const* imgs, const int* H, const int* W,
                                 const int64_t* pitch_bytes, int on_device);
/* Copy the current image of camera `cam` to host memory as `dtype` (F32 or F64). */
olpt_status_t olpt_image_download(olpt_ctx* ctx, int cam, olpt_dtype_t dtype, void* out);

/* ------------------------------------------------------------------ 2D detection */
/* ObjectFinder2D::findObject2D -> findTracer2D (src/srcObject/ObjectFinder.cpp:6-111) on the
 * current image of every active camera, keeping detections on the device (raster order,
 * as the reference).  One read of each image; OLPT_ERR_TIMEOUT if one of the kernel's
 * bounded device waits (tile staging, ordering between row bands) ran out.
 * counts (host, n_cam) receives the number of detections per camera. */
olpt_status_t olpt_find_peaks(olpt_ctx* ctx, double min_obj_int, int64_t* counts);
/* Download detections of one camera in raster order: xy (n x 2, x = col, y = row) and
 * the integer peak pixel rc (n x 2: row, col); either may be NULL. */
olpt_status_t olpt_get_peaks(olpt_ctx* ctx, int cam, double* xy, int32_t* rc, int64_t cap);
/* Failure-detection test hook (no reference counterpart): in the next olpt_find_peaks
 * that uses the staged single-read kernel, the row band with this ticket (tickets
 * number the bands of all cameras in launch order, camera 0 first) never publishes its
 * detection count, and the bands after it give up their bounded look-back wait after
 * wait_limit_ns (at most 2 s) instead of the default 2 s.  That olpt_find_peaks then
 * returns OLPT_ERR_TIMEOUT with its results void, and the context stays usable. */
olpt_status_t olpt_test_hold_detection_band(olpt_ctx* ctx, int ticket, int64_t wait_limit_ns);
/* Replace the detections of every camera with host lists (n_cam arrays of n x 2). */
olpt_status_t olpt_detections_upload(olpt_ctx* ctx, int n_cam, const int64_t* counts,
                                     const double* const* xy);

/* Allocation-free tracer detection on one camera image.  No counterpart in the
 * reference (which is host-only): it exists for callers that cannot allocate device
 * memory -- code that runs inside another framework's memory arena or caching
 * allocator, or a plug-in host that budgets the device memory itself -- so it needs
 * no context and calls no cudaMalloc/cudaFree or allocating library routine.  Same
 * results as olpt_find_peaks (through the two-pass kernels: count, scan, emit); its
 * scratch (per-band counts and offsets) and the log table live in library-owned
 * static device arrays that every GPU loading this library holds until exit.
 *   d_img       device image, H x W elements of `dtype`, rows pitch_bytes apart
 *               (pitch and pointer 16-byte aligned); H, W at most 16384
 *   d_x, d_y    device outputs (capacity doubles each), d_rc device output
 *               (capacity x 2 int32: row, col), raster order
 *   capacity    at least (H * W + 1) / 2
 *   d_count     device int64 receiving the number of detections
 *   stream      cudaStream_t to launch on (NULL = default stream); the call returns
 *               without synchronising.
 * Every call resolves the static arrays' device addresses; the first call in each
 * CUDA context of a device (the first on the device, and the first after a
 * cudaDeviceReset) also fills the log table with a synchronous copy, so make it
 * before any stream capture.  All calls share the static scratch: calls that overlap on
 * the GPU (different streams, host threads) race; serialise them.  Error text:
 * olpt_find_peaks_noalloc_error(). */
olpt_status_t olpt_find_peaks_noalloc(const void* d_img, olpt_dtype_t dtype, int H, int W,
                                      int64_t pitch_bytes, double min_obj_int, double* d_x,
                                      double* d_y, int32_t* d_rc, int64_t capacity,
                                      int64_t* d_count, void* stream);
const char* olpt_find_peaks_noalloc_error(void);

/* ------------------------------------------------------------------ stereo matching */
/* StereoMatch parameters (SMParam, inc/libSTB/Config.h:72-80): limit is the
 * (xmin,xmax,ymin,ymax,zmin,zmax) box of accepted triangulations. */
typedef struct olpt_sm_params {
  int match_cam_count;
  int idmap_cell_px;
  double tol_2d_px;
  double tol_3d_mm;
  double limit[6];
} olpt_sm_params;

/* StereoMatch(cams, obj2d_list, cfg).match() (src/srcSTB/StereoMatch.cpp:20-178) on the
 * current detections of the active cameras.  The selected, triangulated matches
 * become the context's current 3D objects.  n_candidates: size of the checked
 * candidate set (before the prune); n_matches: number of objects. */
olpt_status_t olpt_stereo_match(olpt_ctx* ctx, const olpt_sm_params* p, int64_t* n_candidates,
                                int64_t* n_matches);

/* Near-tolerance decision log of stereo matching (no counterpart in the reference,
 * which decides with the same tests without recording them).  The 2D tests of
 * IDMap::visitPointsInRowSpans (|(q - p) x u|^2 > tol^2, StereoMatch.cpp:1582-1615)
 * and StereoMatch::checkBackProjection (StereoMatch.cpp:1214-1223) whose distance
 * lies within band_px of tol_2d_px are appended to a device log by every
 * subsequent olpt_stereo_match (and every stereo step inside olpt_ipr_run and
 * olpt_stb_process_frame), so that a decision that rounding could flip is visible.
 * enable: band_px > 0 turns the log on with room for `capacity` records and clears
 * it; band_px = 0 turns it off.  read: copies up to `cap` records (in append order,
 * which is not deterministic) and the number of near-tolerance tests seen since the
 * last enable or reset (records beyond the capacity are counted, not stored). */
typedef struct olpt_near_record {
  int32_t kind;      /* 0 = strip test: the target detection against a chosen point's
                        image line; 1 = back-projection: the chosen point against the
                        target detection's image line on the chosen camera */
  int32_t n_chosen;  /* cameras in the partial match when the test ran */
  int32_t cam, id;   /* the tested detection on the target camera */
  int32_t other_cam, other_id; /* the chosen detection it was tested against */
  double margin_px;  /* |distance| - tol_2d_px (negative: accepted side) */
} olpt_near_record;
olpt_status_t olpt_stereo_near_log_enable(olpt_ctx* ctx, double band_px, int64_t capacity);
olpt_status_t olpt_stereo_near_log_read(olpt_ctx* ctx, olpt_near_record* out, int64_t cap,
                                        int64_t* n_total);
olpt_status_t olpt_stereo_near_log_reset(olpt_ctx* ctx);
/* Candidate set of the last match in the reference's order (sorted by ids):
 * ids n_candidates x n_cam (-1 = unused camera), e_check, triangulated xyz. */
olpt_status_t olpt_get_candidates(olpt_ctx* ctx, int32_t* ids, double* e_check, double* xyz);
/* Selected matches of the last match (triangulateMatch output order): ids, xyz. */
olpt_status_t olpt_get_matches(olpt_ctx* ctx, int32_t* ids, double* xyz);
/* StereoMatch::pruneMatch (src/srcSTB/StereoMatch.cpp:631-980) on a host candidate list
 * already in the reference's order (sorted by ids): ids M x n_cam, e_check M,
 * det_counts/active per camera; selected[j] = 1 for kept candidates.  Host only. */
olpt_status_t olpt_prune_matches(int n_cam, int64_t M, const int32_t* ids, const double* e_check,
                                 const int64_t* det_counts, const int* active, uint8_t* selected);
/* The same prune run on the context's device (the path olpt_stereo_match takes):
 * percentile scores and tolerance classes, the greedy order and the greedy itself on
 * the device, the sequential greedy on the host only when a replacement fires.
 * Identical output to olpt_prune_matches. */
olpt_status_t olpt_prune_matches_device(olpt_ctx* ctx, int n_cam, int64_t M, const int32_t* ids,
                                        const double* e_check, const int64_t* det_counts,
                                        const int* active, uint8_t* selected);

/* ------------------------------------------------------------------ 3D objects */
/* Replace the context's 3D objects with n tracers at xyz (n x 3); their 2D
 * projections are computed on the device (Object3D::projectObject2D,
 * src/srcObject/ObjectInfo.cpp:32-47) by the next shake or residual call. */
olpt_status_t olpt_objects_upload(olpt_ctx* ctx, int64_t n, const double* xyz);
olpt_status_t olpt_objects_count(olpt_ctx* ctx, int64_t* n);
/* Download objects: xyz (n x 3), 2D projections uv (n x n_cam x 2), flags (ObjFlag bits:
 * 1 = Ghost, 2 = Repeated, inc/libSTB/Shake.h:19) and shake scores; any may be NULL. */
olpt_status_t olpt_objects_download(olpt_ctx* ctx, double* xyz, double* uv, uint8_t* flags,
                                    double* score);

/* ------------------------------------------------------------------ shake */
/* ShakeParam + tracer radius + tol_3d (inc/libSTB/Config.h:82-89, 190-200).
 * precision: 0 = FP32 residual / OTF Gaussian / squared-error sums (production),
 * 1 = FP64 throughout (parity with the reference's double arithmetic). */
typedef struct olpt_shake_params {
  double shake_width;
  double shakewidth_min;
  int n_shake_loop;
  double thred_ghost;
  int ratio_augimg;
  double radius_obj;
  double tol_3d_mm;
  int precision;
} olpt_shake_params;

/* Shake(cams, cfg).runShake(objs, images) (src/srcSTB/Shake.cpp:36-163) on the context's
 * objects and current images: objects are moved in place; flags and scores are set. */
olpt_status_t olpt_shake(olpt_ctx* ctx, const olpt_shake_params* p);
/* Shake::calResidualImage(objs, images, flags) (Shake.h:41-48, Shake.cpp:165-244 with
 * output_ipr): every camera, clamped at 0; objects with non-zero flags are skipped
 * when use_flags.  make_current != 0 replaces the current images with the residual. */
olpt_status_t olpt_residual(olpt_ctx* ctx, const olpt_shake_params* p, int use_flags,
                            int make_current);
/* Copy the last residual plane of camera `cam` to host memory as F32 or F64. */
olpt_status_t olpt_residual_download(olpt_ctx* ctx, int cam, olpt_dtype_t dtype, void* out);

/* ------------------------------------------------------------------ IPR */
/* ObjectConfig knobs used by IPR::runIPR (IPRParam, SMParam, ShakeParam and the
 * tracer's _min_obj_int / _radius_obj; inc/libSTB/Config.h:37-44, 72-89, 190-195). */
typedef struct olpt_ipr_params {
  double min_obj_int;
  olpt_sm_params sm;
  olpt_shake_params shake;
  int n_cam_reduced;
  int n_loop_ipr;
  int n_loop_ipr_reduced;
  int64_t n_obj2d_process_max;
} olpt_ipr_params;

/* IPR(cams).runIPR(cfg, images) (src/srcSTB/IPR.cpp:195-305) on the current images:
 * full camera set, then reduced subsets, each for its loop count, with the 2D
 * tolerance growing x1.5 per loop.  The current images end as the final residual.
 * n_objects receives the number of reconstructed objects. */
olpt_status_t olpt_ipr_run(olpt_ctx* ctx, const olpt_ipr_params* p, int64_t* n_objects);
/* Launch shapes of the shake (warps per block: 1, 2 or 4; registers a thread: 64, with
 * 8 resident blocks per SM, or 128, with 4) and of the residual image (threads per
 * 32x32 tile block: 128 or 256).  They change only the speed: every result is the same
 * for every choice.  Default {4, 256, 64}. */
typedef struct olpt_tuning {
  int shake_warps_per_block;
  int residual_threads;
  int shake_regs;
} olpt_tuning;
olpt_status_t olpt_tuning_get(olpt_ctx* ctx, olpt_tuning* out);
olpt_status_t olpt_tuning_set(olpt_ctx* ctx, const olpt_tuning* t);
/* The autotuner's candidates (at most OLPT_TUNING_CANDIDATES), in trial order. */
#define OLPT_TUNING_CANDIDATES 8
olpt_status_t olpt_tuning_candidates(olpt_tuning* out, int* n);
/* Autotuner: times olpt_ipr_run on the context's current images (restored before every
 * trial) with each candidate launch shape, `reps` runs each, keeps the fastest in the
 * context and returns it with its mean time (cand_ms, optional: every candidate's mean
 * time in trial order).  Every candidate must reproduce the first candidate's objects
 * bit for bit (OLPT_ERR_INTERNAL otherwise).  The images are left as they were before
 * the call. */
olpt_status_t olpt_autotune_ipr(olpt_ctx* ctx, const olpt_ipr_params* p, int reps,
                                olpt_tuning* best, double* best_ms, double* cand_ms);
/* Independent frames at once (no reference counterpart): olpt_ipr_run on every
 * context, each from its own host thread on its own stream, so the frames' kernels
 * overlap on the device.  n_objects[i] receives context i's count; the first failing
 * context's status is returned (its message in that context's olpt_last_error). */
olpt_status_t olpt_ipr_run_batch(olpt_ctx* const* ctxs, int n_ctx, const olpt_ipr_params* p,
                                 int64_t* n_objects);
/* Objects of the last olpt_ipr_run in the reference's output order: xyz (n x 3) and
 * their 2D projections uv (n x n_cam x 2); either may be NULL. */
olpt_status_t olpt_ipr_result(olpt_ctx* ctx, double* xyz, double* uv);

/* ------------------------------------------------------------------ STB */
/* STB configuration: the tracer's IPR knobs plus STBParam and PFParam
 * (inc/libSTB/Config.h:17-69) and BasicSetting's frame range and axis limit; all
 * lengths in mm (the reference multiplies its config values by voxel_to_mm,
 * src/srcSTB/Config.cpp:195-230).  Replaces STB::STB(setting, "Tracer", cfg_path)
 * (inc/libSTB/STB.h:38-40) once the config files are read. */
typedef struct olpt_stb_params {
  olpt_ipr_params ipr;
  int frame_start;
  int frame_end;
  int n_initial_frames;           /* >= 4 */
  double radius_search_obj_mm;    /* initial-phase link radius */
  double radius_search_track_mm;  /* convergence-phase link radius */
  double limit[6];                /* axis limit: x_min, x_max, y_min, y_max, z_min, z_max */
  int pf_n[3];                    /* predictive-field grid nodes (>= 2 each) */
  double pf_r_mm;                 /* predictive-field search half-width */
  int pf_nbin[3];                 /* displacement PDF bins (reference default 11) */
  int pf_smooth;                  /* smooth the field (reference default 1) */
  double pf_sigma[3];             /* smoothing sigma per component (default 1) */
  const char* output_path;        /* NULL / "": no files; else the reference's outputs
                                     (InitialTrack/, ConvergeTrack/, PredField_*.csv) */
} olpt_stb_params;

enum {
  OLPT_TRACK_LONG_ACTIVE = 0,   /* STB::_long_track_active */
  OLPT_TRACK_SHORT_ACTIVE = 1,  /* STB::_short_track_active */
  OLPT_TRACK_LONG_INACTIVE = 2, /* STB::_long_track_inactive */
  OLPT_TRACK_EXIT = 3           /* STB::_exit_track */
};

/* Reset the tracker and set its parameters. */
olpt_status_t olpt_stb_configure(olpt_ctx* ctx, const olpt_stb_params* p);
/* STB::processFrame(frame_id, img_list) (src/srcSTB/STB.cpp:40-89) on the current
 * images (olpt_images_upload).  Initial phase: IPR, and at the last initial frame the
 * predictive-field linking; convergence phase: predict, shake, IPR on the residual,
 * repeat check, short-track linking, linear-fit pruning.  The current images end as
 * residuals. */
olpt_status_t olpt_stb_process_frame(olpt_ctx* ctx, int frame);
/* Independent sequences at once (no reference counterpart): olpt_stb_process_frame
 * (ctxs[i], frames[i]) for every context, each on a persistent host worker and the
 * context's own stream, so the sequences' kernels overlap on the device.  Each
 * sequence's results are those of running it alone.  The first failing context's
 * status is returned (its message in that context's olpt_last_error). */
olpt_status_t olpt_stb_process_frame_batch(olpt_ctx* const* ctxs, int n_ctx, const int* frames);
/* Sizes of the four track lists (indexed by OLPT_TRACK_*), and the particles of the
 * last frame: predictions extended and new IPR objects (either pointer may be NULL). */
olpt_status_t olpt_stb_counts(olpt_ctx* ctx, int64_t counts[4], int64_t* n_extended,
                              int64_t* n_new);
/* The particles of the last frame, in list order: the extended long tracks' new
 * points, then the new objects of the frame (STB::runConvPhase), or the IPR objects
 * of an initial-phase frame.  Call with xyz = NULL to get n only; else n is the
 * capacity on input and the count on output. */
olpt_status_t olpt_stb_frame_objects(olpt_ctx* ctx, int64_t* n, double* xyz);
/* The image of camera `cam` as STB::processFrame leaves it in img_list after the last
 * frame (the input in the initial phase; in the convergence phase the residual of
 * the shaken predictions, Shake::calResidualImage, STB.cpp:418), as F32 or F64. */
olpt_status_t olpt_stb_frame_image(olpt_ctx* ctx, int cam, olpt_dtype_t dtype, void* out);
/* Number of track points (rows of the track files) with frame id `frame` over the
 * four lists: after olpt_stb_process_frame(frame), the particles that frame added. */
olpt_status_t olpt_stb_frame_points(olpt_ctx* ctx, int frame, int64_t* n);
/* Number of tracks and of points (rows) in one list. */
olpt_status_t olpt_stb_track_rows(olpt_ctx* ctx, int which, int64_t* n_tracks, int64_t* n_rows);
/* The rows of one list in the order of STB::saveTracks: track id (= position in the
 * list), frame id, x, y, z. capacity_rows bounds the output. */
olpt_status_t olpt_stb_get_tracks(olpt_ctx* ctx, int which, int32_t* track_id, int32_t* frame,
                                  double* xyz, int64_t capacity_rows);
/* Replace one list by rows (track ids index the list, as in STB::loadTracks). */
olpt_status_t olpt_stb_set_tracks(olpt_ctx* ctx, int which, const int32_t* track_id,
                                  const int32_t* frame, const double* xyz, int64_t n_rows);
/* STB::saveTracks / loadTracks (src/srcSTB/STB.cpp:967-1047) for one list, in the
 * reference's CSV format. */
olpt_status_t olpt_stb_save_tracks(olpt_ctx* ctx, int which, const char* path);
olpt_status_t olpt_stb_load_tracks(olpt_ctx* ctx, int which, const char* path);
/* OTF::estimateUniformOTFFromImage (src/srcSTB/OTF.cpp:17-144) for one camera, on
 * the device: the context's planes are that camera's images (one plane per image, with
 * one camera description per plane for the sizes); tracer detections above
 * min_obj_int, at most max_per_image of them per image (the reference: 1000, chosen by
 * std::shuffle with std::default_random_engine(123)), the window of radius
 * radius_obj_px around each, and the reference's a = min(mean + 2 std, max) of the
 * centre pixels and least squares for b, c.  abc = (a, b, c), uniform over the grid
 * with alpha = 0; n_samples = window pixels used, 0 when an image has no detection
 * (the reference then leaves the OTF unchanged). */
olpt_status_t olpt_otf_estimate(olpt_ctx* ctx, double min_obj_int, double radius_obj_px,
                                int max_per_image, double abc[3], int64_t* n_samples);
/* Track files (olpt_stb_save_tracks and the per-frame files of olpt_stb_process_frame
 * under output_path, STB::saveTracksAll, src/srcSTB/STB.cpp:926-965) are formatted on
 * the device and written by a writer thread of the context.  enable = 0 (default):
 * each call returns after its files are written.  enable = 1: the calls return once
 * the rows are formatted and the files are written while later frames run, in call
 * order; olpt_track_files_flush waits for them and reports the first write error (a
 * later save reports it too), olpt_stb_load_tracks and olpt_ctx_destroy wait for them
 * first.  The numbers are those of the reference's std::fixed, precision 6 output
 * ("%.6f": the exact binary value rounded to six decimals, ties to even). */
olpt_status_t olpt_track_files_async(olpt_ctx* ctx, int enable);
olpt_status_t olpt_track_files_flush(olpt_ctx* ctx);
/* The device formatter on n host doubles: "%.6f" of each, one per line, into out
 * (capacity bytes; out = NULL: length only).  |v| >= 2^63 gives OLPT_ERR_UNSUPPORTED. */
olpt_status_t olpt_format_fixed6(olpt_ctx* ctx, const double* values, int64_t n, char* out,
                                 int64_t capacity, int64_t* length);

/* ------------------------------------------------------------------ learned proposal */
/* No reference counterpart: a small MLP that reads, for each candidate after stereo
 * matching, C cameras x 11 x 11 patches of max(0, residual + own projection) divided
 * by the candidate's OTF amplitude, the 2 C sub-pixel offsets of its projections and
 * a constant 1 (n_in = 121 C + 2 C + 1 values, camera-major, patches row-major), and
 * predicts a 3D correction (units of out_scale_mm) and a ghost logit.  Layers n_in ->
 * 256 -> 256 -> 256 (GELU, erf form) -> 4; bf16 weights and activations on tcgen05
 * GEMMs with f32 accumulation.  Parameters are one flat f32 array: W1[256][n_in],
 * b1[256], W2[256][256], b2[256], W3[256][256], b3[256], W4[4][256], b4[4].  C is the
 * context's camera count when the network is initialised or set (2..8; 4 when no
 * cameras are uploaded yet); OLPT_MLP_IN / OLPT_MLP_PARAMS are the 4-camera sizes. */
#define OLPT_MLP_IN 493
#define OLPT_MLP_OUT 4
#define OLPT_MLP_PARAMS 259076
/* Input width and parameter count of the network for a rig of n_cam cameras. */
olpt_status_t olpt_mlp_dims(int n_cam, int* n_in, int64_t* n_params);

/* The learned shake used by olpt_ipr_run (and the IPR inside the STB frame loop) when
 * enable != 0, in place of the plain runShake: the network corrects every candidate
 * and drops those with a ghost logit above ghost_logit; refine_loops plain shake
 * iterations from refine_width_mm follow; objects whose residue (divided by the mean
 * squared OTF amplitude) stays above fallback_residual restart the full plain shake
 * from their stereo position.  Repeated / ghost flags as in runShake. */
typedef struct olpt_learned_params {
  int enable;
  double out_scale_mm;
  double ghost_logit;
  int refine_loops;
  double refine_width_mm;
  double fallback_residual;
} olpt_learned_params;

/* Initialise the parameters (He-uniform, seeded; zero biases; Adam state reset). */
olpt_status_t olpt_mlp_init(olpt_ctx* ctx, uint64_t seed);
olpt_status_t olpt_mlp_set_params(olpt_ctx* ctx, const float* params);
olpt_status_t olpt_mlp_get_params(olpt_ctx* ctx, float* params);
/* out (n x 4) = network(x (n x n_in)); host or device pointers (on_device). */
olpt_status_t olpt_mlp_forward(olpt_ctx* ctx, int64_t n, const float* x, float* out,
                               int on_device);
/* One training step on a batch: targets n x 4 (dx, dy, dz in units of out_scale_mm,
 * ghost label 0/1); loss = mean[(1 - ghost) * mean_d (o_d - t_d)^2 + ghost_weight *
 * BCE(o_3, ghost)].  Gradients of the mean loss go to grad (host, n_params floats,
 * optional); update != 0 applies Adam (lr, 0.9, 0.999, 1e-8). */
olpt_status_t olpt_mlp_train_step(olpt_ctx* ctx, int64_t n, const float* x, const float* targets,
                                  int on_device, double lr, double ghost_weight, int update,
                                  double* loss, float* grad);
/* Training on a device-resident dataset: x (n x n_in) and targets (n x 4), host
 * arrays copied to the device once (or device pointers, on_device != 0); `steps` Adam
 * steps on mini-batches of `batch` rows drawn uniformly with replacement (seeded), the
 * learning rate decayed from lr by a cosine to 5%.  losses (host, optional): one per
 * step. */
olpt_status_t olpt_mlp_train(olpt_ctx* ctx, int64_t n, const float* x, const float* targets,
                             int on_device, int batch, int steps, double lr, double ghost_weight,
                             uint64_t seed, float* losses);
/* Features (n_objects x n_in) of the context's objects, against a residual of the
 * current images with every object projected. */
olpt_status_t olpt_mlp_features(olpt_ctx* ctx, const olpt_shake_params* p, float* x,
                                int on_device);
olpt_status_t olpt_learned_configure(olpt_ctx* ctx, const olpt_learned_params* p);
/* The learned shake on the context's objects (as olpt_shake). */
olpt_status_t olpt_shake_learned(olpt_ctx* ctx, const olpt_shake_params* p);
/* Objects that went through the learned shake and how many fell back, since the
 * context was created. */
olpt_status_t olpt_learned_stats(olpt_ctx* ctx, int64_t* n_learned, int64_t* n_fallback);
/* out (M x N, f32) = A (M x K) * B (N x K)^T (+ bias, GELU when gelu != 0) on the
 * tensor-core GEMM; A and B bf16 bit patterns, all host buffers. */
olpt_status_t olpt_bf16_gemm(olpt_ctx* ctx, int M, int N, int K, const uint16_t* A,
                             const uint16_t* B, const float* bias, int gelu, float* out);

#ifdef __cplusplus
}
#endif
#endif /* OLPT_H */
