// C++ drop-in for the OpenLPT tracking classes on the B200 library.
//
// Same class and method names, argument meaning and error behaviour as the
// reference's C++ API for the reconstruction path (inc/libMath/Camera.h,
// inc/libMath/ImageIO.h, inc/libSTB/{Config,OTF,ObjectFinder,StereoMatch,Shake,IPR,STB}.h,
// inc/libObject/ObjectInfo.h); the numerical work runs in libolpt_cuda.so through
// its C ABI (include/olpt.h).  Differences on purpose: classes live in namespace
// `lpt`; images keep their integer sample type (no conversion to double on load);
// errors are lpt::FatalError exceptions carrying the library's status and message.
#pragma once
#include <array>
#include <cstdint>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/olpt.h"

namespace lpt {

// ---------------------------------------------------------------- errors
struct FatalError : std::runtime_error {
  int code;
  FatalError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ---------------------------------------------------------------- basic types
struct Pt2D {
  std::array<double, 2> v{0.0, 0.0};
  Pt2D() = default;
  Pt2D(double x, double y) : v{x, y} {}
  double& operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
};

struct Pt3D {
  std::array<double, 3> v{0.0, 0.0, 0.0};
  Pt3D() = default;
  Pt3D(double x, double y, double z) : v{x, y, z} {}
  double& operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
};

// AxisLimit (inc/libMath/STBCommons.h:118-151)
struct AxisLimit {
  double x_min = 0, x_max = 0, y_min = 0, y_max = 0, z_min = 0, z_max = 0;
  bool check(double x, double y, double z) const {
    return !(x > x_max || x < x_min || y > y_max || y < y_min || z > z_max || z < z_min);
  }
};

// Image (Matrix<double> in the reference, inc/libMath/Matrix.h:171): row-major
// samples of type u8, u16 or f64.
class Image {
 public:
  Image() = default;
  Image(int n_row, int n_col, double val = 0.0);
  static Image fromU8(int n_row, int n_col, const uint8_t* data);
  static Image fromU16(int n_row, int n_col, const uint16_t* data);
  static Image fromF64(int n_row, int n_col, const double* data);
  int getDimRow() const { return n_row_; }
  int getDimCol() const { return n_col_; }
  olpt_dtype_t dtype() const { return dtype_; }
  const void* data() const { return buf_.data(); }
  void* data() { return buf_.data(); }
  double operator()(int r, int c) const;
  void set(int r, int c, double v);
  std::vector<double> toDouble() const;
  void save(const std::string& path) const;  // TIFF: 8-bit for u8, else 16-bit

 private:
  int n_row_ = 0, n_col_ = 0;
  olpt_dtype_t dtype_ = OLPT_F64;
  std::vector<uint8_t> buf_;
};

// ImageIO (inc/libMath/ImageIO.h): the image list of one camera (one path per line,
// prefixed by the folder) and TIFF loading.
class ImageIO {
 public:
  ImageIO() = default;
  ImageIO(const std::string& folder, const std::string& list) { loadImgPath(folder, list); }
  void loadImgPath(const std::string& folder, const std::string& list);
  Image loadImg(int img_id);
  void saveImg(const std::string& path, const Image& img) const { img.save(path); }
  int getCurrImgID() const { return img_id_; }
  const std::vector<std::string>& getImgPath() const { return paths_; }

 private:
  std::vector<std::string> paths_;
  int img_id_ = -1;
};

// ---------------------------------------------------------------- camera / OTF
// Camera (inc/libMath/Camera.h:78-174): PINHOLE and POLYNOMIAL models.
class Camera {
 public:
  Camera() = default;
  explicit Camera(const std::string& file) { loadParameters(file); }
  void loadParameters(const std::string& file);
  int getNRow() const { return desc_.n_row; }
  int getNCol() const { return desc_.n_col; }
  Pt2D project(const Pt3D& pt_world) const;
  std::pair<Pt3D, Pt3D> lineOfSight(const Pt2D& pt_img) const;  // (point, unit vector)
  olpt_camera_desc desc() const;  // coefficient pointers refer to this object
  bool _is_active = true;
  double _max_intensity = 255;

 private:
  olpt_camera_desc desc_{};
  std::vector<double> u_, v_;  // polynomial coefficient tables
};

// OTF (inc/libSTB/OTF.h:33-78): a, b, c, alpha on an nx x ny x nz grid per camera.
struct OTFParam {
  int n_cam = 0, nx = 2, ny = 2, nz = 2, n_grid = 8;
  AxisLimit boundary;
  std::vector<double> a, b, c, alpha;  // n_cam x n_grid
};
class OTF {
 public:
  OTF() = default;
  explicit OTF(const std::string& file) { loadParam(file); }
  void loadParam(int n_cam, int nx, int ny, int nz, const AxisLimit& boundary,
                 const std::vector<Camera>& cams);
  void loadParam(const std::string& file);
  void saveParam(const std::string& file) const;
  std::vector<double> table() const;  // [4][n_cam][n_grid]
  OTFParam _param;
};

// ---------------------------------------------------------------- objects
enum class ObjFlag : uint8_t { None = 0, Ghost = 1, Repeated = 2 };

struct Object2D {
  Pt2D _pt_center;
  virtual ~Object2D() = default;
  virtual std::unique_ptr<Object2D> clone() const = 0;
};
struct Tracer2D : Object2D {
  double _r_px = 2;
  std::unique_ptr<Object2D> clone() const override { return std::make_unique<Tracer2D>(*this); }
};

struct Object3D {
  Pt3D _pt_center;
  std::vector<std::unique_ptr<Object2D>> _obj2d_list;
  bool _is_tracked = false;
  virtual ~Object3D() = default;
  void projectObject2D(const std::vector<Camera>& cams);
  bool isReconstructable(const std::vector<Camera>& cams);
  virtual void saveObject3D(std::ostream& out) const = 0;
};
struct Tracer3D : Object3D {
  double _r2d_px = 2;
  void saveObject3D(std::ostream& out) const override;
};

// ---------------------------------------------------------------- configuration
// BasicSetting (inc/libSTB/Config.h:160-205, src/srcSTB/Config.cpp:8-150)
struct BasicSetting {
  int _frame_start = 0, _frame_end = 0, _fps = 0, _n_thread = 0, _n_cam = 0;
  std::vector<Camera> _cam_list;
  std::vector<std::string> _image_file_paths;
  AxisLimit _axis_limit;
  double _voxel_to_mm = 1;
  std::string _output_path;
  std::vector<std::string> _object_types, _object_config_paths;
  bool _load_track = false;
  int _load_track_frame = 0;
  std::string _load_track_path;
  bool readConfig(const std::string& config_path);
};

struct STBParam {
  double _radius_search_obj = 0;
  int _n_initial_frames = 4;
  double _radius_search_track = 0;
};
struct ShakeParam {
  double _shake_width = 0, _shakewidth_min = 0;
  int _n_shake_loop = 4;
  double _thred_ghost = 0.1;
  int _ratio_augimg = 2;
};
struct PFParam {
  AxisLimit limit;
  int nx = 2, ny = 2, nz = 2;
  double r = 0;
  int nBin_x = 11, nBin_y = 11, nBin_z = 11;
  bool is_smooth = true;
  double sigma_x = 1.0, sigma_y = 1.0, sigma_z = 1.0;
};
struct SMParam {
  int match_cam_count = 4;
  int idmap_cell_px = 4;
  double tol_2d_px = 1.0, tol_3d_mm = 2.4e-2;
  AxisLimit limit;
};
struct IPRParam {
  int n_cam_reduced = 1, n_loop_ipr = 4, n_loop_ipr_reduced = 2;
  int64_t n_obj2d_process_max = 200000;
};

enum class ObjectKind { Tracer = 0, Bubble = 1 };

// ObjectConfig (inc/libSTB/Config.h:154-189): the parameters every object type
// shares (STB, shake, predictive field, IPR, stereo matching).  The hot-path classes
// take it by reference as the reference's do; only tracers are built here, so they
// check the kind and throw FatalError(OLPT_ERR_UNSUPPORTED) for any other.
struct ObjectConfig {
  STBParam _stb_param;
  ShakeParam _shake_param;
  PFParam _pf_param;
  SMParam _sm_param;
  IPRParam _ipr_param;
  // precision of the shake and residual: 0 = FP32 (default), 1 = FP64 (the reference's)
  int precision = 0;
  virtual ~ObjectConfig() = default;
  virtual bool readConfig(const std::string& filepath, BasicSetting& settings) = 0;
  virtual ObjectKind kind() const = 0;
  virtual std::unique_ptr<Object3D> creatObject3D(const Pt3D& center) const = 0;
};

// TracerConfig (inc/libSTB/Config.h:191-205): readCommonConfig + tracer fields; the
// OTF is estimated from the first frames as in TracerConfig::readConfig.
struct TracerConfig : ObjectConfig {
  int _min_obj_int = 30;
  double _radius_obj = 2;
  OTF _otf;
  bool readConfig(const std::string& filepath, BasicSetting& settings) override;
  ObjectKind kind() const override { return ObjectKind::Tracer; }
  std::unique_ptr<Object3D> creatObject3D(const Pt3D& center) const override;
  olpt_ipr_params iprParams() const;
};

// The tracer configuration behind an ObjectConfig reference; FatalError for other kinds.
const TracerConfig& tracer_config(const ObjectConfig& cfg);
TracerConfig& tracer_config(ObjectConfig& cfg);

// ---------------------------------------------------------------- hot path
class ObjectFinder2D {
 public:
  std::vector<std::unique_ptr<Object2D>> findObject2D(const Image& img, const ObjectConfig& cfg);
};

class StereoMatch {
 public:
  StereoMatch(const std::vector<Camera>& cams,
              const std::vector<std::vector<std::unique_ptr<Object2D>>>& obj2d_list,
              const ObjectConfig& cfg);
  std::vector<std::unique_ptr<Object3D>> match() const;

 private:
  const std::vector<Camera>& cams_;
  const std::vector<std::vector<std::unique_ptr<Object2D>>>& obj2d_;
  const TracerConfig& cfg_;
};

class Shake {
 public:
  Shake(const std::vector<Camera>& cams, const ObjectConfig& cfg)
      : cams_(cams), cfg_(tracer_config(cfg)) {}
  std::vector<ObjFlag> runShake(std::vector<std::unique_ptr<Object3D>>& objs,
                                const std::vector<Image>& img_orig);
  std::vector<Image> calResidualImage(const std::vector<std::unique_ptr<Object3D>>& objs,
                                      const std::vector<Image>& img_orig,
                                      const std::vector<ObjFlag>* flags = nullptr);

 private:
  const std::vector<Camera>& cams_;
  const TracerConfig& cfg_;
};

class IPR {
 public:
  explicit IPR(std::vector<Camera>& cams) : cams_(cams) {}
  std::vector<std::unique_ptr<Object3D>> runIPR(ObjectConfig& cfg, std::vector<Image> images);
  void saveObjInfo(const std::string& file, const std::vector<std::unique_ptr<Object3D>>& objs,
                   const ObjectConfig& cfg) const;

 private:
  std::vector<Camera>& cams_;
};

// One track of the STB lists (inc/libSTB/Track.h).
struct Track {
  std::vector<Pt3D> _pt_list;
  std::vector<int> _t_list;
};

class STB {
 public:
  // precision: 0 = FP32 shake and residual (default), 1 = FP64 (the reference's)
  STB(const BasicSetting& setting, const std::string& type, const std::string& obj_cfg_path,
      int precision = 0);
  ~STB();
  STB(STB&&) noexcept;
  STB& operator=(STB&&) = delete;
  void processFrame(int frame_id, std::vector<Image>& img_list);
  void saveTracksAll(const std::string& folder, int frame);
  void loadTracksAll(const std::string& folder, int frame);
  // which: "LongTrackActive", "ShortTrackActive", "LongTrackInactive", "ExitTrack"
  void saveTracks(const std::string& file, const std::string& which);
  void loadTracks(const std::string& file, const std::string& which);
  std::vector<Track> tracks(const std::string& which) const;
  size_t count(const std::string& which) const;
  BasicSetting _basic_setting;
  TracerConfig _obj_config;

 private:
  olpt_ctx* ctx_ = nullptr;
};

// The command-line pipeline (src/main.cpp:40-140): read the main config, build
// one STB per object type, loop over frames.
int run(const std::string& config_path);

// Shared device context of the calling thread (cameras and OTF uploaded per call).
olpt_ctx* default_context();
void check(olpt_ctx* ctx, olpt_status_t st);
void upload_rig(olpt_ctx* ctx, const std::vector<Camera>& cams, const OTF* otf);
void upload_images(olpt_ctx* ctx, const std::vector<Image>& imgs);

}  // namespace lpt
