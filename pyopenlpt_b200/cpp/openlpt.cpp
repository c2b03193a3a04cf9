// C++ drop-in classes over the C ABI (see openlpt.hpp).  Host code only: parsing of
// the reference's text formats, bookkeeping of the object classes, and the calls
// into libolpt_cuda.so; every numerical step of the path runs on the device.
#include "openlpt.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>

#include "tiff.hpp"

namespace lpt {

// ---------------------------------------------------------------- context
void check(olpt_ctx* ctx, olpt_status_t st) {
  if (st != OLPT_OK)
    throw FatalError((int)st, std::string("B200 library: ") + (ctx ? olpt_last_error(ctx) : ""));
}

namespace {
struct CtxHolder {
  olpt_ctx* c = nullptr;
  ~CtxHolder() {
    if (c) olpt_ctx_destroy(c);
  }
};

olpt_ctx* new_context() {
  olpt_ctx* c = nullptr;
  const olpt_status_t st = olpt_ctx_create(&c, 0);
  if (st != OLPT_OK)
    throw FatalError((int)st, "B200 library: no usable CUDA device (this implementation has no "
                              "CPU path)");
  return c;
}

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  const size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

// Config-file lines: trimmed, '#' comments dropped (src/srcSTB/Config.cpp:17-37).
std::vector<std::string> config_lines(const std::string& path) {
  std::ifstream file(path);
  if (!file.is_open())
    throw FatalError(OLPT_ERR_INVALID_ARG, "Config Error: Cannot open file " + path);
  std::vector<std::string> lines;
  std::string line;
  while (std::getline(file, line)) {
    line = trim(line);
    if (line.empty()) continue;
    const size_t c = line.find('#');
    if (c == 0) continue;
    if (c != std::string::npos) line.erase(c);
    line = trim(line);
    if (!line.empty()) lines.push_back(line);
  }
  return lines;
}

// File contents with '#' comments cut and lines joined by tabs, as the camera and
// OTF readers stream them (Camera.cpp:311-338, OTF.cpp:195-212).
std::stringstream comment_stripped(const std::string& path, const std::string& what) {
  std::ifstream in(path);
  if (!in) throw FatalError(OLPT_ERR_INVALID_ARG, what + ": cannot open file: " + path);
  std::stringstream out;
  std::string line;
  while (std::getline(in, line)) {
    const size_t c = line.find('#');
    if (c == 0) continue;
    if (c != std::string::npos) line.erase(c);
    out << line << '\t';
  }
  return out;
}

// Matrix<double>(rows, cols, istream) (Matrix.hpp:102-116): values with one
// optional ',' after each.
void read_values(std::istream& is, int n, double* out) {
  for (int i = 0; i < n; ++i) {
    double v = 0;
    is >> v;
    out[i] = v;
    if (is.peek() == ',') is.ignore();
  }
}

// A camera for calls that only need the image geometry (detection).
olpt_camera_desc dummy_camera(int n_row, int n_col) {
  olpt_camera_desc d{};
  d.type = 0;
  d.n_row = n_row;
  d.n_col = n_col;
  d.is_active = 1;
  d.cam_mtx[0] = d.cam_mtx[4] = d.cam_mtx[8] = 1.0;
  d.r_mtx[0] = d.r_mtx[4] = d.r_mtx[8] = 1.0;
  d.r_inv[0] = d.r_inv[4] = d.r_inv[8] = 1.0;
  return d;
}

// ImageIO::loadImgPath (src/srcMath/ImageIO.cpp): one path per line.
std::vector<std::string> image_list(const std::string& list_file) {
  std::ifstream in(list_file);
  if (!in) throw FatalError(OLPT_ERR_INVALID_ARG, "cannot open image list " + list_file);
  std::vector<std::string> out;
  std::string line;
  while (std::getline(in, line)) {
    line = trim(line);
    if (!line.empty()) out.push_back(line);
  }
  return out;
}

// ImageIO::loadImg: images are kept in their stored type (8/16-bit integer, or
// 32-bit float widened to double).
Image load_image(const std::string& path) {
  TiffImage t;
  try {
    t = read_tiff(path);
  } catch (const std::exception& e) {
    throw FatalError(OLPT_ERR_INVALID_ARG, e.what());
  }
  if (t.bits == 8) return Image::fromU8(t.rows, t.cols, t.data.data());
  if (t.bits == 16)
    return Image::fromU16(t.rows, t.cols, reinterpret_cast<const uint16_t*>(t.data.data()));
  std::vector<double> d((size_t)t.rows * t.cols);
  const float* f = reinterpret_cast<const float*>(t.data.data());
  for (size_t i = 0; i < d.size(); ++i) d[i] = f[i];
  return Image::fromF64(t.rows, t.cols, d.data());
}

}  // namespace

olpt_ctx* default_context() {
  thread_local CtxHolder h;
  if (!h.c) h.c = new_context();
  return h.c;
}

void upload_rig(olpt_ctx* ctx, const std::vector<Camera>& cams, const OTF* otf) {
  std::vector<olpt_camera_desc> d;
  d.reserve(cams.size());
  for (const Camera& c : cams) {
    d.push_back(c.desc());
    d.back().is_active = c._is_active ? 1 : 0;
  }
  check(ctx, olpt_cameras_upload(ctx, d.data(), (int)d.size()));
  if (otf && otf->_param.n_cam == (int)cams.size()) {
    const OTFParam& p = otf->_param;
    const double b6[6] = {p.boundary.x_min, p.boundary.x_max, p.boundary.y_min,
                          p.boundary.y_max, p.boundary.z_min, p.boundary.z_max};
    const std::vector<double> t = otf->table();
    check(ctx, olpt_otf_upload(ctx, p.nx, p.ny, p.nz, b6, t.data()));
  }
}

void upload_images(olpt_ctx* ctx, const std::vector<Image>& imgs) {
  if (imgs.empty()) throw FatalError(OLPT_ERR_INVALID_ARG, "no images");
  const olpt_dtype_t dt = imgs[0].dtype();
  bool same = true;
  for (const Image& im : imgs) same = same && im.dtype() == dt;
  std::vector<std::vector<double>> conv;
  conv.reserve(imgs.size());
  std::vector<const void*> ptr;
  std::vector<int> H, W;
  for (const Image& im : imgs) {
    H.push_back(im.getDimRow());
    W.push_back(im.getDimCol());
    if (same) {
      ptr.push_back(im.data());
    } else {
      conv.push_back(im.toDouble());
      ptr.push_back(conv.back().data());
    }
  }
  check(ctx, olpt_images_upload(ctx, (int)imgs.size(), same ? dt : OLPT_F64, ptr.data(), H.data(),
                                W.data(), nullptr, 0));
}

// ---------------------------------------------------------------- Image
Image::Image(int n_row, int n_col, double val) : n_row_(n_row), n_col_(n_col), dtype_(OLPT_F64) {
  buf_.resize((size_t)n_row * n_col * 8);
  double* p = reinterpret_cast<double*>(buf_.data());
  std::fill(p, p + (size_t)n_row * n_col, val);
}
Image Image::fromU8(int r, int c, const uint8_t* d) {
  Image im;
  im.n_row_ = r;
  im.n_col_ = c;
  im.dtype_ = OLPT_U8;
  im.buf_.assign(d, d + (size_t)r * c);
  return im;
}
Image Image::fromU16(int r, int c, const uint16_t* d) {
  Image im;
  im.n_row_ = r;
  im.n_col_ = c;
  im.dtype_ = OLPT_U16;
  im.buf_.resize((size_t)r * c * 2);
  std::memcpy(im.buf_.data(), d, im.buf_.size());
  return im;
}
Image Image::fromF64(int r, int c, const double* d) {
  Image im;
  im.n_row_ = r;
  im.n_col_ = c;
  im.dtype_ = OLPT_F64;
  im.buf_.resize((size_t)r * c * 8);
  std::memcpy(im.buf_.data(), d, im.buf_.size());
  return im;
}
double Image::operator()(int r, int c) const {
  const size_t i = (size_t)r * n_col_ + c;
  switch (dtype_) {
    case OLPT_U8: return buf_[i];
    case OLPT_U16: return reinterpret_cast<const uint16_t*>(buf_.data())[i];
    case OLPT_F32: return reinterpret_cast<const float*>(buf_.data())[i];
    default: return reinterpret_cast<const double*>(buf_.data())[i];
  }
}
void Image::set(int r, int c, double v) {
  if (dtype_ != OLPT_F64) {
    const std::vector<double> d = toDouble();
    *this = fromF64(n_row_, n_col_, d.data());
  }
  reinterpret_cast<double*>(buf_.data())[(size_t)r * n_col_ + c] = v;
}
std::vector<double> Image::toDouble() const {
  std::vector<double> d((size_t)n_row_ * n_col_);
  for (int r = 0; r < n_row_; ++r)
    for (int c = 0; c < n_col_; ++c) d[(size_t)r * n_col_ + c] = (*this)(r, c);
  return d;
}
void Image::save(const std::string& path) const {
  TiffImage t;
  t.rows = n_row_;
  t.cols = n_col_;
  if (dtype_ == OLPT_U8) {
    t.bits = 8;
    t.data = buf_;
  } else {
    t.bits = 16;
    t.data.resize((size_t)n_row_ * n_col_ * 2);
    uint16_t* p = reinterpret_cast<uint16_t*>(t.data.data());
    for (int r = 0; r < n_row_; ++r)
      for (int c = 0; c < n_col_; ++c) {
        const double v = std::round((*this)(r, c));
        p[(size_t)r * n_col_ + c] = (uint16_t)std::min(65535.0, std::max(0.0, v));
      }
  }
  try {
    write_tiff(path, t);
  } catch (const std::exception& e) {
    throw FatalError(OLPT_ERR_INVALID_ARG, e.what());
  }
}

void ImageIO::loadImgPath(const std::string& folder, const std::string& list) {
  paths_.clear();
  for (const std::string& p : image_list(folder + list)) paths_.push_back(folder + p);
  img_id_ = -1;
}

Image ImageIO::loadImg(int img_id) {
  if (img_id < 0 || img_id >= (int)paths_.size())
    throw FatalError(OLPT_ERR_INVALID_ARG, "ImageIO::loadImg: image index out of range");
  img_id_ = img_id;
  return load_image(paths_[img_id]);
}

// ---------------------------------------------------------------- Camera
// Camera::loadParameters (src/srcMath/Camera.cpp:19-158, 311-338)
void Camera::loadParameters(const std::string& file) {
  std::stringstream is = comment_stripped(file, "Camera::loadParameters");
  desc_ = olpt_camera_desc{};
  u_.clear();
  v_.clear();
  std::string type, useless, tok;
  is >> type;
  auto size_pair = [&](const std::string& s, int& r, int& c) {
    std::stringstream ss(s);
    std::string t;
    std::getline(ss, t, ',');
    r = std::stoi(t);
    std::getline(ss, t, ',');
    c = std::stoi(t);
  };
  try {
    if (type == "PINHOLE") {
      desc_.type = 0;
      is >> useless >> useless >> tok;
      size_pair(tok, desc_.n_row, desc_.n_col);
      read_values(is, 9, desc_.cam_mtx);
      is >> tok;
      std::stringstream ss(tok);
      double d;
      int id = 0;
      bool distorted = false;
      while (ss >> d) {
        if (id < 12) desc_.dist[id] = d;
        ++id;
        if (d > 1e-8) distorted = true;
        if (ss.peek() == ',') ss.ignore();
      }
      if (distorted && id != 4 && id != 5 && id != 8 && id != 12)
        throw FatalError(OLPT_ERR_INVALID_ARG,
                         "Camera::loadParameters: number of distortion coefficients is wrong: " +
                             std::to_string(id));
      desc_.n_dist = std::min(id, 12);
      is >> useless;
      read_values(is, 9, desc_.r_mtx);
      read_values(is, 9, desc_.r_inv);
      read_values(is, 3, desc_.t_vec);
      read_values(is, 3, desc_.t_inv);
    } else if (type == "POLYNOMIAL") {
      desc_.type = 1;
      is >> useless >> tok;
      size_pair(tok, desc_.n_row, desc_.n_col);
      is >> tok;
      std::stringstream ss(tok);
      std::string t;
      std::getline(ss, t, ',');
      if (t == "REF_X")
        desc_.ref_plane = 1;
      else if (t == "REF_Y")
        desc_.ref_plane = 2;
      else if (t == "REF_Z")
        desc_.ref_plane = 3;
      else
        throw FatalError(OLPT_ERR_INVALID_ARG,
                         "Camera::loadParameters: reference plane is wrong: " + t);
      std::getline(ss, t, ',');
      desc_.plane[0] = std::stod(t);
      std::getline(ss, t, ',');
      desc_.plane[1] = std::stod(t);
      is >> desc_.n_coeff;
      u_.resize(4 * (size_t)desc_.n_coeff);
      v_.resize(4 * (size_t)desc_.n_coeff);
      read_values(is, 4 * desc_.n_coeff, u_.data());
      read_values(is, 4 * desc_.n_coeff, v_.data());
    } else {
      throw FatalError(OLPT_ERR_UNSUPPORTED,
                       "Camera::loadParameters: unsupported camera type: " + type +
                           " (PINHOLE and POLYNOMIAL are on this path)");
    }
  } catch (const FatalError&) {
    throw;
  } catch (const std::exception& e) {
    throw FatalError(OLPT_ERR_INVALID_ARG,
                     "Camera::loadParameters: malformed file " + file + ": " + e.what());
  }
  desc_.is_active = 1;
}

olpt_camera_desc Camera::desc() const {
  olpt_camera_desc d = desc_;
  d.u_coeffs = u_.empty() ? nullptr : u_.data();
  d.v_coeffs = v_.empty() ? nullptr : v_.data();
  return d;
}

Pt2D Camera::project(const Pt3D& p) const {
  olpt_ctx* ctx = default_context();
  olpt_camera_desc d = desc();
  check(ctx, olpt_cameras_upload(ctx, &d, 1));
  double uv[2];
  check(ctx, olpt_camera_project(ctx, 0, 1, p.v.data(), uv));
  return Pt2D(uv[0], uv[1]);
}

std::pair<Pt3D, Pt3D> Camera::lineOfSight(const Pt2D& q) const {
  olpt_ctx* ctx = default_context();
  olpt_camera_desc d = desc();
  check(ctx, olpt_cameras_upload(ctx, &d, 1));
  double l[6];
  check(ctx, olpt_camera_los(ctx, 0, 1, q.v.data(), l));
  return {Pt3D(l[0], l[1], l[2]), Pt3D(l[3], l[4], l[5])};
}

// ---------------------------------------------------------------- OTF
// OTF::loadParam(n_cam, nx, ny, nz, boundary, cams) (src/srcSTB/OTF.cpp:160-193)
void OTF::loadParam(int n_cam, int nx, int ny, int nz, const AxisLimit& boundary,
                    const std::vector<Camera>& cams) {
  nx = std::max(nx, 2);
  ny = std::max(ny, 2);
  nz = std::max(nz, 2);
  OTFParam& p = _param;
  p.n_cam = n_cam;
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  p.n_grid = nx * ny * nz;
  p.boundary = boundary;
  p.a.assign((size_t)n_cam * p.n_grid, 0.0);
  for (int c = 0; c < n_cam; ++c)
    for (int g = 0; g < p.n_grid; ++g) p.a[(size_t)c * p.n_grid + g] = cams[c]._max_intensity / 2.0;
  p.b.assign((size_t)n_cam * p.n_grid, 1.5);
  p.c.assign((size_t)n_cam * p.n_grid, 1.5);
  p.alpha.assign((size_t)n_cam * p.n_grid, 0.0);
}

// OTF::loadParam(file) (src/srcSTB/OTF.cpp:195-243)
void OTF::loadParam(const std::string& file) {
  std::stringstream in = comment_stripped(file, "OTF::loadParam");
  OTFParam& p = _param;
  in >> p.n_cam;
  in.ignore();
  in >> p.nx;
  in.ignore();
  in >> p.ny;
  in.ignore();
  in >> p.nz;
  in.ignore();
  in >> p.n_grid;
  double b[6];
  for (int k = 0; k < 6; ++k) {
    in >> b[k];
    if (k < 5) in.ignore();
  }
  p.boundary = AxisLimit{b[0], b[1], b[2], b[3], b[4], b[5]};
  if (!in || p.n_cam <= 0 || p.n_grid <= 0)
    throw FatalError(OLPT_ERR_INVALID_ARG, "OTF::loadParam: malformed file " + file);
  for (std::vector<double>* m : {&p.a, &p.b, &p.c, &p.alpha}) {
    m->resize((size_t)p.n_cam * p.n_grid);
    read_values(in, (int)m->size(), m->data());
  }
  if (!in) throw FatalError(OLPT_ERR_INVALID_ARG, "OTF::loadParam: malformed file " + file);
}

// OTF::saveParam (src/srcSTB/OTF.cpp:245-271)
void OTF::saveParam(const std::string& file) const {
  std::ofstream out(file);
  if (!out) throw FatalError(OLPT_ERR_INVALID_ARG, "Cannot save OTF to file " + file);
  const OTFParam& p = _param;
  out << "# Size: (n_cam,nx,ny,nz,n_grid)\n"
      << p.n_cam << ',' << p.nx << ',' << p.ny << ',' << p.nz << ',' << p.n_grid << '\n';
  out << "# Boundary: (xmin,xmax,ymin,ymax,zmin,zmax)\n"
      << p.boundary.x_min << ',' << p.boundary.x_max << ',' << p.boundary.y_min << ','
      << p.boundary.y_max << ',' << p.boundary.z_min << ',' << p.boundary.z_max << '\n';
  const char* names[4] = {"a", "b", "c", "alpha"};
  const std::vector<double>* mats[4] = {&p.a, &p.b, &p.c, &p.alpha};
  for (int k = 0; k < 4; ++k) {
    out << "# " << names[k] << ": (n_cam,n_grid)\n";
    out.setf(std::ios_base::scientific);
    out.precision(8);
    for (int c = 0; c < p.n_cam; ++c)
      for (int g = 0; g < p.n_grid; ++g)
        out << (*mats[k])[(size_t)c * p.n_grid + g] << (g + 1 < p.n_grid ? "," : "\n");
  }
}

std::vector<double> OTF::table() const {
  const OTFParam& p = _param;
  std::vector<double> t;
  t.reserve(4 * p.a.size());
  for (const std::vector<double>* m : {&p.a, &p.b, &p.c, &p.alpha})
    t.insert(t.end(), m->begin(), m->end());
  return t;
}

// ---------------------------------------------------------------- objects
void Object3D::projectObject2D(const std::vector<Camera>& cams) {
  olpt_ctx* ctx = default_context();
  upload_rig(ctx, cams, nullptr);
  _obj2d_list.clear();
  const Tracer3D* t3 = dynamic_cast<const Tracer3D*>(this);
  for (size_t c = 0; c < cams.size(); ++c) {
    double uv[2];
    check(ctx, olpt_camera_project(ctx, (int)c, 1, _pt_center.v.data(), uv));
    auto t = std::make_unique<Tracer2D>();
    t->_pt_center = Pt2D(uv[0], uv[1]);
    if (t3) t->_r_px = t3->_r2d_px;
    _obj2d_list.push_back(std::move(t));
  }
}

// Object3D::isReconstructable (src/srcObject/ObjectInfo.cpp:3-30; y is compared
// with the column count there, kept as is)
bool Object3D::isReconstructable(const std::vector<Camera>& cams) {
  projectObject2D(cams);
  const int n = (int)cams.size();
  int n_out = 0;
  for (int i = 0; i < n; ++i) {
    const double x = _obj2d_list[i]->_pt_center[0], y = _obj2d_list[i]->_pt_center[1];
    if (x < 0 || x >= cams[i].getNCol() || y < 0 || y >= cams[i].getNCol()) {
      ++n_out;
      if (n - n_out < 2) return false;
    }
  }
  return true;
}

// Tracer3D::saveObject3D (src/srcObject/ObjectInfo.cpp:76-94)
void Tracer3D::saveObject3D(std::ostream& out) const {
  out << _pt_center[0] << "," << _pt_center[1] << "," << _pt_center[2];
  for (const auto& o : _obj2d_list) {
    if (o)
      out << "," << o->_pt_center[0] << "," << o->_pt_center[1];
    else
      out << ",,";
  }
  out << "\n";
}

// ---------------------------------------------------------------- configuration
// BasicSetting::readConfig (src/srcSTB/Config.cpp:8-150)
bool BasicSetting::readConfig(const std::string& config_path) {
  std::vector<std::string> lines;
  try {
    lines = config_lines(config_path);
  } catch (const FatalError&) {
    std::cerr << "Failed to open config file: " << config_path << std::endl;
    return false;
  }
  if (lines.size() < 11) {
    std::cerr << "Invalid config: too few lines." << std::endl;
    return false;
  }
  size_t id = 0;
  auto next = [&]() -> const std::string& {
    if (id >= lines.size())
      throw FatalError(OLPT_ERR_INVALID_ARG, "Invalid config: too few lines in " + config_path);
    return lines[id++];
  };
  std::string tok;
  try {
    {
      std::stringstream ss(next());
      std::getline(ss, tok, ',');
      _frame_start = std::stoi(tok);
      std::getline(ss, tok, ',');
      _frame_end = std::stoi(tok);
    }
    _fps = std::stoi(next());
    _n_thread = std::stoi(next());
    _n_cam = std::stoi(next());
    _cam_list.clear();
    for (int i = 0; i < _n_cam; ++i) {
      std::stringstream ss(next());
      std::string path;
      std::getline(ss, path, ',');
      std::getline(ss, tok, ',');
      Camera cam(path);
      cam._max_intensity = std::stoi(tok);
      cam._is_active = true;
      _cam_list.push_back(cam);
    }
    _image_file_paths.clear();
    for (int i = 0; i < _n_cam; ++i) _image_file_paths.push_back(next());
    {
      std::stringstream ss(next());
      double v[6];
      for (int k = 0; k < 6; ++k) {
        std::getline(ss, tok, ',');
        v[k] = std::stod(tok);
      }
      _axis_limit = AxisLimit{v[0], v[1], v[2], v[3], v[4], v[5]};
    }
    _voxel_to_mm = std::stod(next());
    _output_path = next();
    if (!_output_path.empty() && _output_path.back() != '/' && _output_path.back() != '\\')
      _output_path.push_back('/');
    _object_types.clear();
    {
      std::stringstream ss(next());
      while (std::getline(ss, tok, ','))
        if (!tok.empty()) _object_types.push_back(tok);
    }
    _object_config_paths.clear();
    for (size_t i = 0; i < _object_types.size(); ++i) _object_config_paths.push_back(next());
    {
      std::stringstream ss(next());
      std::getline(ss, tok, ',');
      _load_track = std::stoi(tok) != 0;
      _load_track_frame = _frame_start;
      if (_load_track) {
        if (std::getline(ss, tok, ',') && !tok.empty()) _load_track_frame = std::stoi(tok);
        if (id < lines.size()) _load_track_path = lines[id++];
      }
    }
  } catch (const FatalError&) {
    throw;
  } catch (const std::exception& e) {
    throw FatalError(OLPT_ERR_INVALID_ARG,
                     "Invalid config " + config_path + ": " + std::string(e.what()));
  }
  if (_n_cam <= 0) throw FatalError(OLPT_ERR_INVALID_ARG, "Invalid n_cam in config: " + config_path);
  if (_frame_end < _frame_start)
    throw FatalError(OLPT_ERR_INVALID_ARG, "Invalid frame range in config: " + config_path);
  if (_object_types.size() != _object_config_paths.size())
    throw FatalError(OLPT_ERR_INVALID_ARG,
                     "Object type count != config path count in config: " + config_path);
  if (_n_thread < 0) _n_thread = 0;
  return true;
}

namespace {
// myMATH::inverse with the Gauss method for a 2 x 2 matrix (inc/libMath/myMATH.h:182-255).
// OTF::estimateUniformOTFFromImage (src/srcSTB/OTF.cpp:17-144) through
// olpt_otf_estimate: the camera's images as the context's planes, detections, the
// reference's selection of at most 1000 per image and its least squares on the device.
void estimate_otf(OTF& otf, int cam_id, const TracerConfig& cfg, const std::vector<Image>& imgs) {
  olpt_ctx* ctx = default_context();
  std::vector<olpt_camera_desc> d;
  for (const Image& im : imgs) d.push_back(dummy_camera(im.getDimRow(), im.getDimCol()));
  check(ctx, olpt_cameras_upload(ctx, d.data(), (int)d.size()));
  upload_images(ctx, imgs);
  double abc[3];
  int64_t n = 0;
  check(ctx, olpt_otf_estimate(ctx, (double)cfg._min_obj_int, cfg._radius_obj, 1000, abc, &n));
  if (n == 0) {
    std::cerr << "[WARN] OTF calibration skipped: no tracer found | ctx: cam_id=" << cam_id
              << std::endl;
    return;
  }
  const double a = abc[0];
  const double coef[2] = {abc[1], abc[2]};
  OTFParam& p = otf._param;
  for (int g = 0; g < p.n_grid; ++g) {
    p.a[(size_t)cam_id * p.n_grid + g] = a;
    p.b[(size_t)cam_id * p.n_grid + g] = coef[0];
    p.c[(size_t)cam_id * p.n_grid + g] = coef[1];
    p.alpha[(size_t)cam_id * p.n_grid + g] = 0;
  }
}
}  // namespace

// ObjectConfig::readCommonConfig + TracerConfig::readConfig
// (src/srcSTB/Config.cpp:153-286)
bool TracerConfig::readConfig(const std::string& filepath, BasicSetting& settings) {
  const std::vector<std::string> lines = config_lines(filepath);
  size_t id = 0;
  auto next = [&]() -> const std::string& {
    if (id >= lines.size())
      throw FatalError(OLPT_ERR_INVALID_ARG, "Config Error: Failed to parse common config in " +
                                                 filepath);
    return lines[id++];
  };
  try {
    const double v2mm = settings._voxel_to_mm;
    _stb_param._radius_search_obj = std::stod(next()) * v2mm;
    _stb_param._n_initial_frames = std::max(4, std::stoi(next()));
    _stb_param._radius_search_track = std::stod(next()) * v2mm;
    _shake_param._shake_width = std::stod(next()) * v2mm;
    _shake_param._shakewidth_min = _shake_param._shake_width / 20;
    _pf_param.limit = settings._axis_limit;
    _pf_param.nx = std::stoi(next());
    _pf_param.ny = std::stoi(next());
    _pf_param.nz = std::stoi(next());
    _pf_param.r = std::stod(next()) * v2mm;
    _ipr_param.n_loop_ipr = std::stoi(next());
    _shake_param._n_shake_loop = std::stoi(next());
    _shake_param._thred_ghost = std::stod(next());
    _sm_param.tol_2d_px = std::stod(next());
    _sm_param.tol_3d_mm = std::stod(next()) * v2mm;
    _sm_param.match_cam_count = std::min(_sm_param.match_cam_count, settings._n_cam);
    _sm_param.limit = settings._axis_limit;
    _ipr_param.n_cam_reduced = std::stoi(next());
    _ipr_param.n_loop_ipr_reduced = std::stoi(next());
    _min_obj_int = std::stoi(next());
    _radius_obj = std::stod(next());
  } catch (const FatalError&) {
    throw;
  } catch (...) {
    throw FatalError(OLPT_ERR_INVALID_ARG, "Config Error: Failed to parse common config in " +
                                               filepath);
  }
  _otf.loadParam(settings._n_cam, 5, 5, 5, settings._axis_limit, settings._cam_list);
  const int n_img_otf = 5;
  for (int i = 0; i < settings._n_cam; ++i) {
    ImageIO io("", settings._image_file_paths[i]);
    std::vector<Image> imgs;
    for (int j = 0; j < n_img_otf; ++j) imgs.push_back(io.loadImg(settings._frame_start + j));
    estimate_otf(_otf, i, *this, imgs);
  }
  return true;
}

const TracerConfig& tracer_config(const ObjectConfig& cfg) {
  if (cfg.kind() != ObjectKind::Tracer)
    throw FatalError(OLPT_ERR_UNSUPPORTED, "only tracer objects are supported by this library");
  return static_cast<const TracerConfig&>(cfg);
}

TracerConfig& tracer_config(ObjectConfig& cfg) {
  return const_cast<TracerConfig&>(tracer_config(static_cast<const ObjectConfig&>(cfg)));
}

std::unique_ptr<Object3D> TracerConfig::creatObject3D(const Pt3D& center) const {
  auto t = std::make_unique<Tracer3D>();
  t->_pt_center = center;
  t->_r2d_px = _radius_obj;
  return t;
}

olpt_ipr_params TracerConfig::iprParams() const {
  olpt_ipr_params p{};
  p.min_obj_int = _min_obj_int;
  p.sm.match_cam_count = _sm_param.match_cam_count;
  p.sm.idmap_cell_px = _sm_param.idmap_cell_px;
  p.sm.tol_2d_px = _sm_param.tol_2d_px;
  p.sm.tol_3d_mm = _sm_param.tol_3d_mm;
  const AxisLimit& l = _sm_param.limit;
  const double lim[6] = {l.x_min, l.x_max, l.y_min, l.y_max, l.z_min, l.z_max};
  std::copy(lim, lim + 6, p.sm.limit);
  p.shake.shake_width = _shake_param._shake_width;
  p.shake.shakewidth_min = _shake_param._shakewidth_min;
  p.shake.n_shake_loop = _shake_param._n_shake_loop;
  p.shake.thred_ghost = _shake_param._thred_ghost;
  p.shake.ratio_augimg = _shake_param._ratio_augimg;
  p.shake.radius_obj = _radius_obj;
  p.shake.tol_3d_mm = _sm_param.tol_3d_mm;
  p.shake.precision = precision;
  p.n_cam_reduced = _ipr_param.n_cam_reduced;
  p.n_loop_ipr = _ipr_param.n_loop_ipr;
  p.n_loop_ipr_reduced = _ipr_param.n_loop_ipr_reduced;
  p.n_obj2d_process_max = _ipr_param.n_obj2d_process_max;
  return p;
}

// ---------------------------------------------------------------- hot path
std::vector<std::unique_ptr<Object2D>> ObjectFinder2D::findObject2D(const Image& img,
                                                                    const ObjectConfig& ocfg) {
  const TracerConfig& cfg = tracer_config(ocfg);
  olpt_ctx* ctx = default_context();
  olpt_camera_desc d = dummy_camera(img.getDimRow(), img.getDimCol());
  check(ctx, olpt_cameras_upload(ctx, &d, 1));
  upload_images(ctx, {img});
  int64_t cnt = 0;
  check(ctx, olpt_find_peaks(ctx, (double)cfg._min_obj_int, &cnt));
  std::vector<double> xy(2 * (size_t)cnt + 2);
  check(ctx, olpt_get_peaks(ctx, 0, xy.data(), nullptr, cnt));
  std::vector<std::unique_ptr<Object2D>> out;
  out.reserve(cnt);
  for (int64_t i = 0; i < cnt; ++i) {
    auto t = std::make_unique<Tracer2D>();
    t->_pt_center = Pt2D(xy[2 * i], xy[2 * i + 1]);
    t->_r_px = cfg._radius_obj;
    out.push_back(std::move(t));
  }
  return out;
}

StereoMatch::StereoMatch(const std::vector<Camera>& cams,
                         const std::vector<std::vector<std::unique_ptr<Object2D>>>& obj2d_list,
                         const ObjectConfig& cfg)
    : cams_(cams), obj2d_(obj2d_list), cfg_(tracer_config(cfg)) {
  if (obj2d_list.size() != cams.size())
    throw FatalError(OLPT_ERR_INVALID_ARG, "StereoMatch: obj2d_list size must equal n_cams");
}

std::vector<std::unique_ptr<Object3D>> StereoMatch::match() const {
  olpt_ctx* ctx = default_context();
  upload_rig(ctx, cams_, nullptr);
  const int C = (int)cams_.size();
  std::vector<std::vector<double>> xy(C);
  std::vector<int64_t> counts(C);
  std::vector<const double*> ptr(C);
  for (int c = 0; c < C; ++c) {
    for (const auto& o : obj2d_[c]) {
      xy[c].push_back(o->_pt_center[0]);
      xy[c].push_back(o->_pt_center[1]);
    }
    xy[c].push_back(0.0);  // never empty
    counts[c] = (int64_t)obj2d_[c].size();
    ptr[c] = xy[c].data();
  }
  check(ctx, olpt_detections_upload(ctx, C, counts.data(), ptr.data()));
  const olpt_ipr_params ip = cfg_.iprParams();
  int64_t n_cand = 0, n_match = 0;
  check(ctx, olpt_stereo_match(ctx, &ip.sm, &n_cand, &n_match));
  std::vector<int32_t> ids((size_t)n_match * C + 1);
  std::vector<double> X(3 * (size_t)n_match + 3);
  check(ctx, olpt_get_matches(ctx, ids.data(), X.data()));
  std::vector<std::unique_ptr<Object3D>> out;
  out.reserve(n_match);
  for (int64_t m = 0; m < n_match; ++m) {
    auto t = std::make_unique<Tracer3D>();
    t->_pt_center = Pt3D(X[3 * m], X[3 * m + 1], X[3 * m + 2]);
    t->_r2d_px = cfg_._radius_obj;
    for (int c = 0; c < C; ++c) {
      const int id = ids[(size_t)m * C + c];
      t->_obj2d_list.push_back(id >= 0 ? obj2d_[c][id]->clone() : nullptr);
    }
    out.push_back(std::move(t));
  }
  return out;
}

namespace {
void objects_to_device(olpt_ctx* ctx, const std::vector<std::unique_ptr<Object3D>>& objs) {
  std::vector<double> xyz;
  xyz.reserve(3 * objs.size() + 3);
  for (const auto& o : objs) xyz.insert(xyz.end(), o->_pt_center.v.begin(), o->_pt_center.v.end());
  xyz.resize(3 * objs.size() + 3);
  check(ctx, olpt_objects_upload(ctx, (int64_t)objs.size(), xyz.data()));
}

std::vector<Image> residual_images(olpt_ctx* ctx, const std::vector<Image>& like) {
  std::vector<Image> out;
  for (size_t c = 0; c < like.size(); ++c) {
    std::vector<double> d((size_t)like[c].getDimRow() * like[c].getDimCol());
    check(ctx, olpt_residual_download(ctx, (int)c, OLPT_F64, d.data()));
    out.push_back(Image::fromF64(like[c].getDimRow(), like[c].getDimCol(), d.data()));
  }
  return out;
}
}  // namespace

// Shake::runShake (src/srcSTB/Shake.cpp:36-163): objects move in place and get the
// projections of their final position.
std::vector<ObjFlag> Shake::runShake(std::vector<std::unique_ptr<Object3D>>& objs,
                                     const std::vector<Image>& img_orig) {
  olpt_ctx* ctx = default_context();
  upload_rig(ctx, cams_, &cfg_._otf);
  upload_images(ctx, img_orig);
  objects_to_device(ctx, objs);
  const size_t n = objs.size(), C = cams_.size();
  std::vector<ObjFlag> flags(n);
  if (n == 0) return flags;
  const olpt_ipr_params ip = cfg_.iprParams();
  check(ctx, olpt_shake(ctx, &ip.shake));
  std::vector<double> xyz(3 * n), uv(2 * C * n);
  std::vector<uint8_t> fl(n);
  check(ctx, olpt_objects_download(ctx, xyz.data(), uv.data(), fl.data(), nullptr));
  for (size_t i = 0; i < n; ++i) {
    objs[i]->_pt_center = Pt3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    objs[i]->_obj2d_list.clear();
    const Tracer3D* t3 = dynamic_cast<const Tracer3D*>(objs[i].get());
    for (size_t c = 0; c < C; ++c) {
      auto t = std::make_unique<Tracer2D>();
      t->_pt_center = Pt2D(uv[(i * C + c) * 2], uv[(i * C + c) * 2 + 1]);
      if (t3) t->_r_px = t3->_r2d_px;
      objs[i]->_obj2d_list.push_back(std::move(t));
    }
    flags[i] = (ObjFlag)fl[i];
  }
  return flags;
}

// Shake::calResidualImage (Shake.h:41-48, Shake.cpp:165-244 with output_ipr)
std::vector<Image> Shake::calResidualImage(const std::vector<std::unique_ptr<Object3D>>& objs,
                                           const std::vector<Image>& img_orig,
                                           const std::vector<ObjFlag>* flags) {
  olpt_ctx* ctx = default_context();
  upload_rig(ctx, cams_, &cfg_._otf);
  upload_images(ctx, img_orig);
  if (flags) {
    std::vector<std::unique_ptr<Object3D>> kept;
    for (size_t i = 0; i < objs.size() && i < flags->size(); ++i)
      if ((*flags)[i] == ObjFlag::None) kept.push_back(cfg_.creatObject3D(objs[i]->_pt_center));
    objects_to_device(ctx, kept);
  } else {
    objects_to_device(ctx, objs);
  }
  const olpt_ipr_params ip = cfg_.iprParams();
  check(ctx, olpt_residual(ctx, &ip.shake, 0, 0));
  return residual_images(ctx, img_orig);
}

std::vector<std::unique_ptr<Object3D>> IPR::runIPR(ObjectConfig& ocfg, std::vector<Image> images) {
  const TracerConfig& cfg = tracer_config(ocfg);
  olpt_ctx* ctx = default_context();
  upload_rig(ctx, cams_, &cfg._otf);
  upload_images(ctx, images);
  const olpt_ipr_params ip = cfg.iprParams();
  int64_t n = 0;
  check(ctx, olpt_ipr_run(ctx, &ip, &n));
  const size_t C = cams_.size();
  std::vector<double> xyz(3 * (size_t)n + 3), uv(2 * C * (size_t)n + 2);
  check(ctx, olpt_ipr_result(ctx, xyz.data(), uv.data()));
  std::vector<std::unique_ptr<Object3D>> out;
  for (int64_t i = 0; i < n; ++i) {
    auto t = std::make_unique<Tracer3D>();
    t->_pt_center = Pt3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    t->_r2d_px = cfg._radius_obj;
    for (size_t c = 0; c < C; ++c) {
      auto p = std::make_unique<Tracer2D>();
      p->_pt_center = Pt2D(uv[(i * C + c) * 2], uv[(i * C + c) * 2 + 1]);
      p->_r_px = cfg._radius_obj;
      t->_obj2d_list.push_back(std::move(p));
    }
    out.push_back(std::move(t));
  }
  return out;
}

// IPR::saveObjInfo (src/srcSTB/IPR.cpp:307-343): the tracer header (which names
// Error and Ncam columns the rows do not have), then Tracer3D::saveObject3D rows in
// the stream's default format.
void IPR::saveObjInfo(const std::string& file, const std::vector<std::unique_ptr<Object3D>>& objs,
                      const ObjectConfig&) const {
  std::ofstream out(file);
  if (!out) throw FatalError(OLPT_ERR_INVALID_ARG, "Cannot open file " + file);
  out << "WorldX,WorldY,WorldZ,Error,Ncam";
  for (size_t i = 0; i < cams_.size(); ++i)
    out << ",cam" << i << "_x(col)" << ",cam" << i << "_y(row)";
  out << "\n";
  for (const auto& o : objs)
    if (o) o->saveObject3D(out);
}

// ---------------------------------------------------------------- STB
namespace {
int list_id(const std::string& which) {
  if (which == "LongTrackActive") return OLPT_TRACK_LONG_ACTIVE;
  if (which == "ShortTrackActive") return OLPT_TRACK_SHORT_ACTIVE;
  if (which == "LongTrackInactive") return OLPT_TRACK_LONG_INACTIVE;
  if (which == "ExitTrack") return OLPT_TRACK_EXIT;
  throw FatalError(OLPT_ERR_INVALID_ARG, "unknown track list: " + which);
}
}  // namespace

// STB::STB (src/srcSTB/STB.cpp:6-38)
STB::STB(const BasicSetting& setting, const std::string& type, const std::string& obj_cfg_path,
         int precision)
    : _basic_setting(setting) {
  if (type != "Tracer")
    throw FatalError(OLPT_ERR_UNSUPPORTED,
                     "Unsupported object type: " + type + " (the B200 path covers tracers)");
  _obj_config.precision = precision;
  if (!_obj_config.readConfig(obj_cfg_path, _basic_setting)) {
    std::cerr << "Failed to read Tracer config.\n";
    throw FatalError(OLPT_ERR_INVALID_ARG, "Failed to read Tracer config " + obj_cfg_path);
  }
  ctx_ = new_context();
  try {
    upload_rig(ctx_, _basic_setting._cam_list, &_obj_config._otf);
    olpt_stb_params p{};
    p.ipr = _obj_config.iprParams();
    p.frame_start = _basic_setting._frame_start;
    p.frame_end = _basic_setting._frame_end;
    p.n_initial_frames = _obj_config._stb_param._n_initial_frames;
    p.radius_search_obj_mm = _obj_config._stb_param._radius_search_obj;
    p.radius_search_track_mm = _obj_config._stb_param._radius_search_track;
    const AxisLimit& l = _basic_setting._axis_limit;
    const double lim[6] = {l.x_min, l.x_max, l.y_min, l.y_max, l.z_min, l.z_max};
    std::copy(lim, lim + 6, p.limit);
    const PFParam& pf = _obj_config._pf_param;
    p.pf_n[0] = pf.nx;
    p.pf_n[1] = pf.ny;
    p.pf_n[2] = pf.nz;
    p.pf_r_mm = pf.r;
    p.pf_nbin[0] = pf.nBin_x;
    p.pf_nbin[1] = pf.nBin_y;
    p.pf_nbin[2] = pf.nBin_z;
    p.pf_smooth = pf.is_smooth ? 1 : 0;
    p.pf_sigma[0] = pf.sigma_x;
    p.pf_sigma[1] = pf.sigma_y;
    p.pf_sigma[2] = pf.sigma_z;
    p.output_path = _basic_setting._output_path.c_str();
    check(ctx_, olpt_stb_configure(ctx_, &p));
  } catch (...) {
    olpt_ctx_destroy(ctx_);
    ctx_ = nullptr;
    throw;
  }
}

STB::~STB() {
  if (ctx_) olpt_ctx_destroy(ctx_);
}

STB::STB(STB&& o) noexcept
    : _basic_setting(std::move(o._basic_setting)),
      _obj_config(std::move(o._obj_config)),
      ctx_(o.ctx_) {
  o.ctx_ = nullptr;
}

// STB::processFrame (src/srcSTB/STB.cpp:40-89): img_list ends as the reference
// leaves it (the input in the initial phase, the residual of the shaken predictions
// in the convergence phase).
void STB::processFrame(int frame_id, std::vector<Image>& img_list) {
  upload_images(ctx_, img_list);
  check(ctx_, olpt_stb_process_frame(ctx_, frame_id));
  for (size_t c = 0; c < img_list.size(); ++c) {
    const int H = img_list[c].getDimRow(), W = img_list[c].getDimCol();
    std::vector<double> d((size_t)H * W);
    check(ctx_, olpt_stb_frame_image(ctx_, (int)c, OLPT_F64, d.data()));
    img_list[c] = Image::fromF64(H, W, d.data());
  }
}

void STB::saveTracks(const std::string& file, const std::string& which) {
  check(ctx_, olpt_stb_save_tracks(ctx_, list_id(which), file.c_str()));
}

void STB::loadTracks(const std::string& file, const std::string& which) {
  check(ctx_, olpt_stb_load_tracks(ctx_, list_id(which), file.c_str()));
}

// STB::saveTracksAll (src/srcSTB/STB.cpp:926-965)
void STB::saveTracksAll(const std::string& folder, int frame) {
  namespace fs = std::filesystem;
  const fs::path dir(folder);
  const std::string s = std::to_string(frame);
  if (fs::exists(dir))
    for (const auto& e : fs::directory_iterator(dir)) {
      if (!e.is_regular_file()) continue;
      const std::string name = e.path().filename().string();
      for (const std::string prefix : {"LongTrackActive_", "ShortTrackActive_"})
        if (name.size() >= prefix.size() + 4 && name.compare(0, prefix.size(), prefix) == 0 &&
            name.rfind(".csv") == name.size() - 4) {
          std::error_code ec;
          fs::remove(e.path(), ec);
        }
    }
  saveTracks((dir / ("LongTrackActive_" + s + ".csv")).string(), "LongTrackActive");
  saveTracks((dir / ("ShortTrackActive_" + s + ".csv")).string(), "ShortTrackActive");
  saveTracks((dir / ("ExitTrack_" + s + ".csv")).string(), "ExitTrack");
  saveTracks((dir / ("LongTrackInactive_" + s + ".csv")).string(), "LongTrackInactive");
}

// STB::loadTracksAll (src/srcSTB/STB.cpp:1049-1076)
void STB::loadTracksAll(const std::string& folder, int frame) {
  const std::string s = std::to_string(frame);
  for (const std::string which : {"LongTrackActive", "ShortTrackActive"}) {
    const std::string path = folder + which + "_" + s + ".csv";
    std::ifstream probe(path);
    if (!probe.is_open())
      throw FatalError(OLPT_ERR_INVALID_ARG, "LoadTracks: missing file: " + path);
    loadTracks(path, which);
  }
}

std::vector<Track> STB::tracks(const std::string& which) const {
  const int w = list_id(which);
  int64_t nt = 0, nr = 0;
  check(ctx_, olpt_stb_track_rows(ctx_, w, &nt, &nr));
  std::vector<int32_t> tid(nr + 1), fr(nr + 1);
  std::vector<double> xyz(3 * (size_t)nr + 3);
  check(ctx_, olpt_stb_get_tracks(ctx_, w, tid.data(), fr.data(), xyz.data(), nr));
  std::vector<Track> out(nt);
  for (int64_t r = 0; r < nr; ++r) {
    out[tid[r]]._pt_list.push_back(Pt3D(xyz[3 * r], xyz[3 * r + 1], xyz[3 * r + 2]));
    out[tid[r]]._t_list.push_back(fr[r]);
  }
  return out;
}

size_t STB::count(const std::string& which) const {
  int64_t nt = 0, nr = 0;
  check(ctx_, olpt_stb_track_rows(ctx_, list_id(which), &nt, &nr));
  return (size_t)nt;
}

// The frame loop of src/main.cpp:40-140.
int run(const std::string& config_path) {
  BasicSetting bs;
  if (!bs.readConfig(config_path)) {
    std::cerr << "Error: Failed to read basic configuration from file: " << config_path
              << std::endl;
    return 1;
  }
  std::vector<STB> stbs;
  stbs.reserve(bs._object_types.size());
  for (size_t i = 0; i < bs._object_types.size(); ++i)
    stbs.emplace_back(bs, bs._object_types[i], bs._object_config_paths[i]);
  if (bs._load_track)
    for (STB& s : stbs) s.loadTracksAll(bs._load_track_path, bs._load_track_frame);
  std::vector<ImageIO> io;
  for (const std::string& p : bs._image_file_paths) io.emplace_back("", p);
  int frame_start = bs._frame_start;
  if (bs._load_track) frame_start = bs._load_track_frame + 1;
  std::vector<Image> imgs(io.size());
  for (int f = frame_start; f <= bs._frame_end; ++f) {
    for (size_t c = 0; c < io.size(); ++c) imgs[c] = io[c].loadImg(f);
    for (STB& s : stbs) s.processFrame(f, imgs);
  }
  return 0;
}

}  // namespace lpt
