// Python module of the drop-in classes, under the reference's module name pyopenlpt
// (built as pyopenlpt_b200/pyopenlpt*.so; the shim pyopenlpt_b200/openlpt.py
// re-exports it as the reference's openlpt.py does).  Class and method names follow the reference's bindings
// (src/pybind_OpenLPT/py*.cpp) for the reconstruction path: Camera, OTF, Image,
// ImageIO, Pt2D, Pt3D, Tracer2D, Tracer3D, ObjFlag, BasicSetting, TracerConfig (+
// parameter structs), ObjectFinder2D, StereoMatch, Shake (runShake returns
// (flags, objs)), IPR, STB (process_frame returns the residual images), run.
#include <cstring>
#include <optional>

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "openlpt.hpp"

namespace py = pybind11;
using namespace lpt;

namespace {

std::unique_ptr<Object3D> clone3d(const Object3D& o) {
  auto t = std::make_unique<Tracer3D>();
  t->_pt_center = o._pt_center;
  t->_is_tracked = o._is_tracked;
  if (auto tr = dynamic_cast<const Tracer3D*>(&o)) t->_r2d_px = tr->_r2d_px;
  for (const auto& p : o._obj2d_list) t->_obj2d_list.push_back(p ? p->clone() : nullptr);
  return t;
}

std::vector<Tracer3D*> tracers(const py::list& objs) {
  std::vector<Tracer3D*> v;
  for (py::handle h : objs) v.push_back(h.cast<Tracer3D*>());
  return v;
}

std::vector<std::unique_ptr<Object3D>> own3d(const std::vector<Tracer3D*>& objs) {
  std::vector<std::unique_ptr<Object3D>> v;
  v.reserve(objs.size());
  for (Tracer3D* o : objs) v.push_back(clone3d(*o));
  return v;
}

void copy_back(const std::vector<std::unique_ptr<Object3D>>& src, const std::vector<Tracer3D*>& dst) {
  for (size_t i = 0; i < dst.size(); ++i) {
    dst[i]->_pt_center = src[i]->_pt_center;
    dst[i]->_obj2d_list.clear();
    for (const auto& p : src[i]->_obj2d_list) dst[i]->_obj2d_list.push_back(p ? p->clone() : nullptr);
  }
}

Image image_from_numpy(py::array arr) {
  if (arr.ndim() != 2) throw std::invalid_argument("Image: a 2D array is required");
  const int r = (int)arr.shape(0), c = (int)arr.shape(1);
  if (py::isinstance<py::array_t<uint8_t>>(arr)) {
    auto a = py::array_t<uint8_t, py::array::c_style | py::array::forcecast>(arr);
    return Image::fromU8(r, c, a.data());
  }
  if (py::isinstance<py::array_t<uint16_t>>(arr)) {
    auto a = py::array_t<uint16_t, py::array::c_style | py::array::forcecast>(arr);
    return Image::fromU16(r, c, a.data());
  }
  auto a = py::array_t<double, py::array::c_style | py::array::forcecast>(arr);
  return Image::fromF64(r, c, a.data());
}

py::array image_to_numpy(const Image& im) {
  const std::vector<ssize_t> shape{im.getDimRow(), im.getDimCol()};
  const size_t n = (size_t)im.getDimRow() * im.getDimCol();
  switch (im.dtype()) {
    case OLPT_U8: {
      py::array_t<uint8_t> a(shape);
      std::memcpy(a.mutable_data(), im.data(), n);
      return a;
    }
    case OLPT_U16: {
      py::array_t<uint16_t> a(shape);
      std::memcpy(a.mutable_data(), im.data(), n * 2);
      return a;
    }
    default: {
      py::array_t<double> a(shape);
      const std::vector<double> d = im.toDouble();
      std::memcpy(a.mutable_data(), d.data(), n * 8);
      return a;
    }
  }
}

py::array_t<double> vec_to_numpy(const std::vector<double>& v, int rows, int cols) {
  py::array_t<double> a({rows, cols});
  std::memcpy(a.mutable_data(), v.data(), v.size() * sizeof(double));
  return a;
}

std::vector<double> numpy_to_vec(py::array_t<double, py::array::c_style | py::array::forcecast> a) {
  return std::vector<double>(a.data(), a.data() + a.size());
}

// Holders that own copies of their constructor arguments (the C++ classes keep
// references, as the reference's do).
struct PyStereoMatch {
  std::vector<Camera> cams;
  std::vector<std::vector<std::unique_ptr<Object2D>>> obj2d;
  TracerConfig cfg;
};
struct PyShake {
  std::vector<Camera> cams;
  TracerConfig cfg;
};
struct PyIPR {
  std::vector<Camera> cams;
};

}  // namespace

PYBIND11_MODULE(pyopenlpt, m) {
  m.doc() = "B200 drop-in for the OpenLPT reconstruction path (IPR + Shake-the-Box)";
  py::register_exception<FatalError>(m, "FatalError", PyExc_RuntimeError);

  py::class_<Pt2D>(m, "Pt2D")
      .def(py::init<>())
      .def(py::init<double, double>())
      .def("__getitem__", [](const Pt2D& p, int i) { return p[i]; })
      .def("__setitem__", [](Pt2D& p, int i, double v) { p[i] = v; })
      .def("to_list", [](const Pt2D& p) { return std::vector<double>{p[0], p[1]}; })
      .def("__repr__", [](const Pt2D& p) {
        return "Pt2D(" + std::to_string(p[0]) + ", " + std::to_string(p[1]) + ")";
      });
  py::class_<Pt3D>(m, "Pt3D")
      .def(py::init<>())
      .def(py::init<double, double, double>())
      .def("__getitem__", [](const Pt3D& p, int i) { return p[i]; })
      .def("__setitem__", [](Pt3D& p, int i, double v) { p[i] = v; })
      .def("to_list", [](const Pt3D& p) { return std::vector<double>{p[0], p[1], p[2]}; })
      .def("__repr__", [](const Pt3D& p) {
        return "Pt3D(" + std::to_string(p[0]) + ", " + std::to_string(p[1]) + ", " +
               std::to_string(p[2]) + ")";
      });
  py::class_<AxisLimit>(m, "AxisLimit")
      .def(py::init<>())
      .def(py::init([](double a, double b, double c, double d, double e, double f) {
        return AxisLimit{a, b, c, d, e, f};
      }))
      .def_readwrite("x_min", &AxisLimit::x_min)
      .def_readwrite("x_max", &AxisLimit::x_max)
      .def_readwrite("y_min", &AxisLimit::y_min)
      .def_readwrite("y_max", &AxisLimit::y_max)
      .def_readwrite("z_min", &AxisLimit::z_min)
      .def_readwrite("z_max", &AxisLimit::z_max)
      .def("check", &AxisLimit::check);

  py::class_<Image>(m, "Image")
      .def(py::init<>())
      .def(py::init<int, int, double>(), py::arg("n_row"), py::arg("n_col"), py::arg("val") = 0.0)
      .def_static("from_numpy", &image_from_numpy, py::arg("array"))
      .def("to_numpy", &image_to_numpy)
      .def("getDimRow", &Image::getDimRow)
      .def("getDimCol", &Image::getDimCol)
      .def("__getitem__", [](const Image& im, std::pair<int, int> rc) { return im(rc.first, rc.second); })
      .def("__setitem__", [](Image& im, std::pair<int, int> rc, double v) { im.set(rc.first, rc.second, v); })
      .def("save", &Image::save, py::arg("path"));

  py::class_<ImageIO>(m, "ImageIO")
      .def(py::init<>())
      .def(py::init<const std::string&, const std::string&>(), py::arg("folder_path"),
           py::arg("file_img_path"))
      .def("loadImgPath", &ImageIO::loadImgPath, py::arg("folder_path"), py::arg("file_img_path"))
      .def("loadImg", &ImageIO::loadImg, py::arg("img_id"))
      .def("saveImg", &ImageIO::saveImg, py::arg("save_path"), py::arg("image"))
      .def("getCurrImgID", &ImageIO::getCurrImgID)
      .def("getImgPath", &ImageIO::getImgPath);

  py::class_<Camera>(m, "Camera")
      .def(py::init<>())
      .def(py::init<const std::string&>(), py::arg("file_name"))
      .def("loadParameters", &Camera::loadParameters, py::arg("file_name"))
      .def("getNRow", &Camera::getNRow)
      .def("getNCol", &Camera::getNCol)
      .def("project", &Camera::project, py::arg("pt_world"))
      .def("lineOfSight", &Camera::lineOfSight, py::arg("pt_img"))
      .def_readwrite("_is_active", &Camera::_is_active)
      .def_readwrite("_max_intensity", &Camera::_max_intensity);

  py::class_<OTF>(m, "OTF")
      .def(py::init<>())
      .def(py::init<const std::string&>(), py::arg("otf_file"))
      .def("loadParam", py::overload_cast<const std::string&>(&OTF::loadParam), py::arg("otf_file"))
      .def("loadParam",
           py::overload_cast<int, int, int, int, const AxisLimit&, const std::vector<Camera>&>(
               &OTF::loadParam),
           py::arg("n_cam"), py::arg("nx"), py::arg("ny"), py::arg("nz"), py::arg("boundary"),
           py::arg("cam_list"))
      .def("saveParam", &OTF::saveParam, py::arg("otf_file"))
      .def_property_readonly("n_cam", [](const OTF& o) { return o._param.n_cam; })
      .def_property_readonly("n_grid", [](const OTF& o) { return o._param.n_grid; })
      .def_property("a", [](const OTF& o) { return vec_to_numpy(o._param.a, o._param.n_cam, o._param.n_grid); },
                    [](OTF& o, py::array_t<double> v) { o._param.a = numpy_to_vec(v); })
      .def_property("b", [](const OTF& o) { return vec_to_numpy(o._param.b, o._param.n_cam, o._param.n_grid); },
                    [](OTF& o, py::array_t<double> v) { o._param.b = numpy_to_vec(v); })
      .def_property("c", [](const OTF& o) { return vec_to_numpy(o._param.c, o._param.n_cam, o._param.n_grid); },
                    [](OTF& o, py::array_t<double> v) { o._param.c = numpy_to_vec(v); })
      .def_property("alpha",
                    [](const OTF& o) { return vec_to_numpy(o._param.alpha, o._param.n_cam, o._param.n_grid); },
                    [](OTF& o, py::array_t<double> v) { o._param.alpha = numpy_to_vec(v); });

  py::enum_<ObjFlag>(m, "ObjFlag")
      .value("None_", ObjFlag::None)
      .value("Ghost", ObjFlag::Ghost)
      .value("Repeated", ObjFlag::Repeated);

  py::class_<Object2D, std::unique_ptr<Object2D>>(m, "Object2D")
      .def_readwrite("_pt_center", &Object2D::_pt_center);
  py::class_<Tracer2D, Object2D, std::unique_ptr<Tracer2D>>(m, "Tracer2D")
      .def(py::init<>())
      .def_readwrite("_r_px", &Tracer2D::_r_px);
  py::class_<Object3D, std::unique_ptr<Object3D>>(m, "Object3D")
      .def_readwrite("_pt_center", &Object3D::_pt_center)
      .def_readwrite("_is_tracked", &Object3D::_is_tracked)
      .def("__len__", [](const Object3D& o) { return o._obj2d_list.size(); })
      .def("__getitem__",
           [](const Object3D& o, size_t i) -> py::object {
             if (i >= o._obj2d_list.size()) throw py::index_error();
             if (!o._obj2d_list[i]) return py::none();
             return py::cast(*static_cast<const Tracer2D*>(o._obj2d_list[i].get()));
           })
      .def("projectObject2D", &Object3D::projectObject2D, py::arg("cam_list"))
      .def("isReconstructable", &Object3D::isReconstructable, py::arg("cam_list"));
  py::class_<Tracer3D, Object3D, std::unique_ptr<Tracer3D>>(m, "Tracer3D")
      .def(py::init<>())
      .def(py::init([](const Pt3D& c) {
        auto t = std::make_unique<Tracer3D>();
        t->_pt_center = c;
        return t;
      }))
      .def_readwrite("_r2d_px", &Tracer3D::_r2d_px);

  py::class_<BasicSetting>(m, "BasicSetting")
      .def(py::init<>())
      .def("readConfig", &BasicSetting::readConfig, py::arg("config_file"))
      .def_readwrite("_frame_start", &BasicSetting::_frame_start)
      .def_readwrite("_frame_end", &BasicSetting::_frame_end)
      .def_readwrite("_fps", &BasicSetting::_fps)
      .def_readwrite("_n_thread", &BasicSetting::_n_thread)
      .def_readwrite("_n_cam", &BasicSetting::_n_cam)
      .def_readwrite("_cam_list", &BasicSetting::_cam_list)
      .def_readwrite("_image_file_paths", &BasicSetting::_image_file_paths)
      .def_readwrite("_axis_limit", &BasicSetting::_axis_limit)
      .def_readwrite("_voxel_to_mm", &BasicSetting::_voxel_to_mm)
      .def_readwrite("_output_path", &BasicSetting::_output_path)
      .def_readwrite("_object_types", &BasicSetting::_object_types)
      .def_readwrite("_object_config_paths", &BasicSetting::_object_config_paths)
      .def_readwrite("_load_track", &BasicSetting::_load_track)
      .def_readwrite("_load_track_frame", &BasicSetting::_load_track_frame)
      .def_readwrite("_load_track_path", &BasicSetting::_load_track_path);

  py::class_<STBParam>(m, "STBParam")
      .def(py::init<>())
      .def_readwrite("_radius_search_obj", &STBParam::_radius_search_obj)
      .def_readwrite("_n_initial_frames", &STBParam::_n_initial_frames)
      .def_readwrite("_radius_search_track", &STBParam::_radius_search_track);
  py::class_<ShakeParam>(m, "ShakeParam")
      .def(py::init<>())
      .def_readwrite("_shake_width", &ShakeParam::_shake_width)
      .def_readwrite("_shakewidth_min", &ShakeParam::_shakewidth_min)
      .def_readwrite("_n_shake_loop", &ShakeParam::_n_shake_loop)
      .def_readwrite("_thred_ghost", &ShakeParam::_thred_ghost)
      .def_readwrite("_ratio_augimg", &ShakeParam::_ratio_augimg);
  py::class_<PFParam>(m, "PFParam")
      .def(py::init<>())
      .def_readwrite("limit", &PFParam::limit)
      .def_readwrite("nx", &PFParam::nx)
      .def_readwrite("ny", &PFParam::ny)
      .def_readwrite("nz", &PFParam::nz)
      .def_readwrite("r", &PFParam::r)
      .def_readwrite("nBin_x", &PFParam::nBin_x)
      .def_readwrite("nBin_y", &PFParam::nBin_y)
      .def_readwrite("nBin_z", &PFParam::nBin_z)
      .def_readwrite("is_smooth", &PFParam::is_smooth)
      .def_readwrite("sigma_x", &PFParam::sigma_x)
      .def_readwrite("sigma_y", &PFParam::sigma_y)
      .def_readwrite("sigma_z", &PFParam::sigma_z);
  py::class_<SMParam>(m, "SMParam")
      .def(py::init<>())
      .def_readwrite("match_cam_count", &SMParam::match_cam_count)
      .def_readwrite("idmap_cell_px", &SMParam::idmap_cell_px)
      .def_readwrite("tol_2d_px", &SMParam::tol_2d_px)
      .def_readwrite("tol_3d_mm", &SMParam::tol_3d_mm)
      .def_readwrite("limit", &SMParam::limit);
  py::class_<IPRParam>(m, "IPRParam")
      .def(py::init<>())
      .def_readwrite("n_cam_reduced", &IPRParam::n_cam_reduced)
      .def_readwrite("n_loop_ipr", &IPRParam::n_loop_ipr)
      .def_readwrite("n_loop_ipr_reduced", &IPRParam::n_loop_ipr_reduced)
      .def_readwrite("n_obj2d_process_max", &IPRParam::n_obj2d_process_max);
  py::enum_<ObjectKind>(m, "ObjectKind")
      .value("Tracer", ObjectKind::Tracer)
      .value("Bubble", ObjectKind::Bubble);
  py::class_<ObjectConfig>(m, "ObjectConfig")
      .def("kind", &ObjectConfig::kind)
      .def_readwrite("_stb_param", &ObjectConfig::_stb_param)
      .def_readwrite("_shake_param", &ObjectConfig::_shake_param)
      .def_readwrite("_pf_param", &ObjectConfig::_pf_param)
      .def_readwrite("_sm_param", &ObjectConfig::_sm_param)
      .def_readwrite("_ipr_param", &ObjectConfig::_ipr_param)
      .def_readwrite("precision", &ObjectConfig::precision);
  py::class_<TracerConfig, ObjectConfig>(m, "TracerConfig")
      .def(py::init<>())
      .def("readConfig", &TracerConfig::readConfig, py::arg("filepath"), py::arg("settings"))
      .def_readwrite("_min_obj_int", &TracerConfig::_min_obj_int)
      .def_readwrite("_radius_obj", &TracerConfig::_radius_obj)
      .def_readwrite("_otf", &TracerConfig::_otf);

  py::class_<ObjectFinder2D>(m, "ObjectFinder2D")
      .def(py::init<>())
      .def("findObject2D", &ObjectFinder2D::findObject2D, py::arg("img"), py::arg("obj_cfg"));

  py::class_<PyStereoMatch>(m, "StereoMatch")
      .def(py::init([](const std::vector<Camera>& cams,
                       const std::vector<std::vector<Tracer2D*>>& obj2d_by_cam,
                       const TracerConfig& cfg) {
             auto s = std::make_unique<PyStereoMatch>();
             s->cams = cams;
             s->cfg = cfg;
             for (const auto& cam : obj2d_by_cam) {
               s->obj2d.emplace_back();
               for (const Tracer2D* t : cam) s->obj2d.back().push_back(t->clone());
             }
             return s;
           }),
           py::arg("cams"), py::arg("obj2d_by_cam"), py::arg("obj_cfg"))
      .def("match", [](const PyStereoMatch& s) { return StereoMatch(s.cams, s.obj2d, s.cfg).match(); });

  py::class_<PyShake>(m, "Shake")
      .def(py::init([](const std::vector<Camera>& cams, const TracerConfig& cfg) {
             return PyShake{cams, cfg};
           }),
           py::arg("cams"), py::arg("obj_cfg"))
      .def(
          "runShake",
          [](PyShake& s, py::list objs_py, const std::vector<Image>& imgs) {
            const std::vector<Tracer3D*> objs = tracers(objs_py);
            auto own = own3d(objs);
            auto flags = Shake(s.cams, s.cfg).runShake(own, imgs);
            copy_back(own, objs);
            return py::make_tuple(flags, objs_py);
          },
          py::arg("objs"), py::arg("img_orig"))
      .def(
          "calResidualImage",
          [](PyShake& s, py::list objs_py, const std::vector<Image>& imgs,
             std::optional<std::vector<ObjFlag>> flags) {
            auto own = own3d(tracers(objs_py));
            return Shake(s.cams, s.cfg).calResidualImage(own, imgs, flags ? &*flags : nullptr);
          },
          py::arg("objs"), py::arg("img_orig"), py::arg("flags") = py::none());

  py::class_<PyIPR>(m, "IPR")
      .def(py::init([](const std::vector<Camera>& cams) { return PyIPR{cams}; }), py::arg("cams"))
      .def(
          "runIPR",
          [](PyIPR& s, TracerConfig& cfg, std::vector<Image> images) {
            return IPR(s.cams).runIPR(cfg, std::move(images));
          },
          py::arg("cfg"), py::arg("images"))
      .def(
          "saveObjInfo",
          [](PyIPR& s, const std::string& file, py::list objs, const TracerConfig& cfg) {
            IPR(s.cams).saveObjInfo(file, own3d(tracers(objs)), cfg);
          },
          py::arg("filename"), py::arg("objs"), py::arg("cfg"));

  py::class_<Track>(m, "Track")
      .def(py::init<>())
      .def_readwrite("_pt_list", &Track::_pt_list)
      .def_readwrite("_t_list", &Track::_t_list);

  py::class_<STB>(m, "STB")
      .def(py::init<const BasicSetting&, const std::string&, const std::string&, int>(),
           py::arg("setting"), py::arg("obj_type"), py::arg("obj_cfg_path"),
           py::arg("precision") = 0)
      .def(
          "process_frame",
          [](STB& self, int frame_id, std::vector<Image> img_list) {
            self.processFrame(frame_id, img_list);
            return img_list;
          },
          py::arg("frame_id"), py::arg("img_list"),
          "Run STB on a frame; returns the modified residual images.")
      .def("saveTracksAll", &STB::saveTracksAll, py::arg("folder"), py::arg("t"))
      .def("loadTracksAll", &STB::loadTracksAll, py::arg("folder"), py::arg("t"))
      .def("saveTracks", &STB::saveTracks, py::arg("file"), py::arg("which"))
      .def("loadTracks", &STB::loadTracks, py::arg("file"), py::arg("which"))
      .def_property_readonly("_short_track_active", [](const STB& s) { return s.tracks("ShortTrackActive"); })
      .def_property_readonly("_long_track_active", [](const STB& s) { return s.tracks("LongTrackActive"); })
      .def_property_readonly("_long_track_inactive", [](const STB& s) { return s.tracks("LongTrackInactive"); })
      .def_property_readonly("_exit_track", [](const STB& s) { return s.tracks("ExitTrack"); })
      .def_readonly("_basic_setting", &STB::_basic_setting)
      .def_readonly("_obj_config", &STB::_obj_config);

  m.def(
      "run",
      [](const std::string& config_path) {
        py::gil_scoped_release release;
        return lpt::run(config_path);
      },
      py::arg("config_file_path"));
}
