// Test infrastructure only (oracle build).  Stand-in definitions for the
// reference's TIFF I/O class (inc/libMath/ImageIO.h), whose implementation
// (src/srcMath/ImageIO.cpp) needs the vendored libtiff and a configure-generated
// tif_config.h that this recipe does not produce.
//
// Instead of TIFF, loadImg reads the oracle's own raw frame format so that the
// reference's config readers (TracerConfig::readConfig estimates the OTF from the
// first frames, src/srcSTB/Config.cpp:247-286) can run: 4 bytes "ORIM", int32 rows,
// int32 cols, int32 dtype (0 = u8, 1 = u16, 3 = f64), then rows*cols samples.
// loadImgPath follows ImageIO::loadImgPath (one path per line, prefixed by the
// folder).  Everything else throws.
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "ImageIO.h"

namespace {
[[noreturn]] void no_tiff(const char* what) {
  throw std::runtime_error(std::string("oracle build has no TIFF I/O: ") + what);
}
}  // namespace

void ImageIO::init() {
  _n_row = _n_col = _bits_per_sample = _n_channel = 0;
  _img_id = -1;
  _img_path.clear();
}
ImageIO::ImageIO(std::string folder, std::string list) { loadImgPath(folder, list); }
ImageIO::ImageIO(const ImageIO& o)
    : _n_row(o._n_row), _n_col(o._n_col), _bits_per_sample(o._bits_per_sample),
      _n_channel(o._n_channel), _img_id(o._img_id), _img_path(o._img_path) {}
void ImageIO::loadImgPath(std::string folder, std::string list) {
  std::ifstream in(folder + list);
  if (!in.is_open()) throw std::runtime_error("cannot open image list " + folder + list);
  init();
  std::string line;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (!line.empty()) _img_path.push_back(folder + line);
  }
}
Image ImageIO::loadImg(int id) {
  if (id < 0 || id >= (int)_img_path.size()) throw std::runtime_error("image index out of range");
  std::ifstream in(_img_path[id], std::ios::binary);
  char magic[4];
  int32_t h = 0, w = 0, dt = 0;
  in.read(magic, 4);
  in.read(reinterpret_cast<char*>(&h), 4);
  in.read(reinterpret_cast<char*>(&w), 4);
  in.read(reinterpret_cast<char*>(&dt), 4);
  if (!in || std::string(magic, 4) != "ORIM") throw std::runtime_error("not an oracle raw frame");
  Image img(h, w, 0.0);
  const size_t n = (size_t)h * w;
  if (dt == 0) {
    std::vector<uint8_t> b(n);
    in.read(reinterpret_cast<char*>(b.data()), n);
    for (size_t i = 0; i < n; ++i) img(i / w, i % w) = b[i];
  } else if (dt == 1) {
    std::vector<uint16_t> b(n);
    in.read(reinterpret_cast<char*>(b.data()), n * 2);
    for (size_t i = 0; i < n; ++i) img(i / w, i % w) = b[i];
  } else {
    std::vector<double> b(n);
    in.read(reinterpret_cast<char*>(b.data()), n * 8);
    for (size_t i = 0; i < n; ++i) img(i / w, i % w) = b[i];
  }
  _n_row = h;
  _n_col = w;
  _img_id = id;
  return img;
}
void ImageIO::saveImg(std::string, Image const&) { no_tiff("saveImg"); }
void ImageIO::setImgParam(ImageParam const&) { no_tiff("setImgParam"); }
ImageParam ImageIO::getImgParam() const { no_tiff("getImgParam"); }
void Image::save(const std::string&, int, int, std::uint16_t) const { no_tiff("Image::save"); }

// BubbleRefImg.cpp (bubble reference images, off the tracer path) calls libtiff
// directly; these stand-ins make every TIFF open fail.
extern "C" {
TIFF* TIFFOpen(const char*, const char*) { return nullptr; }
void TIFFClose(TIFF*) {}
int TIFFGetField(TIFF*, uint32, ...) { return 0; }
tmsize_t TIFFScanlineSize(TIFF*) { return 0; }
int TIFFReadScanline(TIFF*, void*, uint32, uint16) { return -1; }
void* _TIFFmalloc(tmsize_t s) { return std::malloc((size_t)s); }
void _TIFFfree(void* p) { std::free(p); }
}
