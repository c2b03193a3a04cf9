// Test infrastructure only (oracle build).  Stand-in definitions for the
// reference's TIFF I/O class (inc/libMath/ImageIO.h), whose implementation
// (src/srcMath/ImageIO.cpp) needs the vendored libtiff and a configure-generated
// tif_config.h that this recipe does not produce.  Nothing on the IPR / Shake /
// STB path calls these: the oracle driver hands images over in memory.
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "ImageIO.h"

namespace {
[[noreturn]] void no_tiff(const char* what) {
  throw std::runtime_error(std::string("oracle build has no TIFF I/O: ") + what);
}
}  // namespace

void ImageIO::init() {}
ImageIO::ImageIO(std::string, std::string) { no_tiff("ImageIO(folder, list)"); }
ImageIO::ImageIO(const ImageIO& o)
    : _n_row(o._n_row), _n_col(o._n_col), _bits_per_sample(o._bits_per_sample),
      _n_channel(o._n_channel), _img_id(o._img_id), _img_path(o._img_path) {}
void ImageIO::loadImgPath(std::string, std::string) { no_tiff("loadImgPath"); }
Image ImageIO::loadImg(int) { no_tiff("loadImg"); }
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
