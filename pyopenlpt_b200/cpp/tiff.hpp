// Minimal TIFF reader/writer for the camera images of the tracking pipeline
// (stands in for the vendored libtiff behind the reference's ImageIO,
// inc/libMath/ImageIO.h, src/srcMath/ImageIO.cpp).
//
// Reads single-channel (grey) images of 8 or 16 bits per sample, or 32-bit float,
// stored in strips or tiles, uncompressed, LZW or PackBits, with or without the
// horizontal-differencing predictor, either byte order.  Writes uncompressed
// 8/16-bit strips.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace lpt {

struct TiffImage {
  int rows = 0, cols = 0;
  int bits = 8;          // 8, 16 (unsigned) or 32 (float)
  int sample_format = 1; // 1 = unsigned integer, 3 = IEEE float
  std::vector<uint8_t> data;  // rows * cols samples, native byte order
};

TiffImage read_tiff(const std::string& path);
void write_tiff(const std::string& path, const TiffImage& img);

}  // namespace lpt
