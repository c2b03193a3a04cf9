// TIFF 6.0 baseline grey images (see tiff.hpp).  LZW follows the TIFF 6.0
// specification, section 13 (MSB-first codes, 9..12 bits, code width growing one
// code early); the predictor is section 14.
#include "tiff.hpp"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <iterator>
#include <stdexcept>

namespace lpt {
namespace {

struct Reader {
  std::vector<uint8_t> b;
  bool le = true;
  uint16_t u16(size_t o) const {
    if (o + 2 > b.size()) throw std::runtime_error("TIFF: truncated file");
    return le ? (uint16_t)(b[o] | (b[o + 1] << 8)) : (uint16_t)((b[o] << 8) | b[o + 1]);
  }
  uint32_t u32(size_t o) const {
    if (o + 4 > b.size()) throw std::runtime_error("TIFF: truncated file");
    return le ? (uint32_t)b[o] | ((uint32_t)b[o + 1] << 8) | ((uint32_t)b[o + 2] << 16) |
                    ((uint32_t)b[o + 3] << 24)
              : ((uint32_t)b[o] << 24) | ((uint32_t)b[o + 1] << 16) | ((uint32_t)b[o + 2] << 8) |
                    (uint32_t)b[o + 3];
  }
};

struct Entry {
  uint16_t type = 0;
  uint32_t count = 0, value = 0;  // value or offset
  bool present = false;
};

size_t type_size(uint16_t t) {
  switch (t) {
    case 1: case 2: case 6: case 7: return 1;
    case 3: case 8: return 2;
    case 4: case 9: case 11: return 4;
    default: return 8;
  }
}

// The SHORT or LONG values of an entry; values that fit in 4 bytes are stored in the
// entry's value field itself (at field_pos).
std::vector<uint32_t> entry_values(const Reader& r, const Entry& e, size_t field_pos) {
  std::vector<uint32_t> v(e.count);
  const size_t sz = type_size(e.type);
  const size_t base = sz * e.count <= 4 ? field_pos : (size_t)e.value;
  for (uint32_t i = 0; i < e.count; ++i)
    v[i] = e.type == 3 ? r.u16(base + 2 * (size_t)i) : r.u32(base + 4 * (size_t)i);
  return v;
}

void lzw_decode(const uint8_t* in, size_t n_in, std::vector<uint8_t>& out) {
  struct Code {
    int prefix;  // -1 for roots
    uint8_t first, last;
    int len;
  };
  std::vector<Code> table(4096);
  for (int i = 0; i < 256; ++i) table[i] = Code{-1, (uint8_t)i, (uint8_t)i, 1};
  int next = 258, width = 9, prev = -1;
  size_t bitpos = 0;
  auto emit = [&](int code) {
    const int len = table[code].len;
    const size_t at = out.size();
    out.resize(at + len);
    int c = code;
    for (int k = len - 1; k >= 0; --k) {
      out[at + k] = table[c].last;
      c = table[c].prefix;
    }
  };
  for (;;) {
    if (bitpos + width > n_in * 8) break;
    int code = 0;
    for (int k = 0; k < width; ++k, ++bitpos)
      code = (code << 1) | ((in[bitpos >> 3] >> (7 - (bitpos & 7))) & 1);
    if (code == 257) break;  // EOI
    if (code == 256) {       // Clear
      next = 258;
      width = 9;
      prev = -1;
      continue;
    }
    if (prev < 0) {
      if (code > 255) throw std::runtime_error("TIFF LZW: bad first code");
      emit(code);
      prev = code;
      continue;
    }
    uint8_t first;
    if (code < next) {
      first = table[code].first;
      emit(code);
    } else if (code == next) {
      first = table[prev].first;
    } else {
      throw std::runtime_error("TIFF LZW: code out of range");
    }
    if (next < 4096) {
      table[next] = Code{prev, table[prev].first, first, table[prev].len + 1};
      if (code == next) emit(next);
      ++next;
    }
    if (next + 1 >= (1 << width) && width < 12) ++width;
    prev = code;
  }
}

void packbits_decode(const uint8_t* in, size_t n_in, std::vector<uint8_t>& out) {
  size_t i = 0;
  while (i < n_in) {
    const int8_t c = (int8_t)in[i++];
    if (c >= 0) {
      const size_t n = (size_t)c + 1;
      if (i + n > n_in) break;
      out.insert(out.end(), in + i, in + i + n);
      i += n;
    } else if (c != -128) {
      if (i >= n_in) break;
      out.insert(out.end(), (size_t)(1 - c), in[i++]);
    }
  }
}

}  // namespace

TiffImage read_tiff(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open image " + path);
  Reader r;
  r.b.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  if (r.b.size() < 8) throw std::runtime_error("TIFF: truncated file " + path);
  if (r.b[0] == 'I' && r.b[1] == 'I')
    r.le = true;
  else if (r.b[0] == 'M' && r.b[1] == 'M')
    r.le = false;
  else
    throw std::runtime_error("not a TIFF file: " + path);
  if (r.u16(2) != 42) throw std::runtime_error("TIFF: bad magic in " + path);
  const uint32_t ifd = r.u32(4);
  const uint16_t n_entries = r.u16(ifd);
  Entry tags[16];  // only the tags below are kept
  auto slot = [](uint16_t tag) -> int {
    switch (tag) {
      case 256: return 0; case 257: return 1; case 258: return 2; case 259: return 3;
      case 262: return 4; case 273: return 5; case 277: return 6; case 278: return 7;
      case 279: return 8; case 284: return 9; case 317: return 10; case 322: return 11;
      case 323: return 12; case 324: return 13; case 325: return 14; case 339: return 15;
      default: return -1;
    }
  };
  size_t pos[16] = {0};
  for (uint16_t i = 0; i < n_entries; ++i) {
    const size_t o = ifd + 2 + 12 * (size_t)i;
    const int s = slot(r.u16(o));
    if (s < 0) continue;
    Entry& e = tags[s];
    e.type = r.u16(o + 2);
    e.count = r.u32(o + 4);
    e.value = r.u32(o + 8);
    e.present = true;
    pos[s] = o + 8;
  }
  auto scalar = [&](int s, uint32_t def) -> uint32_t {
    if (!tags[s].present || tags[s].count == 0) return def;
    return entry_values(r, tags[s], pos[s])[0];
  };
  TiffImage img;
  img.cols = (int)scalar(0, 0);
  img.rows = (int)scalar(1, 0);
  img.bits = (int)scalar(2, 8);
  const uint32_t compression = scalar(3, 1);
  const uint32_t spp = scalar(6, 1);
  const uint32_t predictor = scalar(10, 1);
  img.sample_format = (int)scalar(15, 1);
  if (spp != 1) throw std::runtime_error("TIFF: only single-channel images are supported: " + path);
  if (!(img.bits == 8 || img.bits == 16 || (img.bits == 32 && img.sample_format == 3)))
    throw std::runtime_error("TIFF: unsupported sample size in " + path);
  if (compression != 1 && compression != 5 && compression != 32773)
    throw std::runtime_error("TIFF: unsupported compression in " + path);
  const int bps = img.bits / 8;
  const bool tiled = tags[11].present;
  const int blk_w = tiled ? (int)scalar(11, 0) : img.cols;
  const int blk_h = tiled ? (int)scalar(12, 0) : (int)scalar(7, (uint32_t)img.rows);
  const int off_s = tiled ? 13 : 5, cnt_s = tiled ? 14 : 8;
  if (!tags[off_s].present || !tags[cnt_s].present || blk_w <= 0 || blk_h <= 0 || img.rows <= 0 ||
      img.cols <= 0)
    throw std::runtime_error("TIFF: missing strip/tile layout in " + path);
  const std::vector<uint32_t> offs = entry_values(r, tags[off_s], pos[off_s]);
  const std::vector<uint32_t> cnts = entry_values(r, tags[cnt_s], pos[cnt_s]);
  img.data.assign((size_t)img.rows * img.cols * bps, 0);
  const int across = (img.cols + blk_w - 1) / blk_w;
  const bool host_le = __BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__;
  std::vector<uint8_t> raw;
  for (size_t k = 0; k < offs.size() && k < cnts.size(); ++k) {
    if ((size_t)offs[k] + cnts[k] > r.b.size()) throw std::runtime_error("TIFF: truncated " + path);
    const uint8_t* src = r.b.data() + offs[k];
    raw.clear();
    if (compression == 1)
      raw.assign(src, src + cnts[k]);
    else if (compression == 5)
      lzw_decode(src, cnts[k], raw);
    else
      packbits_decode(src, cnts[k], raw);
    const int r0 = (int)(k / across) * blk_h, c0 = (int)(k % across) * blk_w;
    const size_t row_bytes = (size_t)blk_w * bps;
    for (int y = 0; y < blk_h; ++y) {
      if ((size_t)(y + 1) * row_bytes > raw.size()) break;
      uint8_t* row = raw.data() + (size_t)y * row_bytes;
      if (bps > 1 && r.le != host_le)
        for (int x = 0; x < blk_w; ++x)
          for (int q = 0; q < bps / 2; ++q) std::swap(row[x * bps + q], row[x * bps + bps - 1 - q]);
      if (predictor == 2) {
        if (bps == 1) {
          for (int x = 1; x < blk_w; ++x) row[x] = (uint8_t)(row[x] + row[x - 1]);
        } else if (bps == 2) {
          uint16_t* p = reinterpret_cast<uint16_t*>(row);
          for (int x = 1; x < blk_w; ++x) p[x] = (uint16_t)(p[x] + p[x - 1]);
        }
      }
      const int yy = r0 + y;
      if (yy >= img.rows) break;
      const int w = std::min(blk_w, img.cols - c0);
      if (w > 0)
        std::memcpy(img.data.data() + ((size_t)yy * img.cols + c0) * bps, row, (size_t)w * bps);
    }
  }
  return img;
}

void write_tiff(const std::string& path, const TiffImage& img) {
  if (img.bits != 8 && img.bits != 16) throw std::runtime_error("TIFF: write supports 8/16 bits");
  const uint32_t bps = img.bits / 8;
  const uint32_t bytes = (uint32_t)img.rows * img.cols * bps;
  std::vector<uint8_t> out;
  auto put16 = [&](uint16_t v) {
    out.push_back(v & 255);
    out.push_back(v >> 8);
  };
  auto put32 = [&](uint32_t v) {
    for (int k = 0; k < 4; ++k) out.push_back((v >> (8 * k)) & 255);
  };
  out.push_back('I');
  out.push_back('I');
  put16(42);
  put32(8 + bytes);  // IFD after the pixel data
  out.insert(out.end(), img.data.begin(), img.data.end());
  put16(10);
  auto entry = [&](uint16_t tag, uint16_t type, uint32_t count, uint32_t value) {
    put16(tag);
    put16(type);
    put32(count);
    if (type == 3 && count == 1) {
      put16((uint16_t)value);
      put16(0);
    } else {
      put32(value);
    }
  };
  entry(256, 3, 1, img.cols);
  entry(257, 3, 1, img.rows);
  entry(258, 3, 1, img.bits);
  entry(259, 3, 1, 1);
  entry(262, 3, 1, 1);
  entry(273, 4, 1, 8);
  entry(277, 3, 1, 1);
  entry(278, 3, 1, img.rows);
  entry(279, 4, 1, bytes);
  entry(284, 3, 1, 1);
  put32(0);
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot write image " + path);
  f.write(reinterpret_cast<const char*>(out.data()), (std::streamsize)out.size());
}

}  // namespace lpt
