// dtb_io.cpp -- image files for the C ABI (dtb_image_read / dtb_image_write), the reference's dt::imread /
// dt::imsave (dt/src/imread.cpp, dt/src/imsave.cpp, which use stb_image): 8-bit PNG and binary PGM / PPM here,
// JPEG (read only) in dtb_jpeg.cpp.
//
// PNG follows the published format (ISO/IEC 15948): chunks with CRC-32, one zlib stream over the IDAT chunks,
// per-row filter types 0-4 (None, Sub, Up, Average, Paeth).  Read: colour types 0 (gray), 2 (rgb), 3 (palette,
// expanded to rgb), 4 (gray + alpha) and 6 (rgba) at 8 bits per sample, gray and palette also at 1 / 2 / 4,
// not interlaced.  Write: gray or rgb,
// filter 0 on every row.  zlib (the system library) does the deflate / inflate and the CRC.
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dtb.h"
#include "dtb_imgfile.h"

namespace {

bool ends_with(const std::string& s, const char* suf) {
  const size_t n = std::strlen(suf);
  if (s.size() < n) return false;
  for (size_t i = 0; i < n; ++i)
    if (std::tolower((unsigned char)s[s.size() - n + i]) != suf[i]) return false;
  return true;
}

bool read_file(const char* path, std::vector<uint8_t>& out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (n < 0) {
    std::fclose(f);
    return false;
  }
  out.resize((size_t)n);
  const bool ok = n == 0 || std::fread(out.data(), 1, (size_t)n, f) == (size_t)n;
  std::fclose(f);
  return ok;
}

uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }
void put_be32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back((uint8_t)(x >> 24));
  v.push_back((uint8_t)(x >> 16));
  v.push_back((uint8_t)(x >> 8));
  v.push_back((uint8_t)x);
}

using dtb_io::Pixels;

uint8_t paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return (uint8_t)a;
  return (uint8_t)(pb <= pc ? b : c);
}

dtb_status decode_png(const std::vector<uint8_t>& f, Pixels& out) {
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (f.size() < 8 || std::memcmp(f.data(), sig, 8) != 0) return DTB_ERR_INVALID_ARG;
  size_t pos = 8;
  int w = 0, h = 0, depth = 0, ctype = -1, interlace = 0;
  std::vector<uint8_t> idat, palette;
  bool end = false;
  while (!end && pos + 12 <= f.size()) {
    const uint32_t len = be32(&f[pos]);
    if (pos + 12 + (size_t)len > f.size()) return DTB_ERR_INVALID_ARG;
    const uint8_t* type = &f[pos + 4];
    const uint8_t* body = &f[pos + 8];
    if (crc32(crc32(0L, Z_NULL, 0), type, len + 4) != be32(body + len)) return DTB_ERR_INVALID_ARG;
    if (!std::memcmp(type, "IHDR", 4) && len >= 13) {
      w = (int)be32(body);
      h = (int)be32(body + 4);
      depth = body[8];
      ctype = body[9];
      interlace = body[12];
    } else if (!std::memcmp(type, "PLTE", 4)) {
      palette.assign(body, body + len);
    } else if (!std::memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), body, body + len);
    } else if (!std::memcmp(type, "IEND", 4)) {
      end = true;
    }
    pos += 12 + (size_t)len;
  }
  if (w <= 0 || h <= 0 || interlace != 0) return DTB_ERR_INVALID_ARG;
  if ((uint64_t)w * (uint64_t)h > dtb_io::kMaxFilePixels) return DTB_ERR_INVALID_ARG;
  int comp;
  switch (ctype) {
    case 0: comp = 1; break;
    case 2: comp = 3; break;
    case 3: comp = 1; break;
    case 4: comp = 2; break;
    case 6: comp = 4; break;
    default: return DTB_ERR_INVALID_ARG;
  }
  // Sample depths: 8 for every colour type; 1, 2, 4 also for gray and palette images.
  const bool sub = depth == 1 || depth == 2 || depth == 4;
  if (!(depth == 8 || (sub && (ctype == 0 || ctype == 3)))) return DTB_ERR_INVALID_ARG;
  const size_t stride = ((size_t)w * comp * depth + 7) / 8;  // bytes per row
  const size_t bpp = std::max<size_t>(1, (size_t)comp * depth / 8);  // filter distance in bytes
  std::vector<uint8_t> raw((stride + 1) * (size_t)h);
  uLongf raw_len = (uLongf)raw.size();
  if (uncompress(raw.data(), &raw_len, idat.data(), (uLong)idat.size()) != Z_OK || raw_len != raw.size())
    return DTB_ERR_INVALID_ARG;
  std::vector<uint8_t> rows(stride * (size_t)h);
  for (int y = 0; y < h; ++y) {
    const uint8_t ft = raw[(size_t)y * (stride + 1)];
    const uint8_t* src = &raw[(size_t)y * (stride + 1) + 1];
    uint8_t* cur = &rows[(size_t)y * stride];
    const uint8_t* up = y ? &rows[(size_t)(y - 1) * stride] : nullptr;
    for (size_t i = 0; i < stride; ++i) {
      const int a = i >= bpp ? cur[i - bpp] : 0;
      const int b = up ? up[i] : 0;
      const int c = (up && i >= bpp) ? up[i - bpp] : 0;
      int v;
      switch (ft) {
        case 0: v = src[i]; break;
        case 1: v = src[i] + a; break;
        case 2: v = src[i] + b; break;
        case 3: v = src[i] + ((a + b) >> 1); break;
        case 4: v = src[i] + paeth(a, b, c); break;
        default: return DTB_ERR_INVALID_ARG;
      }
      cur[i] = (uint8_t)v;
    }
  }
  // One byte per sample: unpack sub-byte samples (most significant bits first); gray levels scale to 0..255.
  std::vector<uint8_t> img;
  if (sub) {
    img.resize((size_t)w * h);
    const int maxv = (1 << depth) - 1;
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        const size_t bit = (size_t)x * depth;
        const int v = (rows[(size_t)y * stride + bit / 8] >> (8 - depth - (int)(bit % 8))) & maxv;
        img[(size_t)y * w + x] = (uint8_t)(ctype == 0 ? v * 255 / maxv : v);
      }
  } else {
    img.swap(rows);
  }
  out.w = w;
  out.h = h;
  if (ctype == 3) {  // palette indices -> rgb
    out.channels = 3;
    out.data.resize((size_t)w * h * 3);
    for (size_t i = 0; i < (size_t)w * h; ++i) {
      const size_t k = 3 * (size_t)img[i];
      if (k + 3 > palette.size()) return DTB_ERR_INVALID_ARG;
      std::memcpy(&out.data[3 * i], &palette[k], 3);
    }
  } else {
    out.channels = comp;
    out.data.swap(img);
  }
  return DTB_OK;
}

// Binary PGM (P5) / PPM (P6), maxval <= 255.
dtb_status decode_pnm(const std::vector<uint8_t>& f, Pixels& out) {
  if (f.size() < 2 || f[0] != 'P' || (f[1] != '5' && f[1] != '6')) return DTB_ERR_INVALID_ARG;
  size_t pos = 2;
  long vals[3];
  for (int k = 0; k < 3; ++k) {
    for (;;) {  // whitespace and comments
      while (pos < f.size() && std::isspace(f[pos])) ++pos;
      if (pos < f.size() && f[pos] == '#') {
        while (pos < f.size() && f[pos] != '\n') ++pos;
        continue;
      }
      break;
    }
    if (pos >= f.size() || !std::isdigit(f[pos])) return DTB_ERR_INVALID_ARG;
    long v = 0;
    while (pos < f.size() && std::isdigit(f[pos]) && v < 1000000000L) v = v * 10 + (f[pos++] - '0');
    vals[k] = v;
  }
  ++pos;  // one whitespace byte ends the header
  const int comp = f[1] == '5' ? 1 : 3;
  if (vals[0] <= 0 || vals[1] <= 0 || vals[2] <= 0 || vals[2] > 255) return DTB_ERR_INVALID_ARG;
  const size_t bytes = (size_t)vals[0] * (size_t)vals[1] * comp;
  if (pos + bytes > f.size()) return DTB_ERR_INVALID_ARG;
  out.w = (int)vals[0];
  out.h = (int)vals[1];
  out.channels = comp;
  out.data.assign(f.begin() + (long)pos, f.begin() + (long)(pos + bytes));
  return DTB_OK;
}

void png_chunk(std::vector<uint8_t>& png, const char* type, const uint8_t* body, size_t len) {
  put_be32(png, (uint32_t)len);
  const size_t at = png.size();
  png.insert(png.end(), type, type + 4);
  if (len) png.insert(png.end(), body, body + len);
  put_be32(png, (uint32_t)crc32(crc32(0L, Z_NULL, 0), &png[at], (uInt)(len + 4)));
}

}  // namespace

extern "C" {

static dtb_status image_read(const char* path, int32_t channels, dtb_image* out) {
  if (!path || !out || (channels != 1 && channels != 3)) return DTB_ERR_INVALID_ARG;
  std::vector<uint8_t> f;
  if (!read_file(path, f)) return DTB_ERR_IO;
  Pixels px;
  dtb_status s;
  if (f.size() >= 2 && f[0] == 0xFF && f[1] == 0xD8)  // JPEG start-of-image marker
    s = dtb_io::decode_jpeg(f.data(), f.size(), px);
  else
    s = (f.size() >= 2 && f[0] == 'P') ? decode_pnm(f, px) : decode_png(f, px);
  if (s != DTB_OK) return s;
  if (px.channels != channels) return DTB_ERR_INVALID_ARG;  // as the reference: no conversion between kinds
  if ((s = dtb_image_alloc(px.w, px.h, channels, DTB_CPU, out)) != DTB_OK) return s;
  for (int y = 0; y < px.h; ++y)
    std::memcpy(static_cast<uint8_t*>(out->buffer) + (size_t)y * out->pitch, &px.data[(size_t)y * px.w * channels],
                (size_t)px.w * channels);
  return DTB_OK;
}

static dtb_status image_write(const char* path, const dtb_image* img) {
  if (!path || !img || !img->buffer || img->memory_kind != DTB_CPU || (img->elem_size != 1 && img->elem_size != 3) ||
      img->width <= 0 || img->height <= 0 || img->pitch < img->width * img->elem_size)
    return DTB_ERR_INVALID_ARG;
  const std::string name(path);
  const size_t rb = (size_t)img->width * img->elem_size;
  const uint8_t* base = static_cast<const uint8_t*>(img->buffer);
  std::vector<uint8_t> file;
  if (ends_with(name, ".pgm") || ends_with(name, ".ppm")) {
    if ((img->elem_size == 1) != ends_with(name, ".pgm")) return DTB_ERR_INVALID_ARG;
    char hdr[64];
    const int n = std::snprintf(hdr, sizeof(hdr), "P%c\n%d %d\n255\n", img->elem_size == 1 ? '5' : '6', img->width,
                                img->height);
    file.assign(hdr, hdr + n);
    for (int y = 0; y < img->height; ++y) file.insert(file.end(), base + (size_t)y * img->pitch, base + (size_t)y * img->pitch + rb);
  } else if (ends_with(name, ".png")) {
    std::vector<uint8_t> raw;
    raw.reserve((rb + 1) * (size_t)img->height);
    for (int y = 0; y < img->height; ++y) {
      raw.push_back(0);  // filter type None
      raw.insert(raw.end(), base + (size_t)y * img->pitch, base + (size_t)y * img->pitch + rb);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) return DTB_ERR_IO;
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    file.assign(sig, sig + 8);
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, (uint32_t)img->width);
    put_be32(ihdr, (uint32_t)img->height);
    const uint8_t rest[5] = {8, (uint8_t)(img->elem_size == 1 ? 0 : 2), 0, 0, 0};
    ihdr.insert(ihdr.end(), rest, rest + 5);
    png_chunk(file, "IHDR", ihdr.data(), ihdr.size());
    png_chunk(file, "IDAT", z.data(), zlen);
    png_chunk(file, "IEND", nullptr, 0);
  } else {
    return DTB_ERR_INVALID_ARG;  // .png, .pgm or .ppm
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return DTB_ERR_IO;
  const bool ok = std::fwrite(file.data(), 1, file.size(), f) == file.size();
  return (std::fclose(f) == 0 && ok) ? DTB_OK : DTB_ERR_IO;
}

// No C++ exception crosses the C ABI: an allocation failure becomes a status.
DTB_API dtb_status dtb_image_read(const char* path, int32_t channels, dtb_image* out) {
  try {
    return image_read(path, channels, out);
  } catch (...) {
    return DTB_ERR_OUT_OF_MEMORY;
  }
}

DTB_API dtb_status dtb_image_write(const char* path, const dtb_image* img) {
  try {
    return image_write(path, img);
  } catch (...) {
    return DTB_ERR_OUT_OF_MEMORY;
  }
}

}  // extern "C"
