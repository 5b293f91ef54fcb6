// dtb_imgfile.h -- decoded host pixels shared by the image file readers (dtb_io.cpp: PNG, PGM / PPM;
// dtb_jpeg.cpp: JPEG).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "dtb.h"

namespace dtb_io {

// Host pixels: rows of w * channels bytes (packed).
struct Pixels {
  int w = 0, h = 0, channels = 0;
  std::vector<uint8_t> data;
};

// Largest image (in pixels) a reader accepts: beyond any image the library runs.
constexpr uint64_t kMaxFilePixels = 1ull << 31;

// Decodes a JPEG file held in memory.  Returns DTB_ERR_INVALID_ARG for a file that is not a JPEG this reader
// supports or whose headers are corrupt.
dtb_status decode_jpeg(const uint8_t* file, size_t size, Pixels& out);

}  // namespace dtb_io
