// dt/imread.hpp -- read an image file into a CPU image, reference dt::imread (dt/include/dt/imread.hpp:7-8,
// dt/src/imread.cpp): imread<std::uint8_t> wants a one-component (gray) file, imread<rgb8> a three-component
// one.  Formats: 8-bit PNG, binary PGM / PPM and JPEG (dtb_image_read; gray JPEG samples identical to stb_image's);
// the reference reads any stb_image format.
// Throws std::runtime_error when the file cannot be read, std::invalid_argument when it has the wrong number of
// components or an unsupported encoding.
#pragma once

#include <dt/image2d.hpp>
#include <dt/rgb.hpp>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace dt
{
  template <typename T>
  image2d<T> imread(const char* filename)
  {
    static_assert(std::is_same_v<T, std::uint8_t> || std::is_same_v<T, rgb8>, "imread reads uint8 or rgb8 images");
    dtb_image file{};
    const dtb_status s = dtb_image_read(filename, static_cast<int32_t>(sizeof(T)), &file);
    if (s == DTB_ERR_IO)
      throw std::runtime_error(std::string("Error while loading ") + filename);
    if (s == DTB_ERR_INVALID_ARG)
      throw std::invalid_argument(std::string("Input image must have ") + (sizeof(T) == 1 ? "1 component" : "3 components") +
                                  " of 8 bits (PNG, PGM, PPM or JPEG): " + filename);
    details::check(s, "imread");
    image2d<T> out(file.width, file.height);
    for (int y = 0; y < file.height; ++y)
      std::memcpy(&out(0, y), static_cast<const std::uint8_t*>(file.buffer) + static_cast<size_t>(y) * file.pitch,
                  static_cast<size_t>(file.width) * sizeof(T));
    dtb_image_free(&file);
    return out;
  }
} // namespace dt
