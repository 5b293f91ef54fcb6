// dt/rgb.hpp -- 3-byte interleaved colour pixel, the layout of the reference's dt::rgb8 (dt/include/dt/rgb.hpp:7-12).
// An image2d_view<rgb8> has elem_size 3, the rgb8 input of the C4 geodesic transform.
#pragma once

#include <cstdint>

namespace dt
{
  struct rgb8
  {
    std::uint8_t r;
    std::uint8_t g;
    std::uint8_t b;
  };
  static_assert(sizeof(rgb8) == 3, "rgb8 must be 3 packed bytes");
} // namespace dt
