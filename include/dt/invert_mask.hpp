// dt/invert_mask.hpp -- 1 where a CPU seed mask is 0, 0 elsewhere, reference dt::invert_mask
// (dt/include/dt/invert_mask.hpp:7, dt/src/invert_mask.cpp).
#pragma once

#include <dt/image2d.hpp>

#include <cstdint>

namespace dt
{
  inline image2d<std::uint8_t> invert_mask(const image2d_view<std::uint8_t>& mask)
  {
    image2d<std::uint8_t> out(mask.width(), mask.height());
    for (int y = 0; y < mask.height(); ++y)
      for (int x = 0; x < mask.width(); ++x)
        out(x, y) = mask(x, y) == 0 ? 1 : 0;
    return out;
  }
} // namespace dt
