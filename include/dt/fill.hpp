// dt/fill.hpp -- set every pixel of a CPU view, reference dt::fill (dt/include/dt/fill.hpp:7-16).
#pragma once

#include <dt/image2d_view.hpp>

namespace dt
{
  template <typename T>
  void fill(image2d_view<T>& img, const T& val) noexcept
  {
    for (int y = 0; y < img.height(); ++y)
    {
      T* row = &img(0, y);
      for (int x = 0; x < img.width(); ++x)
        row[x] = val;
    }
  }
} // namespace dt
