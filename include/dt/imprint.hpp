// dt/imprint.hpp -- print a CPU image as rows of numbers, reference dt::imprint (dt/include/dt/imprint.hpp:7-11,
// dt/src/imprint.cpp): one "[a b c]" line per row, uint8 right-aligned in 3 columns, float with 5 decimals.
#pragma once

#include <dt/image2d_view.hpp>

#include <cstdint>
#include <cstdio>
#include <iostream>
#include <type_traits>

namespace dt
{
  template <typename T>
  void imprint(const image2d_view<T>& img, std::ostream& out = std::cout)
  {
    static_assert(std::is_same_v<T, std::uint8_t> || std::is_same_v<T, float>, "imprint: uint8 or float images");
    char buf[64];
    for (int y = 0; y < img.height(); ++y)
    {
      out << '[';
      for (int x = 0; x < img.width(); ++x)
      {
        if constexpr (std::is_same_v<T, std::uint8_t>)
          std::snprintf(buf, sizeof(buf), "%3u", static_cast<unsigned>(img(x, y)));
        else
          std::snprintf(buf, sizeof(buf), "%.5f", static_cast<double>(img(x, y)));
        out << buf << (x + 1 < img.width() ? " " : "]\n");
      }
      if (img.width() == 0)
        out << "]\n";
    }
  }
} // namespace dt
