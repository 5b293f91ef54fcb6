// dt/normalize.hpp -- map a CPU image linearly onto [0, 1] (floating-point output) or onto [0, max of O]
// (integer output), reference dt::minmax / dt::normalize (dt/include/dt/normalize.hpp:11-69): one pass for the
// extremes, one pass computing (v - min) / (max - min) in double, scaled and converted to O.
#pragma once

#include <dt/image2d.hpp>

#include <algorithm>
#include <concepts>
#include <limits>
#include <type_traits>
#include <utility>

namespace dt
{
  template <typename T>
  std::pair<std::remove_cvref_t<T>, std::remove_cvref_t<T>> minmax(const image2d_view<T>& in) noexcept
  {
    using V = std::remove_cvref_t<T>;
    V lo = std::numeric_limits<V>::max();
    V hi = std::numeric_limits<V>::lowest();
    for (int y = 0; y < in.height(); ++y)
      for (int x = 0; x < in.width(); ++x)
      {
        lo = std::min<V>(lo, in(x, y));
        hi = std::max<V>(hi, in(x, y));
      }
    return {lo, hi};
  }

  template <typename T, typename O>
  void normalize(const image2d_view<T>& in, image2d<O>& out) noexcept
  {
    const auto [lo, hi] = minmax(in);
    const double range = static_cast<double>(hi - lo);
    for (int y = 0; y < in.height(); ++y)
      for (int x = 0; x < in.width(); ++x)
      {
        double v = static_cast<double>(in(x, y) - lo) / range;
        if constexpr (!std::floating_point<O>)
          v *= std::numeric_limits<O>::max();
        out(x, y) = static_cast<O>(v);
      }
  }

  template <typename O, typename T>
  image2d<O> normalize(const image2d_view<T>& in)
  {
    image2d<O> out(in.width(), in.height());
    normalize(in, out);
    return out;
  }
} // namespace dt
