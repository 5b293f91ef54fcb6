// dt/c8.hpp -- the 8-neighbourhood, reference dt::c8_t / dt::c8 (dt/include/dt/c8.hpp:9-32), same order: starting
// left and turning clockwise, (-1,0), (-1,-1), (0,-1), (1,-1), (1,0), (1,1), (0,1), (-1,1).  The
// reference-weight transform (lambda blend) relaxes over these neighbours.
#pragma once

#include <dt/point2d.hpp>

#include <array>
#include <ranges>

namespace dt
{
  class c8_t
  {
  public:
    static constexpr std::array<point2d, 8> offsets = {point2d{-1, 0}, point2d{-1, -1}, point2d{0, -1}, point2d{1, -1},
                                                       point2d{1, 0},  point2d{1, 1},   point2d{0, 1},  point2d{-1, 1}};

    constexpr c8_t() noexcept = default;
    auto operator()(const point2d& p) const noexcept
    {
      return std::views::transform(offsets, [p](const point2d& o) { return p + o; });
    }
  };

  inline constexpr c8_t c8 = {};
} // namespace dt
