// dt/c4.hpp -- the 4-neighbourhood, reference dt::c4_t / dt::c4 (dt/include/dt/c4.hpp:9-27).
// c4(p) is the range of p's four neighbours in the order (-1,0), (0,-1), (1,0), (0,1).  Passing dt::c4 to
// generalised_distance_transform selects the C4 geodesic weight w = sqrt(1 + gamma^2 |dI|^2).
#pragma once

#include <dt/point2d.hpp>

#include <array>
#include <ranges>

namespace dt
{
  class c4_t
  {
  public:
    static constexpr std::array<point2d, 4> offsets = {point2d{-1, 0}, point2d{0, -1}, point2d{1, 0}, point2d{0, 1}};

    constexpr c4_t() noexcept = default;
    auto operator()(const point2d& p) const noexcept
    {
      return std::views::transform(offsets, [p](const point2d& o) { return p + o; });
    }
  };

  inline constexpr c4_t c4 = {};
} // namespace dt
