// dt/point2d.hpp -- integer 2-D point, the interface of the reference's dt::point2d
// (dt/include/dt/point2d.hpp:5-38): constexpr construction, x()/y() accessors, equality, +, -, scaling.
#pragma once

namespace dt
{
  class point2d
  {
  public:
    constexpr point2d() noexcept = default;
    constexpr point2d(int x, int y) noexcept : m_x(x), m_y(y) {}

    constexpr int& x() noexcept { return m_x; }
    constexpr int  x() const noexcept { return m_x; }
    constexpr int& y() noexcept { return m_y; }
    constexpr int  y() const noexcept { return m_y; }

    constexpr bool operator==(const point2d& o) const noexcept { return m_x == o.m_x && m_y == o.m_y; }
    constexpr bool operator!=(const point2d& o) const noexcept { return !(*this == o); }

  private:
    int m_x = 0;
    int m_y = 0;
  };

  constexpr point2d operator+(const point2d& a, const point2d& b) noexcept { return {a.x() + b.x(), a.y() + b.y()}; }
  constexpr point2d operator-(const point2d& a, const point2d& b) noexcept { return {a.x() - b.x(), a.y() - b.y()}; }
  constexpr point2d operator*(const point2d& p, int k) noexcept { return {p.x() * k, p.y() * k}; }
  constexpr point2d operator*(int k, const point2d& p) noexcept { return p * k; }
} // namespace dt
