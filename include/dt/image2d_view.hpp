// dt/image2d_view.hpp -- non-owning pitched 2-D views, the interface of the reference's dt::image2d_view
// (dt/include/dt/image2d_view.hpp:9-126): e_memory_kind, image2d_view<void> (buffer, width, height, pitch,
// elem_size, memory kind; pixel (x, y) at buffer + y * pitch + x * elem_size) and the typed image2d_view<T>.
// Copies alias the same pixels; a move leaves the source without buffer (image2d_view.cpp:28-37 behaviour).
//
// These views are plain data and convert to the C ABI's dtb_image (include/dtb.h) field by field.
#pragma once

#include <dt/point2d.hpp>

#include <cassert>
#include <cstdint>
#include <type_traits>
#include <utility>

#include "dtb.h"

namespace dt
{
  enum class e_memory_kind
  {
    CPU = DTB_CPU,
    GPU = DTB_GPU
  };

  template <typename T>
  class image2d_view;

  template <>
  class image2d_view<void>
  {
  public:
    image2d_view() noexcept = default;
    image2d_view(std::uint8_t* buffer, int width, int height, int pitch, int elem_size,
                 e_memory_kind memory_kind = e_memory_kind::CPU) noexcept
      : m_buffer(buffer), m_width(width), m_height(height), m_pitch(pitch), m_elem_size(elem_size),
        m_memory_kind(memory_kind)
    {
    }
    image2d_view(const image2d_view&) noexcept            = default;
    image2d_view& operator=(const image2d_view&) noexcept = default;
    image2d_view(image2d_view&& o) noexcept { *this = std::move(o); }
    image2d_view& operator=(image2d_view&& o) noexcept
    {
      if (this != &o)
      {
        m_buffer      = std::exchange(o.m_buffer, nullptr);
        m_width       = o.m_width;
        m_height      = o.m_height;
        m_pitch       = o.m_pitch;
        m_elem_size   = o.m_elem_size;
        m_memory_kind = o.m_memory_kind;
      }
      return *this;
    }

    int                 width() const noexcept { return m_width; }
    int                 height() const noexcept { return m_height; }
    int                 pitch() const noexcept { return m_pitch; }
    int                 elem_size() const noexcept { return m_elem_size; }
    std::uint8_t*       buffer() noexcept { return m_buffer; }
    const std::uint8_t* buffer() const noexcept { return m_buffer; }
    e_memory_kind       memory_kind() const noexcept { return m_memory_kind; }

    bool valid() const noexcept { return m_buffer != nullptr; }
    bool in_domain(int x, int y) const noexcept { return x >= 0 && y >= 0 && x < m_width && y < m_height; }
    bool in_domain(const point2d& p) const noexcept { return in_domain(p.x(), p.y()); }

    // Address of pixel (x, y).  Dereferencing it is only meaningful for CPU views.
    std::uint8_t* operator()(int x, int y) noexcept
    {
      assert(in_domain(x, y) && m_buffer);
      return m_buffer + (static_cast<std::ptrdiff_t>(y) * m_pitch + static_cast<std::ptrdiff_t>(x) * m_elem_size);
    }
    const std::uint8_t* operator()(int x, int y) const noexcept
    {
      assert(in_domain(x, y) && m_buffer);
      return m_buffer + (static_cast<std::ptrdiff_t>(y) * m_pitch + static_cast<std::ptrdiff_t>(x) * m_elem_size);
    }
    std::uint8_t*       operator()(const point2d& p) noexcept { return (*this)(p.x(), p.y()); }
    const std::uint8_t* operator()(const point2d& p) const noexcept { return (*this)(p.x(), p.y()); }

    // The C ABI descriptor of this view.
    dtb_image desc() const noexcept
    {
      return dtb_image{const_cast<std::uint8_t*>(m_buffer), m_width, m_height, m_pitch, m_elem_size,
                       static_cast<int32_t>(m_memory_kind)};
    }

  protected:
    std::uint8_t* m_buffer      = nullptr;
    int           m_width       = 0;
    int           m_height      = 0;
    int           m_pitch       = 0;
    int           m_elem_size   = 0;
    e_memory_kind m_memory_kind = e_memory_kind::CPU;
  };

  template <typename T>
  class image2d_view : public image2d_view<void>
  {
  public:
    image2d_view() noexcept = default;
    image2d_view(T* buffer, int width, int height, int pitch, e_memory_kind memory_kind = e_memory_kind::CPU) noexcept
      : image2d_view<void>(reinterpret_cast<std::uint8_t*>(const_cast<std::remove_const_t<T>*>(buffer)), width, height,
                           pitch, sizeof(T), memory_kind)
    {
    }

    const T& operator()(int x, int y) const noexcept
    {
      return *reinterpret_cast<const T*>(image2d_view<void>::operator()(x, y));
    }
    T&       operator()(int x, int y) noexcept { return *reinterpret_cast<T*>(image2d_view<void>::operator()(x, y)); }
    const T& operator()(const point2d& p) const noexcept { return (*this)(p.x(), p.y()); }
    T&       operator()(const point2d& p) noexcept { return (*this)(p.x(), p.y()); }
  };
} // namespace dt
