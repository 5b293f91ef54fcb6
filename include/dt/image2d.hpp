// dt/image2d.hpp -- owning pitched image, the interface of the reference's dt::image2d<T>
// (dt/include/dt/image2d.hpp:13-50): image2d(width, height, memory_kind) allocates, copies share ownership of
// the same pixels (shared_ptr), and an image2d is an image2d_view<T>.  Storage comes from dtb_image_alloc: GPU
// rows pitched to 128 bytes, CPU rows packed (pitch = width * sizeof(T)), as the reference allocates them.
#pragma once

#include <dt/details/status.hpp>
#include <dt/image2d_view.hpp>

#include <memory>

namespace dt
{
  template <typename T>
  class image2d final : public image2d_view<T>
  {
  public:
    image2d()                          = default;
    image2d(const image2d&)            = default;
    image2d(image2d&&)                 = default;
    image2d& operator=(const image2d&) = default;
    image2d& operator=(image2d&&)      = default;

    image2d(int width, int height, e_memory_kind memory_kind = e_memory_kind::CPU)
    {
      dtb_image d{};
      details::check(dtb_image_alloc(width, height, static_cast<int32_t>(sizeof(T)), static_cast<int32_t>(memory_kind), &d),
                     "dtb_image_alloc");
      m_data = std::shared_ptr<void>(d.buffer, [d](void*) mutable { dtb_image_free(&d); });
      static_cast<image2d_view<void>&>(*this) =
          image2d_view<void>(static_cast<std::uint8_t*>(d.buffer), d.width, d.height, d.pitch, d.elem_size, memory_kind);
    }

  private:
    std::shared_ptr<void> m_data;
  };
} // namespace dt
