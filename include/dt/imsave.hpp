// dt/imsave.hpp -- write a uint8 or rgb8 image to a file, reference dt::imsave (dt/include/dt/imsave.hpp:9-43,
// dt/src/imsave.cpp): PNG as in the reference, or binary PGM / PPM, chosen by the file name.  Device images are
// copied to the host first.  Throws std::invalid_argument for another extension (the reference accepts .png
// only) and std::runtime_error when the file cannot be written.
#pragma once

#include <dt/details/status.hpp>
#include <dt/image2d_view.hpp>
#include <dt/rgb.hpp>
#include <dt/transfert.hpp>

#include <concepts>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace dt
{
  template <typename T>
    requires(std::same_as<std::remove_cvref_t<T>, std::uint8_t> || std::same_as<std::remove_cvref_t<T>, rgb8>)
  void imsave(const char* filename, const image2d_view<T>& img)
  {
    using V = std::remove_cvref_t<T>;
    image2d<V> host;
    dtb_image d = img.desc();
    if (img.memory_kind() == e_memory_kind::GPU)
    {
      host = image2d<V>(img.width(), img.height(), e_memory_kind::CPU);
      device_to_host(static_cast<const image2d_view<void>&>(img), static_cast<image2d_view<void>&>(host));
      d = host.desc();
    }
    const dtb_status s = dtb_image_write(filename, &d);
    if (s == DTB_ERR_INVALID_ARG)
      throw std::invalid_argument(std::string("Only PNG, PGM (gray) and PPM (rgb8) output is supported: ") + filename);
    if (s != DTB_OK)
      throw std::runtime_error(std::string("Failed to save ") + filename);
  }
} // namespace dt
