// dt/transfert.hpp -- host <-> device copies of pitched images, reference dt::host_to_device / dt::device_to_host
// (dt/include/dt/transfert.hpp:9-39, dt/src/transfert.cpp:10-28): synchronous 2-D copies between views of the
// same size and element size; the templated forms allocate the destination.
#pragma once

#include <dt/details/status.hpp>
#include <dt/image2d.hpp>

namespace dt
{
  inline void host_to_device(const image2d_view<void>& src, image2d_view<void>& dst)
  {
    const dtb_image s = src.desc(), d = dst.desc();
    details::check(dtb_host_to_device(&s, &d, nullptr), "host_to_device");
  }

  inline void device_to_host(const image2d_view<void>& src, image2d_view<void>& dst)
  {
    const dtb_image s = src.desc(), d = dst.desc();
    details::check(dtb_device_to_host(&s, &d, nullptr), "device_to_host");
  }

  template <typename T>
  image2d<T> host_to_device(const image2d_view<T>& src)
  {
    image2d<T> dst(src.width(), src.height(), e_memory_kind::GPU);
    host_to_device(static_cast<const image2d_view<void>&>(src), static_cast<image2d_view<void>&>(dst));
    return dst;
  }

  template <typename T>
  image2d<T> device_to_host(const image2d_view<T>& src)
  {
    image2d<T> dst(src.width(), src.height(), e_memory_kind::CPU);
    device_to_host(static_cast<const image2d_view<void>&>(src), static_cast<image2d_view<void>&>(dst));
    return dst;
  }
} // namespace dt
