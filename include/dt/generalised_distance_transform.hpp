// dt/generalised_distance_transform.hpp -- the reference's GGDT entry points in namespace dt, over the C ABI of
// dtb.h.
//
// Same overloads, argument meaning and defaults as dt/include/dt/generalised_distance_transform.hpp:7-27:
//   generalised_distance_transform{,_blocks,_task}(img, mask, dist, lambda, v = 1e10 [, round_per_blocks])
//   image2d<float> generalised_distance_transform{,_blocks,_task}(img, mask, lambda, v = 1e10 [, round_per_blocks])
// with the reference weight D(q) + (1 - lambda) * {1, sqrt2} + lambda * |I(p) - I(q)| over the 8-neighbourhood.
// All three variants return the same map, bit for bit (the greatest fixpoint of the relaxations); `_blocks` runs
// host-driven rounds and fills round_per_blocks (ceil(W/32) * ceil(H/32) counters, host or device memory) when
// given one.
//
// Added here: the C4 geodesic transform w = sqrt(1 + gamma^2 |dI|^2) on gray or rgb8 images, selected by passing
// dt::c4 (dt/include/dt/c4.hpp), and a ragged batch of such images in one launch.
//
// Differences from the reference, all on the caller's side of the contract: images may live in CPU or GPU
// memory (the reference asserts GPU; CPU views are copied through the device by the library); a precondition
// that the reference asserts (same shapes, 0 <= lambda <= 1) throws dt::error instead; calls are thread-safe.
// Allocating overloads return an image2d<float> in the memory kind of `img`.
#pragma once

#include <dt/c4.hpp>
#include <dt/details/status.hpp>
#include <dt/image2d.hpp>
#include <dt/rgb.hpp>

#include <cstdint>
#include <span>
#include <vector>

namespace dt
{
  namespace details
  {
    inline void gdt_ref(const image2d_view<void>& img, const image2d_view<void>& mask, image2d_view<void>& dist,
                        float lambda, float v, bool rounds, int* round_per_blocks)
    {
      const dtb_image a = img.desc(), b = mask.desc(), c = dist.desc();
      dtb_context ctx = context();
      if (rounds && round_per_blocks)
        check(dtb_gdt_ref_blocks(ctx, &a, &b, &c, lambda, v, round_per_blocks, 0, nullptr),
              "generalised_distance_transform_blocks", ctx);
      else
        check(dtb_gdt_ref(ctx, &a, &b, &c, lambda, v, rounds ? DTB_FLAG_ROUNDS : 0u, nullptr),
              "generalised_distance_transform", ctx);
    }

    inline void gdt_c4(const image2d_view<void>& img, const image2d_view<void>& mask, image2d_view<void>& dist,
                       float gamma, float v)
    {
      const dtb_image a = img.desc(), b = mask.desc(), c = dist.desc();
      dtb_context ctx = context();
      check(dtb_gdt(ctx, &a, &b, &c, gamma, v, 0u, nullptr), "generalised_distance_transform (c4)", ctx);
    }
  } // namespace details

  // ---- reference weight, C8 (generalised_distance_transform.hpp:7-27) ----

  inline void generalised_distance_transform(const image2d_view<std::uint8_t>& img, const image2d_view<std::uint8_t>& mask,
                                             image2d_view<float>& dist, float lambda, float v = 1e10)
  {
    details::gdt_ref(img, mask, dist, lambda, v, false, nullptr);
  }

  inline image2d<float> generalised_distance_transform(const image2d_view<std::uint8_t>& img,
                                                       const image2d_view<std::uint8_t>& mask, float lambda, float v = 1e10)
  {
    image2d<float> dist(img.width(), img.height(), img.memory_kind());
    generalised_distance_transform(img, mask, dist, lambda, v);
    return dist;
  }

  inline void generalised_distance_transform_blocks(const image2d_view<std::uint8_t>& img,
                                                    const image2d_view<std::uint8_t>& mask, image2d_view<float>& dist,
                                                    float lambda, float v = 1e10, int* round_per_blocks = nullptr)
  {
    details::gdt_ref(img, mask, dist, lambda, v, true, round_per_blocks);
  }

  inline image2d<float> generalised_distance_transform_blocks(const image2d_view<std::uint8_t>& img,
                                                              const image2d_view<std::uint8_t>& mask, float lambda,
                                                              float v = 1e10, int* round_per_blocks = nullptr)
  {
    image2d<float> dist(img.width(), img.height(), img.memory_kind());
    generalised_distance_transform_blocks(img, mask, dist, lambda, v, round_per_blocks);
    return dist;
  }

  inline void generalised_distance_transform_task(const image2d_view<std::uint8_t>& img,
                                                  const image2d_view<std::uint8_t>& mask, image2d_view<float>& D,
                                                  float lambda, float v = 1e10)
  {
    details::gdt_ref(img, mask, D, lambda, v, false, nullptr);
  }

  inline image2d<float> generalised_distance_transform_task(const image2d_view<std::uint8_t>& img,
                                                            const image2d_view<std::uint8_t>& mask, float lambda,
                                                            float v = 1e10)
  {
    image2d<float> dist(img.width(), img.height(), img.memory_kind());
    generalised_distance_transform_task(img, mask, dist, lambda, v);
    return dist;
  }

  // ---- C4 geodesic weight w = sqrt(1 + gamma^2 |dI|^2), gray and rgb8 ----

  inline void generalised_distance_transform(const image2d_view<std::uint8_t>& img, const image2d_view<std::uint8_t>& mask,
                                             image2d_view<float>& dist, c4_t, float gamma, float v = 1e10)
  {
    details::gdt_c4(img, mask, dist, gamma, v);
  }

  inline void generalised_distance_transform(const image2d_view<rgb8>& img, const image2d_view<std::uint8_t>& mask,
                                             image2d_view<float>& dist, c4_t, float gamma, float v = 1e10)
  {
    details::gdt_c4(img, mask, dist, gamma, v);
  }

  inline image2d<float> generalised_distance_transform(const image2d_view<std::uint8_t>& img,
                                                       const image2d_view<std::uint8_t>& mask, c4_t nbh, float gamma,
                                                       float v = 1e10)
  {
    image2d<float> dist(img.width(), img.height(), img.memory_kind());
    generalised_distance_transform(img, mask, dist, nbh, gamma, v);
    return dist;
  }

  inline image2d<float> generalised_distance_transform(const image2d_view<rgb8>& img, const image2d_view<std::uint8_t>& mask,
                                                       c4_t nbh, float gamma, float v = 1e10)
  {
    image2d<float> dist(img.width(), img.height(), img.memory_kind());
    generalised_distance_transform(img, mask, dist, nbh, gamma, v);
    return dist;
  }

  // Ragged batch of C4 geodesic transforms in one persistent launch: imgs[i] gray (elem_size 1) or rgb8
  // (elem_size 3), masks[i] uint8, dists[i] float, gammas[i] per image.  All spans have the same length.
  inline void generalised_distance_transform_batch(std::span<const image2d_view<void>> imgs,
                                                   std::span<const image2d_view<void>> masks,
                                                   std::span<image2d_view<void>> dists, std::span<const float> gammas,
                                                   c4_t = c4, float v = 1e10)
  {
    const size_t n = imgs.size();
    if (masks.size() != n || dists.size() != n || gammas.size() != n)
      throw error(DTB_ERR_INVALID_ARG, "generalised_distance_transform_batch: spans of different lengths");
    std::vector<dtb_image> a(n), b(n), c(n);
    for (size_t i = 0; i < n; ++i)
    {
      a[i] = imgs[i].desc();
      b[i] = masks[i].desc();
      c[i] = dists[i].desc();
    }
    dtb_context ctx = details::context();
    details::check(dtb_gdt_batch(ctx, static_cast<int32_t>(n), a.data(), b.data(), c.data(), gammas.data(), v, 0u, nullptr),
                   "generalised_distance_transform_batch", ctx);
  }
} // namespace dt
