// dtb_internal.h -- host-side types shared by the translation units of libdtb.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "dtb.h"

namespace dtb {

// One image of a call, resolved to device memory.
struct Job {
  const uint8_t* img = nullptr;
  int64_t img_pitch = 0;
  int channels = 1;
  const uint8_t* mask = nullptr;
  int64_t mask_pitch = 0;
  float* dist = nullptr;
  int64_t dist_pitch = 0;
  int width = 0, height = 0;
  float g2 = 0.0f, v = 0.0f, l_eucl = 0.0f, l_grad = 0.0f;
  int mode = 0, ref_fma = 1;

  int tiles_x() const { return (width + 31) / 32; }
  int tiles_y() const { return (height + 31) / 32; }

  static Job from(const dtb_image* img, const dtb_image* mask, const dtb_image* dist) {
    Job j;
    j.img = static_cast<const uint8_t*>(img->buffer);
    j.img_pitch = img->pitch;
    j.channels = img->elem_size;
    j.mask = static_cast<const uint8_t*>(mask->buffer);
    j.mask_pitch = mask->pitch;
    j.dist = static_cast<float*>(dist->buffer);
    j.dist_pitch = dist->pitch;
    j.width = img->width;
    j.height = img->height;
    return j;
  }
};

// g2 = fl32(gamma * gamma): the one place gamma is squared, so host and oracle agree on the bits.
inline float gamma_to_g2(float gamma) {
  const float g = gamma;
  return g * g;
}

dtb_status validate_view(dtb_context ctx, const dtb_image* im, const char* name, int elem_a, int elem_b);
dtb_status run_jobs(dtb_context ctx, const std::vector<Job>& jobs, const dtb_image* const* imgs,
                    const dtb_image* const* masks, const dtb_image* const* dists, uint32_t flags, cudaStream_t stream);

}  // namespace dtb
