// ref_passes_driver.cu -- TEST INFRASTRUCTURE: runs the reference's own compiled tile-pass device functions.
//
// This translation unit is compiled (by oracle/Makefile, target `ref`) against the reference's source tree,
// where it lies: it includes dt/src/dt_block_passes.cuh, whose device functions
//   dt::pass<Forward>   (dt/src/dt_block_passes.cuh:12-68)   row sweeps of a 34x34 shared tile, C8 predecessors
//   dt::pass_T<Forward> (dt/src/dt_block_passes.cuh:71-127)  column sweeps
// hold the reference's ref-mode edge arithmetic `D(q) + l_eucl * local_dist2d[.] + l_grad * |dI|` exactly as
// nvcc compiles it (default --fmad=true, the reference's CMake adds no fp flag).  The output goes to
// oracle/_ref/ only and is never part of the product.
//
// Only the driver kernel below is ours.  It exists because the reference's own __global__ kernels take
// image2d_view by reference (host-stack addresses on the device, dt/src/generalised_distance_transform_blocks.cu:8),
// which cannot run on a GPU without HMM.  The driver works on images of at most 32x32 pixels, i.e. one tile
// of the reference's blocks variant: there, iterating the four passes to quiescence inside the tile
// (the loop of generalised_distance_transform_blocks.cu:58-76) is already the global fixpoint, so the result is
// the reference's map for that image.  The tile loader follows generalised_distance_transform_blocks.cu:27-45
// (out-of-image halo: image 0, distance v) and the initialisation follows dt/src/utils.cu:12
// (D = v * (mask == 0)); the weights table follows generalised_distance_transform_blocks.cu:125-126.
//
// The iteration count is capped (REFP_MAX_ITERS) so that every launch ends; hitting the cap is an error.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "dt_block_passes.cuh"

namespace {

constexpr int REFP_MAX_ITERS = 4096;

__global__ void __launch_bounds__(32) refp_tile_fixpoint(const uint8_t* __restrict__ img, const uint8_t* __restrict__ mask,
                                                         float* __restrict__ out, int w, int h, float v, float l_eucl,
                                                         float l_grad, int* __restrict__ err) {
  __shared__ std::uint8_t s_img[dt::TILE_SIZE][dt::TILE_SIZE];
  __shared__ float s_D[dt::TILE_SIZE][dt::TILE_SIZE];
  __shared__ int any_changed;

  const size_t base = static_cast<size_t>(blockIdx.x) * w * h;
  for (int i = threadIdx.x; i < dt::TILE_SIZE * dt::TILE_SIZE; i += blockDim.x) {
    const int ty = i / dt::TILE_SIZE, tx = i % dt::TILE_SIZE;
    const int gx = tx - 1, gy = ty - 1;
    const bool valid = gx >= 0 && gx < w && gy >= 0 && gy < h;
    s_img[ty][tx] = valid ? img[base + gy * w + gx] : 0;
    s_D[ty][tx] = valid ? v * (mask[base + gy * w + gx] == 0) : v;
  }
  __syncthreads();

  int iters = 0;
  for (;;) {
    int t = 0;
    t |= dt::pass<true>(s_img, s_D, w, h, l_eucl, l_grad, 0, 0, 1);
    __syncthreads();
    t |= dt::pass<false>(s_img, s_D, w, h, l_eucl, l_grad, 0, 0, 1);
    __syncthreads();
    t |= dt::pass_T<true>(s_img, s_D, w, h, l_eucl, l_grad, 0, 0, 1);
    __syncthreads();
    t |= dt::pass_T<false>(s_img, s_D, w, h, l_eucl, l_grad, 0, 0, 1);
    __syncthreads();
    if (threadIdx.x == 0) any_changed = 0;
    __syncthreads();
    if (t) atomicOr(&any_changed, 1);
    __syncthreads();
    const int c = any_changed;
    __syncthreads();
    if (!c) break;
    if (++iters >= REFP_MAX_ITERS) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
  }

  for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
    const int gy = i / w, gx = i % w;
    out[base + i] = s_D[gy + 1][gx + 1];
  }
}

}  // namespace

// n images of w x h pixels (w, h in [1, 32]), packed row-major in HOST memory: img and mask n*w*h bytes,
// out n*w*h floats.  Returns 0 on success, 1 on invalid arguments, 2 on a CUDA error, 3 if a tile hit the
// iteration cap.
extern "C" __attribute__((visibility("default"))) int refp_gdt_tiles(const uint8_t* img, const uint8_t* mask, float* out,
                                                                     int n, int w, int h, float lambda, float v) {
  if (n <= 0 || w < 1 || h < 1 || w > dt::BLOCK_SIZE || h > dt::BLOCK_SIZE || !img || !mask || !out) return 1;
  if (!(lambda >= 0.0f && lambda <= 1.0f)) return 1;
  const float l_grad = lambda;
  const float l_eucl = 1 - lambda;
  const float local_dist[] = {std::sqrt(2.f), 1.f, std::sqrt(2.f)};
  if (cudaMemcpyToSymbol(dt::local_dist2d, local_dist, sizeof(local_dist)) != cudaSuccess) return 2;

  const size_t px = static_cast<size_t>(n) * w * h;
  uint8_t *dimg = nullptr, *dmask = nullptr;
  float* dout = nullptr;
  int* derr = nullptr;
  int rc = 0, herr = 0;
  if (cudaMalloc(&dimg, px) != cudaSuccess || cudaMalloc(&dmask, px) != cudaSuccess ||
      cudaMalloc(&dout, px * sizeof(float)) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
    rc = 2;
  } else if (cudaMemcpy(dimg, img, px, cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemcpy(dmask, mask, px, cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemset(derr, 0, sizeof(int)) != cudaSuccess) {
    rc = 2;
  } else {
    refp_tile_fixpoint<<<n, 32>>>(dimg, dmask, dout, w, h, v, l_eucl, l_grad, derr);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(out, dout, px * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = 2;
    else if (herr)
      rc = 3;
  }
  cudaFree(dimg);
  cudaFree(dmask);
  cudaFree(dout);
  cudaFree(derr);
  return rc;
}
