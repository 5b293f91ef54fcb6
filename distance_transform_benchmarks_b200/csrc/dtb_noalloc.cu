// dtb_noalloc.cu -- dtb_gdt_noalloc: the single-image C4 geodesic distance transform without any allocation.
//
// Who needs it: a host that owns all device memory through its own pool or a fixed budget (a plugin inside a
// framework with its own allocator, a server that reserves its memory at start-up) cannot let a library call
// cudaMalloc behind its back, and a latency-critical loop cannot afford the device-wide synchronisation that
// cudaMalloc / cudaFree imply.  The regular entry points keep their scratch in a dtb_context, which allocates;
// this one keeps it in a fixed file-scope device array instead, so a call allocates nothing.
//
// The scratch (queue header, one state word per tile, one FIFO ticket ring -- no priority buckets -- and the
// image descriptor with its two TMA tensor maps) lives in g_noalloc_scratch below: NOALLOC_BYTES (about 324 KB) on every GPU that loads the
// library, held until the process exits.  It bounds the image to NOALLOC_MAX_TILES tiles of 32 x 32 pixels.
// All calls share the array and find the previous call's contents there; every call clears the queue header
// and the ring before use and rewrites the rest.  Two calls that overlap on the GPU (different host threads or
// streams) race on the array: callers must serialise them.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "dtb.h"
#include "dtb_kernels.cuh"

using namespace dtb;

namespace {

constexpr uint32_t NOALLOC_MAX_TILES = 16384;  // e.g. 4096 x 4096 pixels
constexpr uint32_t NOALLOC_RING = 65536;       // power of two, >= 2 * (tiles + resident warps + 64)
constexpr int NOALLOC_WPC = 4;
constexpr int NOALLOC_MINB = 2;
constexpr size_t NOALLOC_SMEM = NOALLOC_WPC * sizeof(WarpSmem) + 128;
constexpr uint64_t NOALLOC_TIMEOUT_NS = 2000000000ull;

constexpr size_t na_align(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t OFF_HDR = 0;
constexpr size_t OFF_DESC = na_align(OFF_HDR + sizeof(QueueHdr));
constexpr size_t OFF_TMAP = na_align(OFF_DESC + sizeof(ImgDesc));
constexpr size_t OFF_STATES = na_align(OFF_TMAP + 2 * sizeof(CUtensorMap));
constexpr size_t OFF_RING = na_align(OFF_STATES + 4ull * NOALLOC_MAX_TILES);
constexpr size_t NOALLOC_BYTES = na_align(OFF_RING + 4ull * NOALLOC_RING);

// The only scratch of dtb_gdt_noalloc.  In host code this name is a stand-in, not a device address: host code
// obtains the address with cudaGetSymbolAddress (once per device, see noalloc_setup).
static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_BYTES];

__device__ __forceinline__ QueueHdr* na_hdr() { return reinterpret_cast<QueueHdr*>(g_noalloc_scratch + OFF_HDR); }
__device__ __forceinline__ const ImgDesc* na_desc() {
  return reinterpret_cast<const ImgDesc*>(g_noalloc_scratch + OFF_DESC);
}
__device__ __forceinline__ const CUtensorMap* na_tmaps() {
  return reinterpret_cast<const CUtensorMap*>(g_noalloc_scratch + OFF_TMAP);
}
__device__ __forceinline__ uint32_t* na_states() { return reinterpret_cast<uint32_t*>(g_noalloc_scratch + OFF_STATES); }
__device__ __forceinline__ Queue na_queue(uint32_t max_visits, uint32_t tiles) {
  return Queue{na_hdr(), reinterpret_cast<uint32_t*>(g_noalloc_scratch + OFF_RING), NOALLOC_RING - 1, NOALLOC_TIMEOUT_NS,
               max_visits, tiles};
}

// Seed-tile scan of the one image (same work as ggdt_scan).
__global__ void __launch_bounds__(128) noalloc_scan(uint32_t max_visits, uint32_t tiles) {
  const Queue q = na_queue(max_visits, tiles);
  const ImgDesc& dd = *na_desc();
  uint32_t* states = na_states();
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tiles; t += nwarps) {
    const int tx = (int)(t % (uint32_t)dd.tiles_x), ty = (int)(t / (uint32_t)dd.tiles_x);
    const int x0 = tx * TILE, y0 = ty * TILE;
    const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
    bool nz = false;
    if (lane < vh) {
      const uint8_t* row = dd.mask + (int64_t)(y0 + lane) * dd.mask_pitch + x0;
      for (int c = 0; c < vw; ++c) nz |= row[c] != 0;
    }
    nz = __any_sync(~0u, nz);
    if (lane == 0) {
      states[t] = nz ? (ST_SEED | ST_PENDING) : 0u;
      if (nz) queue_push(q, t);
    }
  }
}

// Persistent tile worker of the one image (same loop as ggdt_persistent, ns-mode).
__global__ void __launch_bounds__(NOALLOC_WPC * 32, NOALLOC_MINB) noalloc_persistent(uint32_t max_visits, uint32_t tiles) {
  extern __shared__ uint8_t smem_raw[];
  WarpSmem& sm = warp_slot(smem_raw);
  warp_slot_init(sm);
  const Queue q = na_queue(max_visits, tiles);
  uint32_t* states = na_states();
  const QueueSched sch{q, states};
  const int lane = threadIdx.x & 31;
  uint32_t parity = 0;
  WarpStats ws;
  for (;;) {
    const uint32_t t = queue_pop(q);  // one FIFO ring: this scratch holds no priority buckets
    if (t == POP_NONE) break;
    uint32_t old = 0;
    if (lane == 0) old = atomicXor(&states[t], ST_PENDING | ST_RUNNING);
    old = __shfl_sync(~0u, old, 0);
    const ImgDesc dd = *na_desc();
    visit_tile<MODE_NS>(dd, na_tmaps(), 0u, t, old, sm, parity, sch, ws);
  }
  flush_stats(ws, q);
}

// v into tiles never reached.
__global__ void __launch_bounds__(128) noalloc_finalize(uint32_t tiles) {
  const ImgDesc& dd = *na_desc();
  const uint32_t* states = na_states();
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tiles; t += nwarps) {
    if (states[t] & ST_VISITED) continue;
    const int tx = (int)(t % (uint32_t)dd.tiles_x), ty = (int)(t / (uint32_t)dd.tiles_x);
    const int x0 = tx * TILE, y0 = ty * TILE;
    const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
    if (lane < vw)
      for (int y = 0; y < vh; ++y) dist_row(dd, y0 + y)[x0 + lane] = dd.v;
  }
}

// Per-device set-up, done by the first call on each device with that device current, and again after the
// device's context changed (cudaDeviceReset ends the primary context; the symbol address and the kernel
// attribute belong to the old one).
typedef CUresult (*PFN_ctx_get_current)(CUcontext*);
struct NoallocDevice {
  bool ready = false;
  CUcontext ctx = nullptr;     // context the entry below was set up in
  uint8_t* scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int num_sms = 0;
  int blocks_per_sm = 0;
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
};
constexpr int NOALLOC_MAX_DEVICES = 64;
NoallocDevice g_devices[NOALLOC_MAX_DEVICES];
std::mutex g_setup_mu;

PFN_ctx_get_current g_ctx_get_current = nullptr;

dtb_status noalloc_setup(int dev, NoallocDevice** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return DTB_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_ctx_get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess || !fn)
      return DTB_ERR_NO_DEVICE;
    g_ctx_get_current = reinterpret_cast<PFN_ctx_get_current>(fn);
  }
  // cudaSetDevice on the current device makes its primary context current (initialising it if needed).
  if (cudaSetDevice(dev) != cudaSuccess) return DTB_ERR_CUDA;
  CUcontext cur = nullptr;
  if (g_ctx_get_current(&cur) != CUDA_SUCCESS || !cur) return DTB_ERR_NO_DEVICE;
  NoallocDevice& d = g_devices[dev];
  if (d.ready && d.ctx != cur) d = NoallocDevice{};
  if (!d.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DTB_ERR_CUDA;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess || !fn)
      return DTB_ERR_NO_DEVICE;
    int sms = 0, bps = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return DTB_ERR_CUDA;
    if (cudaFuncSetAttribute(noalloc_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)NOALLOC_SMEM) != cudaSuccess)
      return DTB_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, noalloc_persistent, NOALLOC_WPC * 32, NOALLOC_SMEM) != cudaSuccess ||
        bps < 1)
      return DTB_ERR_NO_DEVICE;
    d.scratch = static_cast<uint8_t*>(p);
    d.num_sms = sms;
    d.blocks_per_sm = bps;
    d.encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    d.ctx = cur;
    d.ready = true;
  }
  *out = &d;
  return DTB_OK;
}

bool noalloc_encode(const NoallocDevice& d, CUtensorMap* out, const void* base, uint64_t row_bytes, uint64_t rows,
                    uint64_t pitch, uint32_t box_w, uint32_t box_h) {
  cuuint64_t dims[2] = {row_bytes, rows};
  cuuint64_t strides[1] = {pitch};
  cuuint32_t box[2] = {box_w, box_h};
  cuuint32_t estr[2] = {1, 1};
  return d.encode(out, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool aligned16(const dtb_image* im) {
  return (reinterpret_cast<uintptr_t>(im->buffer) & 15u) == 0 && (im->pitch & 15) == 0;
}

}  // namespace

extern "C" DTB_API dtb_status dtb_gdt_noalloc(const dtb_image* img, const dtb_image* mask, const dtb_image* dist,
                                              float gamma, float v, void* stream) {
  if (!img || !mask || !dist) return DTB_ERR_INVALID_ARG;
  if ((img->elem_size != 1 && img->elem_size != 3) || mask->elem_size != 1 || dist->elem_size != 4)
    return DTB_ERR_INVALID_ARG;
  if (img->width != mask->width || img->height != mask->height || img->width != dist->width || img->height != dist->height)
    return DTB_ERR_INVALID_ARG;
  if (img->width < 0 || img->height < 0) return DTB_ERR_INVALID_ARG;
  if (!(gamma >= 0.0f) || std::isinf(gamma) || !(v >= 0.0f)) return DTB_ERR_INVALID_ARG;
  const int W = img->width, H = img->height;
  const uint64_t tiles64 = (uint64_t)((W + TILE - 1) / TILE) * (uint64_t)((H + TILE - 1) / TILE);
  if (tiles64 > NOALLOC_MAX_TILES) return DTB_ERR_CAPACITY;
  if (W == 0 || H == 0) return DTB_OK;
  if (img->memory_kind != DTB_GPU || mask->memory_kind != DTB_GPU || dist->memory_kind != DTB_GPU)
    return DTB_ERR_INVALID_ARG;
  if (!img->buffer || !mask->buffer || !dist->buffer) return DTB_ERR_INVALID_ARG;
  if ((int64_t)img->pitch < (int64_t)W * img->elem_size || mask->pitch < W || (int64_t)dist->pitch < (int64_t)W * 4)
    return DTB_ERR_INVALID_ARG;
  if (!aligned16(img) || !aligned16(mask) || (reinterpret_cast<uintptr_t>(dist->buffer) & 3u) || (dist->pitch & 3))
    return DTB_ERR_INVALID_ARG;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DTB_ERR_NO_DEVICE;
  NoallocDevice* nd = nullptr;
  dtb_status s = noalloc_setup(dev, &nd);
  if (s != DTB_OK) return s;

  const uint32_t tiles = (uint32_t)tiles64;
  const uint32_t workers = (uint32_t)(nd->num_sms * nd->blocks_per_sm * NOALLOC_WPC);
  uint32_t grid = (uint32_t)(nd->num_sms * nd->blocks_per_sm);
  if (2ull * (tiles + workers + 64) > NOALLOC_RING) {
    // keep every waiting popper and every queued tile on a distinct ring slot
    const uint32_t max_workers = NOALLOC_RING / 2 - tiles - 64;
    grid = std::max<uint32_t>(1, max_workers / NOALLOC_WPC);
  }
  const uint32_t max_visits = (uint32_t)std::min<uint64_t>(0xF0000000ull, 4096ull * tiles + (1ull << 20));

  ImgDesc desc{};
  desc.img = static_cast<const uint8_t*>(img->buffer);
  desc.mask = static_cast<const uint8_t*>(mask->buffer);
  desc.dist = static_cast<float*>(dist->buffer);
  desc.img_pitch = img->pitch;
  desc.mask_pitch = mask->pitch;
  desc.dist_pitch = dist->pitch;
  desc.width = W;
  desc.height = H;
  desc.channels = img->elem_size;
  desc.tiles_x = (W + TILE - 1) / TILE;
  desc.tiles_y = (H + TILE - 1) / TILE;
  desc.tile_base = 0;
  desc.g2 = gamma * gamma;
  desc.v = v;
  desc.mode = MODE_NS;
  alignas(64) CUtensorMap tm[2];
  if (!noalloc_encode(*nd, &tm[0], img->buffer, (uint64_t)W * img->elem_size, (uint64_t)H, (uint64_t)img->pitch,
                      img->elem_size == 3 ? IMG_BOX_RGB : IMG_BOX_GRAY, IMG_BOX_ROWS) ||
      !noalloc_encode(*nd, &tm[1], mask->buffer, (uint64_t)W, (uint64_t)H, (uint64_t)mask->pitch, TILE, TILE))
    return DTB_ERR_INVALID_ARG;

  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  uint8_t* sc = nd->scratch;
  // Source buffers are pageable host memory: each copy has consumed its source when the call returns.
  if (cudaMemcpyAsync(sc + OFF_DESC, &desc, sizeof(desc), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(sc + OFF_TMAP, tm, sizeof(tm), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(sc + OFF_HDR, 0, sizeof(QueueHdr), st) != cudaSuccess ||
      cudaMemsetAsync(sc + OFF_RING, 0, 4ull * NOALLOC_RING, st) != cudaSuccess)
    return DTB_ERR_CUDA;
  const uint32_t scan_blocks = std::min<uint32_t>((tiles + 3) / 4, (uint32_t)nd->num_sms * 16);
  noalloc_scan<<<scan_blocks, 128, 0, st>>>(max_visits, tiles);
  if (cudaGetLastError() != cudaSuccess) return DTB_ERR_CUDA;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(NOALLOC_WPC * 32);
  cfg.dynamicSmemBytes = NOALLOC_SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, noalloc_persistent, max_visits, tiles) != cudaSuccess) return DTB_ERR_CUDA;
  noalloc_finalize<<<scan_blocks, 128, 0, st>>>(tiles);
  if (cudaGetLastError() != cudaSuccess) return DTB_ERR_CUDA;
  uint32_t err = 0;
  if (cudaMemcpyAsync(&err, sc + OFF_HDR + offsetof(QueueHdr, error), sizeof(err), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return DTB_ERR_CUDA;
  if (err == DERR_QUEUE_TIMEOUT || err == DERR_TMA_TIMEOUT) return DTB_ERR_TIMEOUT;
  if (err != DERR_NONE) return DTB_ERR_DEVICE;
  return DTB_OK;
}
