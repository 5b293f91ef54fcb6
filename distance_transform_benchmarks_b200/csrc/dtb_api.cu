// dtb_api.cu -- kernels and the C ABI (include/dtb.h) of the B200 GGDT.
//
// Host flow of one call (all stream-ordered, no host round trip except in the plain rounds path):
//   descriptor tables + TMA tensor maps -> device (one copy), queue header reset,
//   ggdt_scan (seed tiles), ggdt_persistent (cooperative, all tiles of all images), ggdt_finalize.
// The reference's host drivers (dt/src/generalised_distance_transform*.cu) instead poll a managed flag
// after every round; the plain path (DTB_FLAG_ROUNDS) keeps that structure as the per-image baseline.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dtb.h"
#include "dtb_internal.h"
#include "dtb_kernels.cuh"

using namespace dtb;

// ======================================================================================================
// Kernels
// ======================================================================================================
namespace dtb {

// Seed-tile scan: one warp per tile, every mask byte read once (lane = row, two 16-byte loads per row).
// Writes the tile state (image index, SEED, PENDING / VISITED) and queues (or marks active) seed tiles.
__global__ void __launch_bounds__(128) ggdt_scan(const ImgDesc* __restrict__ descs, const uint32_t* __restrict__ tile_base,
                                                 int n, uint32_t total, uint32_t* __restrict__ states, Queue q,
                                                 uint8_t* __restrict__ active, int warm) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = warp; t < total; t += nwarps) {
    const uint32_t img = image_of_tile(tile_base, n, t);
    const ImgDesc& dd = descs[img];
    const uint32_t local = t - dd.tile_base;
    const int tx = (int)(local % (uint32_t)dd.tiles_x), ty = (int)(local / (uint32_t)dd.tiles_x);
    const int x0 = tx * TILE, y0 = ty * TILE;
    const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
    bool nz = false;
    if (lane < vh) {
      const uint8_t* row = dd.mask + (int64_t)(y0 + lane) * dd.mask_pitch + x0;
      if (vw == TILE && (reinterpret_cast<uintptr_t>(row) & 15u) == 0) {
        const uint4 a = reinterpret_cast<const uint4*>(row)[0];
        const uint4 b = reinterpret_cast<const uint4*>(row)[1];
        nz = (a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) != 0u;
      } else {
        for (int c = 0; c < vw; ++c) nz |= row[c] != 0;
      }
    }
    nz = __any_sync(~0u, nz);
    if (lane == 0) {
      uint32_t st = (img << ST_IMG_SHIFT) | (warm ? ST_VISITED : 0u);
      if (nz) st |= ST_SEED | (active ? 0u : ST_PENDING);
      states[t] = st;
      if (nz) {
        if (active) active[t] = 1;
        else queue_push(q, t);
      }
    }
  }
}

// Persistent tile worker.  Every warp loops: take the tile its last visit kept (QueueSched::keep_out) or pop
// one, visit it, until the queue drains.
template <int MODE, int WPC, int MINB>
__global__ void __launch_bounds__(WPC * 32, MINB)
    ggdt_persistent(const ImgDesc* __restrict__ descs, const CUtensorMap* __restrict__ tmaps, uint32_t* states, Queue q) {
  extern __shared__ uint8_t smem_raw[];
  WarpSmem& sm = warp_slot(smem_raw);
  warp_slot_init(sm);
  uint32_t parity = 0;
  const int lane = threadIdx.x & 31;
  if (lane == 0) sm.keep = POP_NONE;
  __syncwarp();
  const QueueSched sch{q, states, &sm.keep};
  WarpStats ws;
  uint32_t prev = POP_NONE;  // the tile this warp visited last
  for (;;) {
    uint32_t t = sm.keep;
    __syncwarp();
    const bool again = t != POP_NONE && t == prev;  // kept its own tile: its weights and distances are in smem
    if (t == POP_NONE) {
      t = queue_pop(q);
      if (t == POP_NONE) break;
    } else if (lane == 0) {
      sm.keep = POP_NONE;
    }
    prev = t;
    uint32_t old = 0;
    if (lane == 0) {
      old = atomicXor(&states[t], ST_PENDING | ST_RUNNING);
      if (q.keys) q.keys[t] = KEY_NONE;  // activations from here on belong to the next queue entry
    }
    old = __shfl_sync(~0u, old, 0);
    const uint32_t img = old >> ST_IMG_SHIFT;
    if constexpr (MODE == MODE_NS) {
      const ImgDesc dd = descs[img];
      // A re-run needs the tile visited (weights and B from that visit) and no new seeds to apply.
      visit_tile<MODE>(dd, tmaps, img, t, old, sm, parity, sch, ws, again && (old & ST_VISITED) && !(old & ST_SEED));
    } else {
      // ref-mode reads the descriptor fields where it uses them (read-only, cached) instead of holding a copy
      // in registers through the visit.
      visit_tile<MODE>(descs[img], tmaps, img, t, old, sm, parity, sch, ws,
                       again && (old & ST_VISITED) && !(old & ST_SEED));
    }
  }
  flush_stats(ws, q);
}

// Persistent tile worker that stages ahead (ns-mode): while a warp visits tile k it has the image box of its
// next tile in flight into the other box of its slot.  The next tile comes from a non-blocking pop (an item a
// pusher has already reserved); when there is none, the warp pops blocking after the visit, as the worker
// above does.  A tile is claimed (PENDING -> RUNNING) only when its visit starts, so activations that reach
// it while it waits are covered by that visit (it reads its halo after the claim) instead of forcing a re-run.
template <int WPC, int MINB>
__global__ void __launch_bounds__(WPC * 32, MINB)
    ggdt_persistent_ahead(const ImgDesc* __restrict__ descs, const CUtensorMap* __restrict__ tmaps, uint32_t* states,
                          Queue q) {
  extern __shared__ uint8_t smem_raw[];
  WarpSmemP& sm = warp_slot_p(smem_raw);
  warp_slot_init(sm);
  const QueueSched sch{q, states};
  const int lane = threadIdx.x & 31;
  WarpStats ws;
  uint32_t pbits = 0;  // bit k: phase parity of box k's barrier; bit 2: the mask barrier's
  uint32_t k = 0;      // box of the tile being visited
  uint32_t cur = queue_pop(q);
  if (cur != POP_NONE) stage_ahead(descs, tmaps, states, cur, sm.box[0], &sm.bar[0]);
  while (cur != POP_NONE) {
    uint32_t nxt = queue_try_pop(q);
    if (nxt != POP_NONE) stage_ahead(descs, tmaps, states, nxt, sm.box[k ^ 1u], &sm.bar[k ^ 1u]);
    uint32_t old = 0;
    if (lane == 0) {
      old = atomicXor(&states[cur], ST_PENDING | ST_RUNNING);
      if (q.keys) q.keys[cur] = KEY_NONE;  // activations from here on belong to the next queue entry
    }
    old = __shfl_sync(~0u, old, 0);
    const uint32_t img = old >> ST_IMG_SHIFT;
    const ImgDesc dd = descs[img];
    const VisitBufs vb{sm.box[k], sm.Wh, sm.Wv, &sm.bar[k], &sm.mbar, 1u << k, 4u, &pbits};
    uint32_t nph, nact;
    visit_ns<true>(dd, tmaps + 2 * img, tmaps + 2 * img + 1, cur, old, vb, sch, &nph, &nact);
    count_visit(ws, q, nph, nact);
    if (nxt == POP_NONE) {
      nxt = queue_pop(q);
      if (nxt != POP_NONE) stage_ahead(descs, tmaps, states, nxt, sm.box[k ^ 1u], &sm.bar[k ^ 1u]);
    }
    cur = nxt;
    k ^= 1u;
  }
  flush_stats(ws, q);
}

// One host-driven round: one warp per tile, inactive tiles return at once.
template <int MODE, int WPC>
__global__ void __launch_bounds__(WPC * 32)
    ggdt_round(const ImgDesc* __restrict__ descs, const CUtensorMap* __restrict__ tmaps, uint32_t* states,
               const uint8_t* __restrict__ active, uint8_t* next_active, uint32_t* changed, uint32_t total, Queue q) {
  extern __shared__ uint8_t smem_raw[];
  WarpSmem& sm = warp_slot(smem_raw);
  const uint32_t t = blockIdx.x * WPC + (threadIdx.x >> 5);
  if (t >= total || !active[t]) return;
  warp_slot_init(sm);
  uint32_t parity = 0;
  const uint32_t old = ld_volatile(&states[t]);
  const uint32_t img = old >> ST_IMG_SHIFT;
  const RoundSched sch{q, states, next_active, changed};
  const ImgDesc dd = descs[img];
  WarpStats ws;
  visit_tile<MODE>(dd, tmaps, img, t, old, sm, parity, sch, ws);
  flush_stats(ws, q);
}

// dtb_gdt_ref_blocks: counts[t] += 1 for every tile visited in this round.
__global__ void __launch_bounds__(256) ggdt_count_round(int32_t* __restrict__ counts, const uint8_t* __restrict__ active,
                                                        uint32_t total) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) counts[t] += active[t] ? 1 : 0;
}

// counts[t] += add[t] (device-resident caller counters of dtb_gdt_ref_blocks).
__global__ void __launch_bounds__(256) ggdt_add_counts(int32_t* __restrict__ counts, const int32_t* __restrict__ add,
                                                       uint32_t total) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) counts[t] += add[t];
}

// dtb_debug_inject_queue_stall: counts one queued tile that is never pushed, so `pending` cannot reach 0 and the
// workers idle in queue_pop until the no-progress watchdog sets DERR_QUEUE_TIMEOUT and every worker returns.
__global__ void ggdt_phantom_pending(QueueHdr* hdr) { atomicAdd(&hdr->pending.v, 1u); }

// Tiles never reached keep uninitialised memory: write v there.  With `fold`, one thread also adds the run's
// queue header `hdr` into the accumulator `fold` (first error kept, counters summed): runs of the host-buffer
// pipeline report their status this way, on their own stream, without a separate kernel.
__global__ void __launch_bounds__(128) ggdt_finalize(const ImgDesc* __restrict__ descs, const uint32_t* __restrict__ tile_base,
                                                     int n, uint32_t total, const uint32_t* __restrict__ states,
                                                     const QueueHdr* hdr, QueueHdr* fold) {
  const int lane = threadIdx.x & 31;
  if (fold && blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t err = hdr->error.v;
    if (err != 0u && atomicCAS(&fold->error.v, 0u, err) == 0u) fold->err_info.v = hdr->err_info.v;
    atomicAdd(&fold->progress.v, hdr->progress.v);
    atomicAdd(&fold->phases.v, hdr->phases.v);
    atomicAdd(&fold->activations.v, hdr->activations.v);
  }
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = warp; t < total; t += nwarps) {
    if (states[t] & ST_VISITED) continue;
    const uint32_t img = image_of_tile(tile_base, n, t);
    const ImgDesc& dd = descs[img];
    const uint32_t local = t - dd.tile_base;
    const int tx = (int)(local % (uint32_t)dd.tiles_x), ty = (int)(local / (uint32_t)dd.tiles_x);
    const int x0 = tx * TILE, y0 = ty * TILE;
    const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
    if (lane < vw)
      for (int y = 0; y < vh; ++y) dist_row(dd, y0 + y)[x0 + lane] = dd.v;
  }
}

}  // namespace dtb

// ======================================================================================================
// Host side
// ======================================================================================================
namespace dtb {

static nvtxDomainHandle_t trace_domain() {
  static nvtxDomainHandle_t d = nvtxDomainCreateA("dtb");
  return d;
}
TraceRange::TraceRange(const char* name) {
  nvtxEventAttributes_t a{};
  a.version = NVTX_VERSION;
  a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
  a.messageType = NVTX_MESSAGE_TYPE_ASCII;
  a.message.ascii = name;
  nvtxDomainRangePushEx(trace_domain(), &a);
}
TraceRange::~TraceRange() { nvtxDomainRangePop(trace_domain()); }

dtb_status fail(dtb_context ctx, dtb_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->msg = buf;
  return s;
}

dtb_status cuda_fail(dtb_context ctx, cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) return fail(ctx, DTB_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return fail(ctx, DTB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

static uint32_t next_pow2(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

dtb_status grow(dtb_context ctx, void** p, size_t* size, size_t need) {
  if (*size >= need) return DTB_OK;
  if (*p) {
    cudaDeviceSynchronize();
    cudaFree(*p);
    *p = nullptr;
    *size = 0;
  }
  const size_t sz = align_up(need + need / 4, 1 << 20);
  cudaError_t e = cudaMalloc(p, sz);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(ctx, e, "cudaMalloc(scratch)");
  }
  *size = sz;
  return DTB_OK;
}

static bool encode_u8_2d(dtb_context ctx, CUtensorMap* out, const void* base, uint64_t row_bytes, uint64_t rows,
                         uint64_t pitch, uint32_t box_w, uint32_t box_h) {
  cuuint64_t dims[2] = {row_bytes, rows};
  cuuint64_t strides[1] = {pitch};
  cuuint32_t box[2] = {box_w, box_h};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = ctx->encode(out, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

dtb_status validate_view(dtb_context ctx, const dtb_image* im, const char* name, int elem_a, int elem_b) {
  if (!im) return fail(ctx, DTB_ERR_INVALID_ARG, "%s is NULL", name);
  if (im->width < 0 || im->height < 0) return fail(ctx, DTB_ERR_INVALID_ARG, "%s has a negative size", name);
  if (im->elem_size != elem_a && im->elem_size != elem_b)
    return fail(ctx, DTB_ERR_INVALID_ARG, "%s: unsupported elem_size %d", name, im->elem_size);
  if (im->memory_kind != DTB_CPU && im->memory_kind != DTB_GPU)
    return fail(ctx, DTB_ERR_INVALID_ARG, "%s: unknown memory_kind %d", name, im->memory_kind);
  if (im->width > 0 && im->height > 0) {
    if (!im->buffer) return fail(ctx, DTB_ERR_INVALID_ARG, "%s: NULL buffer", name);
    if ((int64_t)im->pitch < (int64_t)im->width * im->elem_size)
      return fail(ctx, DTB_ERR_INVALID_ARG, "%s: pitch %d < width * elem_size", name, im->pitch);
  }
  return DTB_OK;
}

dtb_status check_triplet(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist,
                         bool allow_rgb) {
  dtb_status s;
  if ((s = validate_view(ctx, img, "img", 1, allow_rgb ? 3 : 1)) != DTB_OK) return s;
  if ((s = validate_view(ctx, mask, "mask", 1, 1)) != DTB_OK) return s;
  if ((s = validate_view(ctx, dist, "dist", 4, 4)) != DTB_OK) return s;
  if (img->width != mask->width || img->height != mask->height || img->width != dist->width || img->height != dist->height)
    return fail(ctx, DTB_ERR_INVALID_ARG, "img, mask and dist must have the same size");
  return DTB_OK;
}

dtb_status count_tiles(dtb_context ctx, const std::vector<Job>& jobs, uint32_t* total) {
  uint64_t t = 0;
  for (const Job& j : jobs) t += (uint64_t)j.tiles_x() * j.tiles_y();
  // 2^28 tiles (275 Gpx) is far beyond device memory; the limit keeps the ring capacity (a power of two >=
  // 2 * (tiles + workers)) and the 31-bit tile ids of the queue items in range.
  if (t >= (1ull << 28) || jobs.size() >= (1u << 23))
    return fail(ctx, DTB_ERR_CAPACITY, "too many tiles (%llu) or images (%zu)", (unsigned long long)t, jobs.size());
  *total = (uint32_t)t;
  return DTB_OK;
}

uint32_t resident_workers(dtb_context ctx, int mode, const LaunchTuning& t) {
  const int bps = mode == MODE_NS ? ctx->ns_blocks_per_sm[t.variant] : ctx->ref_blocks_per_sm;
  const uint32_t ctas = std::max<uint32_t>(1u, (uint32_t)(ctx->num_sms * bps) * (uint32_t)t.grid_percent / 100u);
  return ctas * (uint32_t)(mode == MODE_NS ? NS_VARIANT_TABLE[t.variant].wpc : PERSIST_WPC);
}

ScratchLayout layout_for(int n, uint32_t total, uint32_t workers, bool rounds, uint32_t buckets) {
  ScratchLayout L;
  L.n = n;
  L.total = total;
  L.cap = next_pow2((uint32_t)std::min<uint64_t>(2ull * ((uint64_t)total + workers + 64u), 1ull << 31));
  L.nb = std::max<uint32_t>(1u, std::min<uint32_t>(next_pow2(std::max<uint32_t>(buckets, 1u)), NBUCKET_MAX));
  size_t off = 0;
  L.o_hdr = off;    off = align_up(off + sizeof(QueueHdr), 256);
  L.o_states = off; off = align_up(off + 4ull * std::max<uint32_t>(total, 1), 256);
  L.o_ring = off;   off = align_up(off + L.ring_bytes(), 256);
  L.o_keys = off;   off = align_up(off + (L.nb > 1 ? 4ull * std::max<uint32_t>(total, 1) : 0), 256);
  L.o_wacc = off;   off = align_up(off + (L.nb > 1 ? 8ull * (size_t)std::max(n, 1) : 0), 256);
  L.o_desc = off;   off = align_up(off + sizeof(ImgDesc) * (size_t)std::max(n, 1), 256);
  L.o_tmap = off;   off = align_up(off + sizeof(CUtensorMap) * 2 * (size_t)std::max(n, 1), 256);
  L.o_base = off;   off = align_up(off + 4ull * (n + 1), 256);
  L.o_act = off;    off = align_up(off + (rounds ? 2ull * std::max<uint32_t>(total, 1) : 0), 256);
  L.o_chg = off;    off = align_up(off + 4, 256);
  L.bytes = off;
  return L;
}

dtb_status fill_desc(dtb_context ctx, const Job& j, uint32_t tile_base, int index, ImgDesc* d, CUtensorMap* tm) {
  d->img = j.img;
  d->mask = j.mask;
  d->dist = j.dist;
  d->img_pitch = j.img_pitch;
  d->mask_pitch = j.mask_pitch;
  d->dist_pitch = j.dist_pitch;
  d->width = j.width;
  d->height = j.height;
  d->channels = j.channels;
  d->tiles_x = j.tiles_x();
  d->tiles_y = j.tiles_y();
  d->tile_base = tile_base;
  d->g2 = j.g2;
  d->v = j.v;
  d->l_eucl = j.l_eucl;
  d->l_grad = j.l_grad;
  d->mode = j.mode;
  d->ref_fma = j.ref_fma;
  if (j.width > 0 && j.height > 0) {
    const uint32_t bw = j.channels == 3 ? IMG_BOX_RGB : IMG_BOX_GRAY;
    if (!encode_u8_2d(ctx, &tm[0], j.img, (uint64_t)j.width * j.channels, (uint64_t)j.height, (uint64_t)j.img_pitch, bw,
                      IMG_BOX_ROWS))
      return fail(ctx, DTB_ERR_INVALID_ARG, "image %d: cuTensorMapEncodeTiled rejected the image layout", index);
    if (!encode_u8_2d(ctx, &tm[1], j.mask, (uint64_t)j.width, (uint64_t)j.height, (uint64_t)j.mask_pitch, TILE, TILE))
      return fail(ctx, DTB_ERR_INVALID_ARG, "image %d: cuTensorMapEncodeTiled rejected the mask layout", index);
  }
  return DTB_OK;
}

dtb_status build_tables(dtb_context ctx, const std::vector<Job>& jobs, const ScratchLayout& L, std::vector<uint8_t>& out) {
  const int n = (int)jobs.size();
  out.assign(L.o_act - L.o_desc, 0);
  ImgDesc* hdesc = reinterpret_cast<ImgDesc*>(out.data());
  CUtensorMap* htm = reinterpret_cast<CUtensorMap*>(out.data() + (L.o_tmap - L.o_desc));
  uint32_t* hbase = reinterpret_cast<uint32_t*>(out.data() + (L.o_base - L.o_desc));
  uint32_t base = 0;
  for (int i = 0; i < n; ++i) {
    const dtb_status s = fill_desc(ctx, jobs[i], base, i, &hdesc[i], &htm[2 * i]);
    if (s != DTB_OK) return s;
    hbase[i] = base;
    base += (uint32_t)(hdesc[i].tiles_x * hdesc[i].tiles_y);
  }
  hbase[n] = base;
  return DTB_OK;
}

dtb_status pinned_stage(dtb_context ctx, size_t need, uint8_t** out, cudaEvent_t* ev) {
  const int i = ctx->hpin_cur;
  ctx->hpin_cur ^= 1;
  if (!ctx->hpin_ev[i]) DTB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->hpin_ev[i], cudaEventDisableTiming));
  if (ctx->hpin_used[i]) DTB_CUDA(ctx, cudaEventSynchronize(ctx->hpin_ev[i]));
  if (ctx->hpin_size[i] < need) {
    if (ctx->hpin[i]) cudaFreeHost(ctx->hpin[i]);
    ctx->hpin[i] = nullptr;
    ctx->hpin_size[i] = 0;
    const size_t sz = std::max<size_t>(need + need / 4, 1 << 20);
    if (cudaHostAlloc(&ctx->hpin[i], sz, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, DTB_ERR_OUT_OF_MEMORY, "cudaHostAlloc of %zu bytes failed", sz);
    }
    ctx->hpin_size[i] = sz;
  }
  ctx->hpin_used[i] = true;
  *out = static_cast<uint8_t*>(ctx->hpin[i]);
  *ev = ctx->hpin_ev[i];
  return DTB_OK;
}

uint64_t tuning_key(int n, uint32_t total) {
  return ((uint64_t)next_pow2((uint32_t)std::max(n, 1)) << 32) | next_pow2(std::max<uint32_t>(total, 1));
}

bool valid_policy(int buckets, float bucket_tiles) {
  return buckets >= 1 && buckets <= (int)NBUCKET_MAX && (buckets & (buckets - 1)) == 0 && bucket_tiles > 0.0f &&
         bucket_tiles <= 64.0f;
}

Queue make_queue(uint8_t* dbase, const ScratchLayout& L, uint64_t timeout_ns, const LaunchTuning* t) {
  const uint64_t cap_visits = std::min<uint64_t>(0xF0000000ull, 4096ull * L.total + (1ull << 20));
  // A tile is re-visited only after a strict decrease of a neighbour's border; real inputs stay far below
  // this cap, which only turns a scheduling bug into an error instead of an endless run.
  Queue q{reinterpret_cast<QueueHdr*>(dbase + L.o_hdr), reinterpret_cast<uint32_t*>(dbase + L.o_ring), L.cap - 1,
          timeout_ns, (uint32_t)cap_visits, L.total};
  const uint32_t nb = t ? std::min<uint32_t>(L.nb, (uint32_t)t->buckets) : L.nb;
  if (nb > 1) {
    q.nb_mask = nb - 1;
    q.keys = reinterpret_cast<uint32_t*>(dbase + L.o_keys);
    q.wacc = reinterpret_cast<float*>(dbase + L.o_wacc);
  }
  q.bucket_tiles = t ? t->bucket_tiles : DEFAULT_BUCKET_TILES;
  return q;
}

dtb_status reset_queue(dtb_context ctx, uint8_t* dbase, const ScratchLayout& L, cudaStream_t stream) {
  DTB_CUDA(ctx, cudaMemsetAsync(dbase + L.o_hdr, 0, sizeof(QueueHdr), stream));
  DTB_CUDA(ctx, cudaMemsetAsync(dbase + L.o_ring, 0, L.ring_bytes(), stream));
  if (L.nb > 1) {
    DTB_CUDA(ctx, cudaMemsetAsync(dbase + L.o_keys, 0xFF, 4ull * std::max<uint32_t>(L.total, 1), stream));  // KEY_NONE
    DTB_CUDA(ctx, cudaMemsetAsync(dbase + L.o_wacc, 0, 8ull * (size_t)std::max(L.n, 1), stream));
  }
  return DTB_OK;
}

dtb_status enqueue_persistent(dtb_context ctx, uint8_t* dbase, const ScratchLayout& L, int mode, const LaunchTuning& t,
                              cudaStream_t stream, cudaEvent_t ev0, cudaEvent_t ev1, QueueHdr* fold) {
  const uint64_t stall_ns = ctx->inject_stall_ns;
  ctx->inject_stall_ns = 0;
  Queue q = make_queue(dbase, L, stall_ns ? stall_ns : DEFAULT_TIMEOUT_NS, &t);
  const ImgDesc* ddesc = reinterpret_cast<const ImgDesc*>(dbase + L.o_desc);
  const CUtensorMap* dtm = reinterpret_cast<const CUtensorMap*>(dbase + L.o_tmap);
  const uint32_t* dtile_base = reinterpret_cast<const uint32_t*>(dbase + L.o_base);
  uint32_t* states = reinterpret_cast<uint32_t*>(dbase + L.o_states);
  dtb_status rs = reset_queue(ctx, dbase, L, stream);
  if (rs != DTB_OK) return rs;
  if (L.total == 0) return DTB_OK;
  const int n = L.n;
  const uint32_t total = L.total;
  const uint32_t scan_blocks = std::min<uint32_t>((total + 3) / 4, (uint32_t)ctx->num_sms * 16);
  ggdt_scan<<<scan_blocks, 128, 0, stream>>>(ddesc, dtile_base, n, total, states, q, nullptr, 0);
  DTB_CUDA(ctx, cudaGetLastError());
  if (stall_ns) {
    ggdt_phantom_pending<<<1, 1, 0, stream>>>(q.hdr);
    DTB_CUDA(ctx, cudaGetLastError());
  }
  if (ev0) DTB_CUDA(ctx, cudaEventRecord(ev0, stream));
  dtb_status ls = launch_tile_kernel(ctx, mode, t, ddesc, dtm, states, q, stream);
  if (ls != DTB_OK) return ls;
  if (ev1) DTB_CUDA(ctx, cudaEventRecord(ev1, stream));
  ggdt_finalize<<<scan_blocks, 128, 0, stream>>>(ddesc, dtile_base, n, total, states, q.hdr, fold);
  DTB_CUDA(ctx, cudaGetLastError());
  return DTB_OK;
}

dtb_status launch_tile_kernel(dtb_context ctx, int mode, const LaunchTuning& t, const ImgDesc* descs,
                              const CUtensorMap* tmaps, uint32_t* states, const Queue& q, cudaStream_t stream) {
  cudaLaunchConfig_t cfg{};
  const int wpc = mode == MODE_NS ? NS_VARIANT_TABLE[t.variant].wpc : PERSIST_WPC;
  cfg.gridDim = dim3(resident_workers(ctx, mode, t) / (uint32_t)wpc);
  cfg.blockDim = dim3((uint32_t)wpc * 32u);
  cfg.dynamicSmemBytes = mode == MODE_NS ? ctx->ns_smem[t.variant] : PERSIST_SMEM;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;  // guarantees co-residency of all workers (the slot waits need it)
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  Queue qa = q;
  void* args[4] = {(void*)&descs, (void*)&tmaps, (void*)&states, (void*)&qa};
  const void* fn = mode == MODE_NS ? ctx->ns_fn[t.variant]
                   : mode == MODE_REF ? (const void*)ggdt_persistent<MODE_REF, PERSIST_WPC, REF_CTAS>
                                      : (const void*)ggdt_persistent<MODE_REF_NOFMA, PERSIST_WPC, REF_CTAS>;
  DTB_CUDA(ctx, cudaLaunchKernelExC(&cfg, fn, args));
  return DTB_OK;
}

// Host-driven rounds (the plain per-image path).  Synchronises once per round, like the reference's
// blocks variant (generalised_distance_transform_blocks.cu:156-163).
static dtb_status run_rounds(dtb_context ctx, uint8_t* dbase, const ScratchLayout& L, int mode, cudaStream_t stream,
                             uint64_t* nrounds) {
  Queue q = make_queue(dbase, L);  // rounds use only the counters and the error word of the queue
  const ImgDesc* ddesc = reinterpret_cast<const ImgDesc*>(dbase + L.o_desc);
  const CUtensorMap* dtm = reinterpret_cast<const CUtensorMap*>(dbase + L.o_tmap);
  const uint32_t* dtile_base = reinterpret_cast<const uint32_t*>(dbase + L.o_base);
  uint32_t* states = reinterpret_cast<uint32_t*>(dbase + L.o_states);
  QueueHdr* hdr = reinterpret_cast<QueueHdr*>(dbase + L.o_hdr);
  const uint32_t total = L.total;
  uint8_t* act0 = dbase + L.o_act;
  uint8_t* act1 = dbase + L.o_act + total;
  uint32_t* changed = reinterpret_cast<uint32_t*>(dbase + L.o_chg);
  DTB_CUDA(ctx, cudaMemsetAsync(hdr, 0, sizeof(QueueHdr), stream));
  *nrounds = 0;
  if (total == 0) return DTB_OK;
  const uint32_t scan_blocks = std::min<uint32_t>((total + 3) / 4, (uint32_t)ctx->num_sms * 16);
  DTB_CUDA(ctx, cudaMemsetAsync(act0, 0, 2ull * total, stream));
  ggdt_scan<<<scan_blocks, 128, 0, stream>>>(ddesc, dtile_base, L.n, total, states, q, act0, 0);
  DTB_CUDA(ctx, cudaGetLastError());
  // ref-mode: the first round visits every tile, as the reference's blocks variant does (all blocks active,
  // dt/src/generalised_distance_transform_blocks.cu:149-151), so per-tile round counters count the same rounds.
  if (mode != MODE_NS) DTB_CUDA(ctx, cudaMemsetAsync(act0, 1, total, stream));
  uint8_t* cur = act0;
  uint8_t* nxt = act1;
  uint32_t hchanged = 1;
  while (hchanged) {
    DTB_CUDA(ctx, cudaMemsetAsync(nxt, 0, total, stream));
    DTB_CUDA(ctx, cudaMemsetAsync(changed, 0, 4, stream));
    const uint32_t blocks = (total + ROUND_WPC - 1) / ROUND_WPC;
    if (ctx->count_rounds) {
      ggdt_count_round<<<std::min<uint32_t>((total + 255) / 256, (uint32_t)ctx->num_sms * 8), 256, 0, stream>>>(
          ctx->dround_counts, cur, total);
      DTB_CUDA(ctx, cudaGetLastError());
    }
    if (mode == MODE_NS)
      ggdt_round<MODE_NS, ROUND_WPC><<<blocks, ROUND_WPC * 32, ROUND_SMEM, stream>>>(ddesc, dtm, states, cur, nxt, changed, total, q);
    else if (mode == MODE_REF)
      ggdt_round<MODE_REF, ROUND_WPC><<<blocks, ROUND_WPC * 32, ROUND_SMEM, stream>>>(ddesc, dtm, states, cur, nxt, changed, total, q);
    else
      ggdt_round<MODE_REF_NOFMA, ROUND_WPC><<<blocks, ROUND_WPC * 32, ROUND_SMEM, stream>>>(ddesc, dtm, states, cur, nxt, changed,
                                                                                           total, q);
    DTB_CUDA(ctx, cudaGetLastError());
    uint32_t err_prog[2] = {0, 0};
    DTB_CUDA(ctx, cudaMemcpyAsync(&hchanged, changed, 4, cudaMemcpyDeviceToHost, stream));
    DTB_CUDA(ctx, cudaMemcpyAsync(&err_prog[0], &hdr->error.v, 4, cudaMemcpyDeviceToHost, stream));
    DTB_CUDA(ctx, cudaMemcpyAsync(&err_prog[1], &hdr->progress.v, 4, cudaMemcpyDeviceToHost, stream));
    DTB_CUDA(ctx, cudaStreamSynchronize(stream));
    std::swap(cur, nxt);
    ++*nrounds;
    if (err_prog[0]) break;
    if (err_prog[1] > q.max_visits)
      return fail(ctx, DTB_ERR_DEVICE, "visit limit exceeded after %llu rounds", (unsigned long long)*nrounds);
  }
  ggdt_finalize<<<scan_blocks, 128, 0, stream>>>(ddesc, dtile_base, L.n, total, states, nullptr, nullptr);
  DTB_CUDA(ctx, cudaGetLastError());
  return DTB_OK;
}

// Resolves the user views of one or more images into device jobs, staging copies where the user memory is
// on the host or lacks the 16-byte alignment of TMA (input) / 4-byte alignment of float rows (output).
struct Staged {
  const dtb_image* user;
  uint8_t* dev;
  int64_t pitch;
  bool copy_in;
  bool copy_out;
};

static bool tma_ok(const dtb_image* im) {
  return im->memory_kind == DTB_GPU && (reinterpret_cast<uintptr_t>(im->buffer) & 15u) == 0 && (im->pitch & 15) == 0;
}
static bool dist_ok(const dtb_image* im) {
  return im->memory_kind == DTB_GPU && (reinterpret_cast<uintptr_t>(im->buffer) & 3u) == 0 && (im->pitch & 3) == 0;
}

dtb_status run_jobs(dtb_context ctx, const std::vector<Job>& jobs_in, const dtb_image* const* imgs,
                    const dtb_image* const* masks, const dtb_image* const* dists, uint32_t flags, cudaStream_t stream) {
  const TraceRange trace("dtb call");
  const int n = (int)jobs_in.size();
  std::vector<Job> jobs = jobs_in;

  // Serialise with a previous asynchronous call on another stream (the scratch is shared; host-buffer pipeline
  // calls have their own).
  if (ctx->async_pending && ctx->last_stream != stream) DTB_CUDA(ctx, cudaStreamSynchronize(ctx->last_stream));
  ctx->async_pending = false;

  bool all_host = n > 0 && !(flags & DTB_FLAG_ROUNDS);
  for (int i = 0; i < n && all_host; ++i)
    all_host = jobs[i].mode == MODE_NS && imgs[i]->memory_kind == DTB_CPU && masks[i]->memory_kind == DTB_CPU &&
               dists[i]->memory_kind == DTB_CPU;
  if (all_host) return run_host_pipeline(ctx, jobs, imgs, masks, dists, flags, stream);

  // ---- staging of inputs / outputs that are on the host or not aligned for TMA ----
  std::vector<Staged> staged;
  size_t stage_bytes = 0;
  for (int i = 0; i < n; ++i) {
    if (jobs[i].width == 0 || jobs[i].height == 0) continue;
    const dtb_image* in3[3] = {imgs[i], masks[i], dists[i]};
    for (int k = 0; k < 3; ++k) {
      const dtb_image* u = in3[k];
      if ((k < 2) ? tma_ok(u) : dist_ok(u)) continue;
      const int64_t row = (int64_t)u->width * u->elem_size;
      const int64_t pitch = (int64_t)align_up((size_t)row, 128);
      staged.push_back({u, reinterpret_cast<uint8_t*>(stage_bytes), pitch, k < 2, k == 2});
      stage_bytes += align_up((size_t)(pitch * u->height), 256);
    }
  }
  if (stage_bytes) {
    dtb_status s = grow(ctx, &ctx->dstage, &ctx->dstage_size, stage_bytes);
    if (s != DTB_OK) return s;
    for (auto& st : staged) st.dev = reinterpret_cast<uint8_t*>(ctx->dstage) + reinterpret_cast<uintptr_t>(st.dev);
  }
  auto find_stage = [&](const dtb_image* u) -> const Staged* {
    for (auto& st : staged)
      if (st.user == u) return &st;
    return nullptr;
  };
  for (int i = 0; i < n; ++i) {
    if (jobs[i].width == 0 || jobs[i].height == 0) continue;
    if (const Staged* st = find_stage(imgs[i])) {
      jobs[i].img = st->dev;
      jobs[i].img_pitch = st->pitch;
    }
    if (const Staged* st = find_stage(masks[i])) {
      jobs[i].mask = st->dev;
      jobs[i].mask_pitch = st->pitch;
    }
    if (const Staged* st = find_stage(dists[i])) {
      jobs[i].dist = reinterpret_cast<float*>(st->dev);
      jobs[i].dist_pitch = st->pitch;
    }
  }
  for (auto& st : staged) {
    if (!st.copy_in) continue;
    const dtb_image* u = st.user;
    const cudaMemcpyKind kind = u->memory_kind == DTB_CPU ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    DTB_CUDA(ctx, cudaMemcpy2DAsync(st.dev, (size_t)st.pitch, u->buffer, (size_t)u->pitch, (size_t)u->width * u->elem_size,
                                    (size_t)u->height, kind, stream));
  }

  // ---- descriptor tables and scratch ----
  uint32_t total = 0;
  dtb_status s = count_tiles(ctx, jobs, &total);
  if (s != DTB_OK) return s;
  const bool rounds = (flags & DTB_FLAG_ROUNDS) != 0;
  for (int i = 1; i < n; ++i)
    if (jobs[i].mode != jobs[0].mode || jobs[i].ref_fma != jobs[0].ref_fma)
      return fail(ctx, DTB_ERR_INVALID_ARG, "one call covers images of one weight mode");
  // Kernel mode: ref-mode calls with left-to-right rounding run their own kernels.
  const int mode = n == 0 ? MODE_NS : (jobs[0].mode == MODE_REF && !jobs[0].ref_fma) ? MODE_REF_NOFMA : jobs[0].mode;
  LaunchTuning tuning = ctx->tuning;
  auto it = ctx->tuned.find(tuning_key(n, total));
  if (it != ctx->tuned.end()) tuning = it->second;
  const ScratchLayout L = layout_for(n, total, resident_workers(ctx, mode, tuning), rounds,
                                     rounds ? 1u : (uint32_t)tuning.buckets);
  if ((s = grow(ctx, &ctx->dscratch, &ctx->dscratch_size, L.bytes)) != DTB_OK) return s;
  uint8_t* dbase = reinterpret_cast<uint8_t*>(ctx->dscratch);
  if ((s = build_tables(ctx, jobs, L, ctx->hstage)) != DTB_OK) return s;
  {  // from pinned memory: the copy never waits for earlier work on the stream
    uint8_t* hp = nullptr;
    cudaEvent_t ev_host = nullptr;
    if ((s = pinned_stage(ctx, ctx->hstage.size(), &hp, &ev_host)) != DTB_OK) return s;
    std::copy(ctx->hstage.begin(), ctx->hstage.end(), hp);
    DTB_CUDA(ctx, cudaMemcpyAsync(dbase + L.o_desc, hp, ctx->hstage.size(), cudaMemcpyHostToDevice, stream));
    DTB_CUDA(ctx, cudaEventRecord(ev_host, stream));
  }

  uint64_t nrounds = 1;
  const bool timed = (flags & DTB_FLAG_TIMING) && !rounds && total > 0;
  if (rounds) {
    if ((s = run_rounds(ctx, dbase, L, mode, stream, &nrounds)) != DTB_OK) return s;
  } else {
    if ((s = enqueue_persistent(ctx, dbase, L, mode, tuning, stream, timed ? ctx->ev[0] : nullptr,
                                timed ? ctx->ev[1] : nullptr)) != DTB_OK)
      return s;
  }

  // ---- copy staged outputs back ----
  bool host_io = false;
  for (auto& st : staged) {
    host_io |= st.user->memory_kind == DTB_CPU;
    if (!st.copy_out) continue;
    const dtb_image* u = st.user;
    const cudaMemcpyKind kind = u->memory_kind == DTB_CPU ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    DTB_CUDA(ctx, cudaMemcpy2DAsync(u->buffer, (size_t)u->pitch, st.dev, (size_t)st.pitch, (size_t)u->width * u->elem_size,
                                    (size_t)u->height, kind, stream));
  }

  ctx->last_hdr = reinterpret_cast<QueueHdr*>(dbase + L.o_hdr);
  ctx->last_stream = stream;
  ctx->stats = dtb_stats{};
  ctx->stats.tiles = total;
  ctx->stats.rounds = nrounds;
  ctx->timed = timed;
  ctx->async_pending = true;
  if ((flags & DTB_FLAG_ASYNC) && !host_io) return DTB_OK;
  return dtb_sync(ctx, stream);
}

void tuning_to_abi(dtb_context ctx, const LaunchTuning& lt, dtb_tuning* t) {
  t->ctas_per_sm = NS_VARIANT_TABLE[lt.variant].ctas;
  t->grid_percent = lt.grid_percent;
  t->host_chunk_kpx = (int32_t)(ctx->host_chunk_px / 1024ull);
  t->queue_buckets = lt.buckets;
  t->bucket_width_pct = (int32_t)lrintf(lt.bucket_tiles * 100.0f);
  t->staging = NS_VARIANT_TABLE[lt.variant].ahead ? 2 : 1;
  t->warps_per_cta = NS_VARIANT_TABLE[lt.variant].wpc;
}

dtb_status read_device_status(dtb_context ctx, const QueueHdr* hdr_dev, dtb_stats* st) {
  QueueHdr h;
  DTB_CUDA(ctx, cudaMemcpy(&h, hdr_dev, sizeof(QueueHdr), cudaMemcpyDeviceToHost));
  st->tile_visits = h.progress.v;
  st->phases = h.phases.v;
  st->activations = h.activations.v;
  st->device_error = h.error.v;
  st->device_error_info = h.err_info.v;
  switch (h.error.v) {
    case DERR_NONE: return DTB_OK;
    case DERR_QUEUE_TIMEOUT:
      return fail(ctx, DTB_ERR_TIMEOUT, "tile queue made no progress within the time limit (ticket %u)", h.err_info.v);
    case DERR_TMA_TIMEOUT: return fail(ctx, DTB_ERR_TIMEOUT, "TMA transfer of tile %u did not complete", h.err_info.v);
    case DERR_PHASE_LIMIT: return fail(ctx, DTB_ERR_DEVICE, "tile %u did not converge within %d phases", h.err_info.v, PHASE_LIMIT);
    case DERR_RING_FULL: return fail(ctx, DTB_ERR_DEVICE, "queue ring slot stayed occupied (tile %u)", h.err_info.v);
    case DERR_VISIT_LIMIT: return fail(ctx, DTB_ERR_DEVICE, "tile visit limit exceeded (%u)", h.err_info.v);
    case DERR_BAD_TILE: return fail(ctx, DTB_ERR_DEVICE, "internal error: activation of tile %u outside the call", h.err_info.v);
    default: return fail(ctx, DTB_ERR_DEVICE, "device error %u", h.error.v);
  }
}

}  // namespace dtb

// ======================================================================================================
// C ABI
// ======================================================================================================
extern "C" {

DTB_API int32_t dtb_abi_version(void) { return DTB_ABI_VERSION; }

DTB_API const char* dtb_status_string(dtb_status s) {
  switch (s) {
    case DTB_OK: return "ok";
    case DTB_ERR_INVALID_ARG: return "invalid argument";
    case DTB_ERR_CUDA: return "CUDA error";
    case DTB_ERR_OUT_OF_MEMORY: return "out of device memory";
    case DTB_ERR_TIMEOUT: return "device wait timed out";
    case DTB_ERR_DEVICE: return "device-side error";
    case DTB_ERR_NO_DEVICE: return "no usable device";
    case DTB_ERR_CAPACITY: return "capacity exceeded";
    case DTB_ERR_IO: return "image file could not be read or written";
  }
  return "unknown status";
}

DTB_API dtb_status dtb_context_create(int32_t device, dtb_context* out) {
  if (!out) return DTB_ERR_INVALID_ARG;
  *out = nullptr;
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return DTB_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return DTB_ERR_NO_DEVICE;
  if (prop.major < 10) return DTB_ERR_NO_DEVICE;
  if (cudaSetDevice(dev) != cudaSuccess) return DTB_ERR_NO_DEVICE;
  dtb_context ctx = new (std::nothrow) dtb_context_s();
  if (!ctx) return DTB_ERR_OUT_OF_MEMORY;
  ctx->device = dev;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->gpu_name = prop.name;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    delete ctx;
    return DTB_ERR_NO_DEVICE;
  }
  ctx->encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  if (cudaEventCreate(&ctx->ev[0]) != cudaSuccess || cudaEventCreate(&ctx->ev[1]) != cudaSuccess) {
    delete ctx;
    return DTB_ERR_NO_DEVICE;
  }
  static_assert(NS_VARIANT_TABLE[0].ctas == 2 && !NS_VARIANT_TABLE[0].ahead && NS_VARIANT_TABLE[1].ctas == 3 &&
                    NS_VARIANT_TABLE[2].ctas == 4 && NS_VARIANT_TABLE[3].ctas == 2 && NS_VARIANT_TABLE[3].ahead &&
                    NS_VARIANT_TABLE[4].ctas == 3 && NS_VARIANT_TABLE[4].ahead && NS_VARIANT_TABLE[0].wpc == 4 &&
                    NS_VARIANT_TABLE[1].wpc == 4 && NS_VARIANT_TABLE[2].wpc == 4 && NS_VARIANT_TABLE[3].wpc == 4 &&
                    NS_VARIANT_TABLE[4].wpc == 4 && NS_VARIANT_TABLE[5].ctas == 6 && NS_VARIANT_TABLE[5].wpc == 2 &&
                    NS_VARIANT_TABLE[6].ctas == 2 && NS_VARIANT_TABLE[6].wpc == 6 && NS_VARIANT_TABLE[7].ctas == 2 &&
                    NS_VARIANT_TABLE[7].wpc == 8 && !NS_VARIANT_TABLE[5].ahead && !NS_VARIANT_TABLE[6].ahead &&
                    !NS_VARIANT_TABLE[7].ahead,
                "kernel instantiations below follow NS_VARIANT_TABLE");
  ctx->ns_fn[0] = (const void*)ggdt_persistent<MODE_NS, PERSIST_WPC, 2>;
  ctx->ns_fn[1] = (const void*)ggdt_persistent<MODE_NS, PERSIST_WPC, 3>;
  ctx->ns_fn[2] = (const void*)ggdt_persistent<MODE_NS, PERSIST_WPC, 4>;
  ctx->ns_fn[3] = (const void*)ggdt_persistent_ahead<PERSIST_WPC, 2>;
  ctx->ns_fn[4] = (const void*)ggdt_persistent_ahead<PERSIST_WPC, 3>;
  ctx->ns_fn[5] = (const void*)ggdt_persistent<MODE_NS, 2, 6>;
  ctx->ns_fn[6] = (const void*)ggdt_persistent<MODE_NS, 6, 2>;
  ctx->ns_fn[7] = (const void*)ggdt_persistent<MODE_NS, 8, 2>;
  const void* kref = (const void*)ggdt_persistent<MODE_REF, PERSIST_WPC, REF_CTAS>;
  const void* kref_nofma = (const void*)ggdt_persistent<MODE_REF_NOFMA, PERSIST_WPC, REF_CTAS>;
  bool ok = true;
  for (int k = 0; k < NS_VARIANTS && ok; ++k) {
    const int wpc = NS_VARIANT_TABLE[k].wpc;
    ctx->ns_smem[k] = wpc * (NS_VARIANT_TABLE[k].ahead ? sizeof(WarpSmemP) : sizeof(WarpSmem)) + 128;
    ok = cudaFuncSetAttribute(ctx->ns_fn[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->ns_smem[k]) ==
             cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->ns_blocks_per_sm[k], ctx->ns_fn[k], wpc * 32,
                                                       ctx->ns_smem[k]) == cudaSuccess &&
         ctx->ns_blocks_per_sm[k] >= 1;
  }
  int ref_bps_nofma = 0;
  ok = ok && cudaFuncSetAttribute(kref, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PERSIST_SMEM) == cudaSuccess &&
       cudaFuncSetAttribute(kref_nofma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PERSIST_SMEM) == cudaSuccess &&
       cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->ref_blocks_per_sm, kref, PERSIST_WPC * 32, PERSIST_SMEM) ==
           cudaSuccess &&
       cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ref_bps_nofma, kref_nofma, PERSIST_WPC * 32, PERSIST_SMEM) ==
           cudaSuccess;
  ctx->ref_blocks_per_sm = std::min(ctx->ref_blocks_per_sm, ref_bps_nofma);  // one grid size for both roundings
  ok = ok && ctx->ref_blocks_per_sm >= 1;
  ok = ok &&
       cudaFuncSetAttribute((const void*)ggdt_round<MODE_NS, ROUND_WPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)ROUND_SMEM) == cudaSuccess &&
       cudaFuncSetAttribute((const void*)ggdt_round<MODE_REF, ROUND_WPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)ROUND_SMEM) == cudaSuccess &&
       cudaFuncSetAttribute((const void*)ggdt_round<MODE_REF_NOFMA, ROUND_WPC>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROUND_SMEM) == cudaSuccess;
  if (!ok) {
    delete ctx;
    return DTB_ERR_NO_DEVICE;
  }
  if (const char* e = getenv("DTB_NS_VARIANT")) {  // index into NS_VARIANT_TABLE
    const int k = atoi(e);
    if (k >= 0 && k < NS_VARIANTS) ctx->tuning.variant = k;
  }
  if (const char* e = getenv("DTB_AUTOTUNE_CACHE")) {  // autotuner cache of earlier processes
    ctx->tune_cache_path = e;
    load_tuning_cache(ctx);
  }
  *out = ctx;
  return DTB_OK;
}

DTB_API void dtb_context_destroy(dtb_context ctx) {
  if (!ctx) return;
  if (ctx->async_pending) cudaStreamSynchronize(ctx->last_stream);
  if (ctx->pipe_pending) cudaEventSynchronize(ctx->ev_pipe_done);
  if (ctx->dpipe) cudaFree(ctx->dpipe);
  if (ctx->ev_pipe_done) cudaEventDestroy(ctx->ev_pipe_done);
  if (ctx->ev_pipe_start) cudaEventDestroy(ctx->ev_pipe_start);
  for (int i = 0; i < 2; ++i) {
    if (ctx->pstage[i]) cudaFree(ctx->pstage[i]);
    if (ctx->pscratch[i]) cudaFree(ctx->pscratch[i]);
    if (ctx->ev_pset_free[i]) cudaEventDestroy(ctx->ev_pset_free[i]);
  }
  if (ctx->dscratch) cudaFree(ctx->dscratch);
  if (ctx->dround_counts) cudaFree(ctx->dround_counts);
  for (int i = 0; i < 2; ++i) {
    if (ctx->hpin[i]) cudaFreeHost(ctx->hpin[i]);
    if (ctx->hpin_ev[i]) cudaEventDestroy(ctx->hpin_ev[i]);
  }
  if (ctx->dstage) cudaFree(ctx->dstage);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : ctx->evpool)
    if (e) cudaEventDestroy(e);
  if (ctx->s_in) cudaStreamDestroy(ctx->s_in);
  if (ctx->s_out) cudaStreamDestroy(ctx->s_out);
  if (ctx->s_lane) cudaStreamDestroy(ctx->s_lane);
  if (ctx->s_lane0) cudaStreamDestroy(ctx->s_lane0);
  delete ctx;
}

DTB_API const char* dtb_context_message(dtb_context ctx) { return ctx ? ctx->msg.c_str() : ""; }

DTB_API dtb_status dtb_last_stats(dtb_context ctx, dtb_stats* out) {
  if (!ctx || !out) return DTB_ERR_INVALID_ARG;
  *out = ctx->stats;
  return DTB_OK;
}

DTB_API dtb_status dtb_context_set_tuning(dtb_context ctx, const dtb_tuning* t) {
  if (!ctx || !t) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  LaunchTuning nt = ctx->tuning;
  const NsVariant cur = NS_VARIANT_TABLE[nt.variant];
  const int ctas = t->ctas_per_sm != 0 ? t->ctas_per_sm : cur.ctas;
  const bool ahead = t->staging != 0 ? t->staging == 2 : cur.ahead;
  // Warps per CTA: as given, else the current shape's if it goes with ctas_per_sm, else 4.
  const int wpc = t->warps_per_cta != 0 ? t->warps_per_cta
                  : ns_variant_of(ctas, ahead, cur.wpc) >= 0 ? cur.wpc
                                                             : PERSIST_WPC;
  if (t->staging < 0 || t->staging > 2) return fail(ctx, DTB_ERR_INVALID_ARG, "staging must be 1 or 2");
  const int variant = ns_variant_of(ctas, ahead, wpc);
  if (variant < 0)
    return fail(ctx, DTB_ERR_INVALID_ARG,
                "(ctas_per_sm, warps_per_cta) must be (2|3|4, 4), (6, 2), (2, 6) or (2, 8); staging 2 needs (2|3, 4)");
  const int pct = t->grid_percent == 0 ? 100 : t->grid_percent;
  if (pct < 1 || pct > 100) return fail(ctx, DTB_ERR_INVALID_ARG, "grid_percent must be in [1, 100]");
  if (t->host_chunk_kpx < 0) return fail(ctx, DTB_ERR_INVALID_ARG, "host_chunk_kpx must be >= 0");
  const int buckets = t->queue_buckets != 0 ? t->queue_buckets : nt.buckets;
  const float width = t->bucket_width_pct != 0 ? (float)t->bucket_width_pct / 100.0f : nt.bucket_tiles;
  if (t->bucket_width_pct < 0 || !valid_policy(buckets, width))
    return fail(ctx, DTB_ERR_INVALID_ARG, "queue_buckets must be 1, 2, 4, 8 or 16 and bucket_width_pct in 1..6400");
  nt.variant = variant;
  nt.grid_percent = pct;
  nt.buckets = buckets;
  nt.bucket_tiles = width;
  ctx->tuning = nt;
  if (t->host_chunk_kpx > 0) ctx->host_chunk_px = (uint64_t)t->host_chunk_kpx * 1024ull;
  ctx->tuned.clear();
  return DTB_OK;
}

DTB_API dtb_status dtb_context_get_tuning(dtb_context ctx, dtb_tuning* t) {
  if (!ctx || !t) return DTB_ERR_INVALID_ARG;
  tuning_to_abi(ctx, ctx->tuning, t);
  return DTB_OK;
}

DTB_API dtb_status dtb_sync(dtb_context ctx, void* stream) {
  if (!ctx) return DTB_ERR_INVALID_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  DTB_CUDA(ctx, cudaStreamSynchronize(st));
  if (ctx->pipe_pending) {
    DTB_CUDA(ctx, cudaEventSynchronize(ctx->ev_pipe_done));  // the last call's end (copies out run in call order)
    return finish_pipeline(ctx);
  }
  if (!ctx->async_pending) return DTB_OK;
  ctx->async_pending = false;
  const dtb_status s = read_device_status(ctx, ctx->last_hdr, &ctx->stats);
  if (ctx->timed) {
    float ms = 0.0f;
    DTB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    ctx->stats.kernel_ms = ms;
    ctx->timed = false;
  }
  return s;
}

static bool valid_v(float v) { return v >= 0.0f; }  // also rejects NaN

DTB_API dtb_status dtb_gdt_ref(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist,
                               float lambda, float v, uint32_t flags, void* stream) {
  if (!ctx) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->msg.clear();
  dtb_status s = check_triplet(ctx, img, mask, dist, false);
  if (s != DTB_OK) return s;
  if (!(lambda >= 0.0f && lambda <= 1.0f)) return fail(ctx, DTB_ERR_INVALID_ARG, "lambda must be in [0, 1]");
  if (!valid_v(v)) return fail(ctx, DTB_ERR_INVALID_ARG, "v must be >= 0");
  DTB_CUDA(ctx, cudaSetDevice(ctx->device));
  Job j = Job::from(img, mask, dist);
  j.mode = MODE_REF;
  j.v = v;
  j.l_grad = lambda;
  j.l_eucl = 1.0f - lambda;  // reference generalised_distance_transform.cu:108-109
  j.ref_fma = (flags & DTB_FLAG_REF_NO_FMA) ? 0 : 1;
  const dtb_image* a[1] = {img};
  const dtb_image* b[1] = {mask};
  const dtb_image* c[1] = {dist};
  return run_jobs(ctx, {j}, a, b, c, flags, reinterpret_cast<cudaStream_t>(stream));
}

DTB_API dtb_status dtb_gdt_ref_blocks(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist,
                                      float lambda, float v, int32_t* rounds_per_tile, uint32_t flags, void* stream) {
  if (!ctx) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->msg.clear();
  dtb_status s = check_triplet(ctx, img, mask, dist, false);
  if (s != DTB_OK) return s;
  if (!(lambda >= 0.0f && lambda <= 1.0f)) return fail(ctx, DTB_ERR_INVALID_ARG, "lambda must be in [0, 1]");
  if (!valid_v(v)) return fail(ctx, DTB_ERR_INVALID_ARG, "v must be >= 0");
  DTB_CUDA(ctx, cudaSetDevice(ctx->device));
  Job j = Job::from(img, mask, dist);
  j.mode = MODE_REF;
  j.v = v;
  j.l_grad = lambda;
  j.l_eucl = 1.0f - lambda;
  j.ref_fma = (flags & DTB_FLAG_REF_NO_FMA) ? 0 : 1;
  const dtb_image* a[1] = {img};
  const dtb_image* b[1] = {mask};
  const dtb_image* c[1] = {dist};
  const uint32_t total = (uint32_t)j.tiles_x() * (uint32_t)j.tiles_y();
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const bool counting = rounds_per_tile != nullptr && total > 0;
  if (counting) {
    if ((s = grow(ctx, reinterpret_cast<void**>(&ctx->dround_counts), &ctx->dround_counts_size, total * sizeof(int32_t))) != DTB_OK)
      return s;
    DTB_CUDA(ctx, cudaMemsetAsync(ctx->dround_counts, 0, total * sizeof(int32_t), st));
  }
  ctx->count_rounds = counting;
  s = run_jobs(ctx, {j}, a, b, c, (flags | DTB_FLAG_ROUNDS) & ~DTB_FLAG_ASYNC, st);
  ctx->count_rounds = false;
  if (s != DTB_OK || !counting) return s;
  // Add this call's counters into the caller's (host or device memory).
  cudaPointerAttributes pa{};
  const bool on_device = cudaPointerGetAttributes(&pa, rounds_per_tile) == cudaSuccess &&
                         (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
  cudaGetLastError();  // cudaPointerGetAttributes on plain host memory may leave an error behind on older drivers
  if (on_device) {
    ggdt_add_counts<<<std::min<uint32_t>((total + 255) / 256, (uint32_t)ctx->num_sms * 8), 256, 0, st>>>(
        rounds_per_tile, ctx->dround_counts, total);
    DTB_CUDA(ctx, cudaGetLastError());
    DTB_CUDA(ctx, cudaStreamSynchronize(st));
  } else {
    std::vector<int32_t> h(total);
    DTB_CUDA(ctx, cudaMemcpyAsync(h.data(), ctx->dround_counts, total * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DTB_CUDA(ctx, cudaStreamSynchronize(st));
    for (uint32_t t = 0; t < total; ++t) rounds_per_tile[t] += h[t];
  }
  return DTB_OK;
}

DTB_API dtb_status dtb_gdt(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist, float gamma,
                           float v, uint32_t flags, void* stream) {
  if (!ctx) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->msg.clear();
  dtb_status s = check_triplet(ctx, img, mask, dist, true);
  if (s != DTB_OK) return s;
  if (!(gamma >= 0.0f) || std::isinf(gamma)) return fail(ctx, DTB_ERR_INVALID_ARG, "gamma must be finite and >= 0");
  if (!valid_v(v)) return fail(ctx, DTB_ERR_INVALID_ARG, "v must be >= 0");
  DTB_CUDA(ctx, cudaSetDevice(ctx->device));
  Job j = Job::from(img, mask, dist);
  j.mode = MODE_NS;
  j.v = v;
  j.g2 = gamma_to_g2(gamma);
  const dtb_image* a[1] = {img};
  const dtb_image* b[1] = {mask};
  const dtb_image* c[1] = {dist};
  return run_jobs(ctx, {j}, a, b, c, flags, reinterpret_cast<cudaStream_t>(stream));
}

DTB_API dtb_status dtb_gdt_batch(dtb_context ctx, int32_t n, const dtb_image* imgs, const dtb_image* masks,
                                 const dtb_image* dists, const float* gammas, float v, uint32_t flags, void* stream) {
  if (!ctx) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->msg.clear();
  if (n < 0 || (n > 0 && (!imgs || !masks || !dists || !gammas))) return fail(ctx, DTB_ERR_INVALID_ARG, "bad batch arrays");
  if (!valid_v(v)) return fail(ctx, DTB_ERR_INVALID_ARG, "v must be >= 0");
  std::vector<Job> jobs;
  std::vector<const dtb_image*> a(n), b(n), c(n);
  jobs.reserve(n);
  for (int i = 0; i < n; ++i) {
    dtb_status s = check_triplet(ctx, &imgs[i], &masks[i], &dists[i], true);
    if (s != DTB_OK) return fail(ctx, s, "image %d: %s", i, ctx->msg.c_str());
    if (!(gammas[i] >= 0.0f) || std::isinf(gammas[i])) return fail(ctx, DTB_ERR_INVALID_ARG, "image %d: bad gamma", i);
    Job j = Job::from(&imgs[i], &masks[i], &dists[i]);
    j.mode = MODE_NS;
    j.v = v;
    j.g2 = gamma_to_g2(gammas[i]);
    jobs.push_back(j);
    a[i] = &imgs[i];
    b[i] = &masks[i];
    c[i] = &dists[i];
  }
  DTB_CUDA(ctx, cudaSetDevice(ctx->device));
  if (flags & DTB_FLAG_ROUNDS) {
    // Plain per-image path: one image after the other.
    dtb_stats acc{};
    for (int i = 0; i < n; ++i) {
      dtb_status s = run_jobs(ctx, {jobs[i]}, &a[i], &b[i], &c[i], flags & ~DTB_FLAG_ASYNC, reinterpret_cast<cudaStream_t>(stream));
      if (s != DTB_OK) return s;
      acc.tiles += ctx->stats.tiles;
      acc.tile_visits += ctx->stats.tile_visits;
      acc.phases += ctx->stats.phases;
      acc.activations += ctx->stats.activations;
      acc.rounds += ctx->stats.rounds;
    }
    ctx->stats = acc;
    return DTB_OK;
  }
  return run_jobs(ctx, jobs, a.data(), b.data(), c.data(), flags, reinterpret_cast<cudaStream_t>(stream));
}

static dtb_status copy2d(const dtb_image* src, const dtb_image* dst, cudaMemcpyKind kind, void* stream) {
  if (!src || !dst) return DTB_ERR_INVALID_ARG;
  if (src->width != dst->width || src->height != dst->height || src->elem_size != dst->elem_size) return DTB_ERR_INVALID_ARG;
  if (src->width == 0 || src->height == 0) return DTB_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpy2DAsync(dst->buffer, (size_t)dst->pitch, src->buffer, (size_t)src->pitch,
                                    (size_t)src->width * src->elem_size, (size_t)src->height, kind, st);
  if (e == cudaSuccess && !stream) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? DTB_OK : DTB_ERR_CUDA;
}

DTB_API dtb_status dtb_debug_inject_queue_stall(dtb_context ctx, uint32_t timeout_ms) {
  if (!ctx || timeout_ms == 0 || timeout_ms > 60000) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->inject_stall_ns = (uint64_t)timeout_ms * 1000000ull;
  return DTB_OK;
}

DTB_API dtb_status dtb_image_alloc(int32_t width, int32_t height, int32_t elem_size, int32_t memory_kind, dtb_image* out) {
  if (!out || width < 0 || height < 0 || elem_size <= 0 || (memory_kind != DTB_CPU && memory_kind != DTB_GPU))
    return DTB_ERR_INVALID_ARG;
  const size_t row = (size_t)width * (size_t)elem_size;
  const size_t pitch = memory_kind == DTB_GPU ? align_up(std::max<size_t>(row, 1), 128) : row;
  if (pitch > (size_t)INT32_MAX) return DTB_ERR_INVALID_ARG;
  const size_t bytes = pitch * (size_t)height;
  void* p = nullptr;
  if (bytes > 0) {
    if (memory_kind == DTB_GPU) {
      const cudaError_t e = cudaMalloc(&p, bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        if (e == cudaErrorMemoryAllocation) return DTB_ERR_OUT_OF_MEMORY;
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return DTB_ERR_NO_DEVICE;
        return DTB_ERR_CUDA;
      }
    } else {
      p = std::aligned_alloc(64, align_up(bytes, 64));
      if (!p) return DTB_ERR_OUT_OF_MEMORY;
    }
  }
  *out = dtb_image{p, width, height, (int32_t)pitch, elem_size, memory_kind};
  return DTB_OK;
}

DTB_API dtb_status dtb_image_free(dtb_image* img) {
  if (!img) return DTB_ERR_INVALID_ARG;
  if (img->buffer) {
    if (img->memory_kind == DTB_GPU) {
      if (cudaFree(img->buffer) != cudaSuccess) return DTB_ERR_CUDA;
    } else {
      std::free(img->buffer);
    }
  }
  img->buffer = nullptr;
  return DTB_OK;
}

DTB_API dtb_status dtb_host_to_device(const dtb_image* src, const dtb_image* dst, void* stream) {
  if (!src || !dst || src->memory_kind != DTB_CPU || dst->memory_kind != DTB_GPU) return DTB_ERR_INVALID_ARG;
  return copy2d(src, dst, cudaMemcpyHostToDevice, stream);
}

DTB_API dtb_status dtb_device_to_host(const dtb_image* src, const dtb_image* dst, void* stream) {
  if (!src || !dst || src->memory_kind != DTB_GPU || dst->memory_kind != DTB_CPU) return DTB_ERR_INVALID_ARG;
  return copy2d(src, dst, cudaMemcpyDeviceToHost, stream);
}

}  // extern "C"
