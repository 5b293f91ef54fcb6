// dtb_device.cuh -- device-side building blocks of the B200 GGDT: tile states, the persistent tile queue,
// TMA staging, edge weights, exact single-edge sweeps and the warp-per-tile visit.
//
// The computed map is the greatest fixpoint of single-edge relaxations D(p) <- min(D(p), relax(D(q), q->p))
// from D = mask ? 0 : v (reference dt/src/utils.cu:12).  relax() is monotone in D(q), so any schedule that
// runs to quiescence reaches the same fixpoint bit for bit; this is what lets a warp-per-tile schedule with
// a device queue reproduce the reference's raster rounds (dt/src/generalised_distance_transform.cu:126-134)
// exactly.  Every relaxation below is a single edge with the exact per-edge arithmetic; no step ever
// combines two edge weights before adding them to a distance.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace dtb {

constexpr int TILE = 32;                  // tile side (pixels); one warp owns one tile
constexpr int IMG_BOX_ROWS = TILE + 2;    // image box rows: 1-pixel halo above and below
constexpr int IMG_BOX_GRAY = 64;          // gray box width (bytes): x0-16 .. x0+47 covers x0-1 .. x0+32
constexpr int IMG_BOX_RGB = 128;          // rgb8 box width (bytes): 3*x0-16 .. 3*x0+111 covers 3*(x0-1) .. 3*(x0+33)
// Gray visits keep a 256-entry weight table (1 KB) in the image box past the 34 x 64-byte gray rows.
constexpr int GRAY_LUT_OFFSET = 2304;
static_assert(GRAY_LUT_OFFSET >= IMG_BOX_ROWS * IMG_BOX_GRAY && GRAY_LUT_OFFSET + 1024 <= IMG_BOX_ROWS * IMG_BOX_RGB,
              "gray weight table must fit the unused part of the image box");
constexpr int S_STRIDE = TILE + 1;        // padded transpose buffer stride (floats): conflict-free both ways

// Tile state word: flags in the low byte, image index of the tile in the upper 24 bits.
constexpr uint32_t ST_PENDING = 1u;   // queued (or: re-run requested while running)
constexpr uint32_t ST_RUNNING = 2u;   // a warp is visiting the tile
constexpr uint32_t ST_VISITED = 4u;   // the tile's distances in global memory are valid
constexpr uint32_t ST_SEED = 8u;      // the next visit applies the seed mask of the tile
constexpr int ST_IMG_SHIFT = 8;

// Weight modes.
constexpr int32_t MODE_NS = 0;   // C4, w = sqrt(1 + g2 * dI2), gray or rgb8
constexpr int32_t MODE_REF = 1;  // C8, D(q) + l_eucl * {1, sqrt2} + l_grad * |dI|, gray (reference weight)
// Kernel selection only (descriptors keep MODE_REF with ref_fma = 0): ref-mode with left-to-right rounding.  Each
// rounding has its own tile kernels, so a kernel holds one copy of the ref-mode phase loop.
constexpr int32_t MODE_REF_NOFMA = 2;

// Device error codes (written once into Queue::error).
constexpr uint32_t DERR_NONE = 0;
constexpr uint32_t DERR_QUEUE_TIMEOUT = 1;   // no global progress for the configured time
constexpr uint32_t DERR_TMA_TIMEOUT = 2;     // a TMA transaction did not complete in time
constexpr uint32_t DERR_PHASE_LIMIT = 3;     // a tile did not converge within the phase limit
constexpr uint32_t DERR_RING_FULL = 4;       // a ring slot stayed occupied
constexpr uint32_t DERR_VISIT_LIMIT = 5;     // more tile visits than the call's cap (a safety net)
constexpr uint32_t DERR_BAD_TILE = 6;        // an activation named a tile outside the call (internal bug)

// One image of a (possibly ragged) batch.  Pitches are in bytes.
struct alignas(64) ImgDesc {
  const uint8_t* img;
  const uint8_t* mask;
  float* dist;
  int64_t img_pitch;
  int64_t mask_pitch;
  int64_t dist_pitch;
  int32_t width, height, channels, tiles_x, tiles_y;
  uint32_t tile_base;
  float g2;       // ns-mode: fl32(gamma * gamma)
  float v;        // value of unreached pixels (>= 0)
  float l_eucl;   // ref-mode: 1 - lambda
  float l_grad;   // ref-mode: lambda
  int32_t mode;
  int32_t ref_fma;  // ref-mode: 1 = fma(l_grad, dI, fma(l_eucl, d, D)), 0 = left-to-right rounding
};

// Counters live on separate 128-byte lines.
constexpr uint32_t NBUCKET_MAX = 16;  // priority buckets of the tile queue at most (the count is a power of two)
struct alignas(128) Line { uint32_t v; uint32_t pad[31]; };
struct QueueHdr {
  Line heads[NBUCKET_MAX];  // next pop ticket, per bucket
  Line tails[NBUCKET_MAX];  // next push position, per bucket
  Line base;       // absolute index of the lowest bucket that may hold work (a hint: order is a heuristic)
  Line pending;    // tiles queued or running
  Line error;      // first device error code
  Line progress;   // completed visits (flushed per warp in batches; watchdog and visit cap)
  Line phases;     // total sweep phases
  Line activations;  // neighbour activations issued
  Line err_info;   // tile id / detail of the first error
  Line done;       // set once when pending reached 0
};

// The tile queue.  nb_mask = 0: one FIFO ring.  nb_mask = 2^k - 1 (k = 1..4): 2^k rings ordered by distance: an
// activation carries the smallest value it can bring into the tile (a border distance plus an edge weight);
// its bucket is that value in units of `bucket_tiles` tile-widths of path cost of its image, relative to
// `base`.  Workers
// take from the lowest non-empty bucket, which approximates visiting tiles in order of distance (Dijkstra
// order on the tile graph) and so avoids most re-visits of tiles reached first by a costlier path.  The map
// does not depend on the order: every order ends in the same fixpoint.
struct Queue {
  QueueHdr* hdr;
  uint32_t* ring;           // (nb_mask + 1) rings of (mask + 1) slots
  uint32_t mask;            // ring capacity - 1 (capacity is a power of two)
  uint64_t timeout_ns;      // watchdog: give up after this long without any completed visit
  uint32_t max_visits;      // safety net against endless re-activation
  uint32_t total_tiles;     // tile ids are < total_tiles
  uint32_t nb_mask = 0;     // bucket count - 1
  uint32_t* keys = nullptr;  // per tile: smallest pending activation value (float bits), KEY_NONE if none
  float* wacc = nullptr;     // per image: [sum, count] of the internal edge weights seen by first visits
  float bucket_tiles = 0.5f; // bucket width in tile-widths of path cost (32 x the image's mean edge weight)
};
constexpr uint32_t KEY_NONE = 0xFFFFFFFFu;

// Per-warp shared memory slot (14 KB: 12 warps per SM, the 168-register launch, fit in 228 KB).
// Weight and tile buffers keep 36 floats a row.  A lane-per-column access ([k * 36 + lane]) is conflict-free; a
// lane-per-row access ([lane * 36 + k]) is conflict-free as 16-byte vectors (the rows of a quarter-warp start in
// 8 different 16-byte bank groups), so the row-layout phase moves its weights and the tile in 128-bit accesses:
// 17 loads of weights instead of 65, 8 accesses instead of 32 on its side of each transpose (4 % faster than
// 33-float rows with scalar accesses on the 1024-image batch).
constexpr int W_STRIDE = TILE + 4;
constexpr int TILE_BUF_BYTES = TILE * W_STRIDE * 4;
constexpr int IMG_REGION = IMG_BOX_ROWS * IMG_BOX_RGB > TILE_BUF_BYTES ? IMG_BOX_ROWS * IMG_BOX_RGB : TILE_BUF_BYTES;
struct alignas(128) WarpSmem {
  uint8_t img[IMG_REGION];                   // TMA destination of the image box (gray uses IMG_BOX_ROWS x 64); once
                                             // the weights are computed, the tile buffer B[y * 36 + x]
  float Wh[TILE * W_STRIDE];                 // ns-mode: Wh[y * 36 + x] = weight of edge (x-1, x) on row y, x = 0..32
  float Wv[(TILE + 1) * W_STRIDE];           // ns-mode: Wv[y * 36 + x] = weight of edge (y-1, y) on column x, y = 0..32;
                                             // its first 1 KB receives the seed-mask TMA box before the weights
  uint64_t bar;                              // TMA mbarrier
  uint32_t keep;                             // tile this warp keeps for its next visit (POP_NONE: none)
};
__device__ __forceinline__ uint8_t* mask_box(WarpSmem& sm) { return reinterpret_cast<uint8_t*>(sm.Wv); }

// Per-warp shared memory of the staged-ahead tile kernel (17 KB: 12 warps per SM fit in 228 KB): the image
// boxes of the tile being visited and of the warp's next tile, each the tile buffer B of its own visit once its
// weights are computed; the weights; a barrier per box and one for the seed-mask box.
constexpr int IMG_BOX_BYTES = IMG_REGION;
struct alignas(128) WarpSmemP {
  uint8_t box[2][IMG_BOX_BYTES];
  float Wh[TILE * W_STRIDE];
  float Wv[(TILE + 1) * W_STRIDE];   // its first 1 KB receives the seed-mask TMA box before the weights
  uint64_t bar[2];                   // image box k
  uint64_t mbar;                     // seed-mask box
};
static_assert(TILE * W_STRIDE * 4 <= IMG_BOX_BYTES, "the tile buffer must fit an image box");

// ------------------------------------------------------------------------------------------------------
// PTX helpers
// ------------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// Acquire-release fence at GPU scope: the release (data before a flag or counter update) and acquire (a flag
// or counter read before the data) points of the tile visit and the queue.  Lighter than __threadfence()'s
// sequentially consistent fence, which only the end-of-queue handshake (a store then a load of another word,
// signal_done_warp) needs.
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 2-D tiled TMA load into this CTA's shared memory.  The innermost coordinate x must be a multiple of 16
// bytes / element size; every call site below passes x0 - 16, 3*x0 - 16 (gray/rgb8 boxes) or x0, with x0 a
// multiple of 32.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tmap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// ------------------------------------------------------------------------------------------------------
// Queue: one or 2^k ticket rings of tile ids (buckets ordered by distance) with one pending counter for
// termination.
//   push: pending grows first, then a position of the item's bucket is reserved, then the item goes into its
//         slot (the slot must be free: CAS from 0; a slot given back by a waiter is skipped).
//   pop:  a head ticket in the lowest bucket holding work (or in the base bucket when there is none), then the
//         popper waits on its own slot only (no shared hot line is polled) until an item or the termination
//         sentinel arrives; in the bucketed queue a waiter whose item is not reserved gives the ticket back
//         when another bucket holds work.  Termination: the visit whose completion brings pending to 0 sets
//         `done` and writes the sentinel into every slot that has a waiting popper.
// Items are interchangeable, so a popper that takes an item meant for another ticket of the same slot is
// harmless: every item is taken exactly once (atomicExch) and no slot is written twice (CAS from 0).  Each
// ring holds at least 2 * (tiles + workers) slots, more than items and waiting poppers together.
// All waits are bounded by a no-global-progress watchdog and end with an error code, never a hang.
// ------------------------------------------------------------------------------------------------------
constexpr uint32_t SLOT_SENTINEL = 0xFFFFFFFFu;  // never an item: items are tile id + 1 < 2^31
constexpr uint32_t POP_NONE = 0xFFFFFFFFu;
constexpr uint64_t POLL_CHECK_NS = 2000;         // checks of done / error / watchdog / other buckets while waiting

__device__ __forceinline__ void set_error(const Queue& q, uint32_t code, uint32_t info) {
  if (atomicCAS(&q.hdr->error.v, 0u, code) == 0u) atomicExch(&q.hdr->err_info.v, info);
}

__device__ __forceinline__ uint32_t* ring_slot(const Queue& q, uint32_t b, uint32_t p) {
  return &q.ring[(size_t)b * (q.mask + 1) + (p & q.mask)];
}

// A waiter that gave its ticket back marks its slot; the pusher that reaches the slot clears it and takes the
// next position instead.  Never an item (items are tile id + 1 < 2^31) nor the sentinel.
constexpr uint32_t SLOT_CANCELLED = 0xFFFFFFFEu;

// Writes item into bucket b at position p once the slot is free (bounded wait); a cancelled slot is cleared and
// the item goes to the next position of the bucket.
__device__ __forceinline__ void slot_write(const Queue& q, uint32_t b, uint32_t p, uint32_t item) {
  uint32_t ns = 32;
  const uint64_t t0 = globaltimer();
  for (;;) {
    uint32_t* slot = ring_slot(q, b, p);
    const uint32_t prev = atomicCAS(slot, 0u, item + 1u);
    if (prev == 0u) return;
    if (prev == SLOT_CANCELLED) {
      atomicCAS(slot, SLOT_CANCELLED, 0u);
      p = atomicAdd(&q.hdr->tails[b].v, 1u);
      continue;
    }
    if (globaltimer() - t0 > q.timeout_ns) { set_error(q, DERR_RING_FULL, item); return; }
    __nanosleep(ns);
    ns = ns < 1024 ? ns * 2 : ns;
  }
}

// Bucket of an activation value `key` (distance units) for an image whose bucket width is 1 / inv_width.
// (Idle workers waiting in another bucket give their tickets back within POLL_CHECK_NS and find the item.)
__device__ __forceinline__ uint32_t bucket_of(const Queue& q, float key, float inv_width) {
  if (q.nb_mask == 0) return 0;
  const uint32_t base = ld_volatile(&q.hdr->base.v);
  const float r = key * inv_width;  // absolute bucket; NaN / huge values land in the last bucket
  uint32_t rel = q.nb_mask;
  if (r < 4.0e9f) {
    const uint32_t kb = (uint32_t)r;
    rel = kb <= base ? 0u : min(kb - base, q.nb_mask);
  }
  return (base + rel) & q.nb_mask;
}

// Bucket of an activation value relative to a base the caller read (bucket_of with the base given).
__device__ __forceinline__ uint32_t bucket_at(const Queue& q, float key, float inv_width, uint32_t base) {
  if (q.nb_mask == 0) return 0;
  const float r = key * inv_width;
  uint32_t rel = q.nb_mask;
  if (r < 4.0e9f) {
    const uint32_t kb = (uint32_t)r;
    rel = kb <= base ? 0u : min(kb - base, q.nb_mask);
  }
  return (base + rel) & q.nb_mask;
}

// Pushes one item into bucket b: pending += 1 before the item becomes visible.
__device__ __forceinline__ void queue_push_to(const Queue& q, uint32_t b, uint32_t item) {
  atomicAdd(&q.hdr->pending.v, 1u);
  fence_acq_rel();
  slot_write(q, b, atomicAdd(&q.hdr->tails[b].v, 1u), item);
}

// Single-item push at the current base bucket (seed scans, warm starts).
__device__ __forceinline__ void queue_push(const Queue& q, uint32_t item) {
  queue_push_to(q, q.nb_mask ? (ld_volatile(&q.hdr->base.v) & q.nb_mask) : 0u, item);
}

// Called by the whole warp of the visit that brought pending to 0: wakes every popper waiting on a slot.
__device__ __forceinline__ void signal_done_warp(const Queue& q) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) atomicExch(&q.hdr->done.v, 1u);
  __threadfence();
  for (uint32_t b = 0; b <= q.nb_mask; ++b) {
    uint32_t h = 0, t = 0;
    if (lane == 0) {
      h = ld_volatile(&q.hdr->heads[b].v);
      t = ld_volatile(&q.hdr->tails[b].v);
    }
    h = __shfl_sync(~0u, h, 0);
    t = __shfl_sync(~0u, t, 0);
    for (uint32_t p = t + (uint32_t)lane; (int32_t)(h - p) > 0; p += 32u)
      *(volatile uint32_t*)ring_slot(q, b, p) = SLOT_SENTINEL;
  }
}

// Watchdog state of one popper, kept across the tickets it gives back.
struct PopWatch {
  uint64_t t_prog;
  uint32_t seen;
};

constexpr uint32_t POP_RESCAN = 0xFFFFFFFDu;  // the ticket was given back: look for work elsewhere

// Lowest bucket other than b with an item reserved and not taken (one lane, a few loads).
__device__ __forceinline__ bool other_bucket_has_work(const Queue& q, uint32_t b) {
  for (uint32_t i = 0; i <= q.nb_mask; ++i)
    if (i != b && (int32_t)(ld_volatile(&q.hdr->tails[i].v) - ld_volatile(&q.hdr->heads[i].v)) > 0) return true;
  return false;
}

// Waits for the item of ticket h of bucket b (one lane).  Bounded: done / error / pending / watchdog.  In the
// bucketed queue a waiter whose item is not reserved yet gives the ticket back (POP_RESCAN) when another bucket
// holds work, so idle workers never sit in a cold bucket while work waits elsewhere.
__device__ __forceinline__ uint32_t slot_take(const Queue& q, uint32_t b, uint32_t h, PopWatch& w) {
  uint32_t* slot = ring_slot(q, b, h);
  uint32_t ns = 32;
  uint64_t t_check = globaltimer();
  for (;;) {
    const uint32_t cur = ld_volatile(slot);
    if (cur != 0u && cur != SLOT_CANCELLED) {
      const uint32_t v = atomicExch(slot, 0u);
      if (v == SLOT_SENTINEL) return POP_NONE;
      if (v != 0u && v != SLOT_CANCELLED) return v - 1u;
    }
    __nanosleep(ns);
    ns = ns < 256 ? ns * 2 : ns;
    const uint64_t now = globaltimer();
    if (now - t_check > POLL_CHECK_NS) {
      t_check = now;
      if (ld_volatile(&q.hdr->done.v) | ld_volatile(&q.hdr->error.v)) return POP_NONE;
      if (ld_volatile(&q.hdr->pending.v) == 0u) return POP_NONE;
      const uint32_t prog = ld_volatile(&q.hdr->progress.v);
      if (prog > q.max_visits) { set_error(q, DERR_VISIT_LIMIT, prog); return POP_NONE; }
      if (prog != w.seen) { w.seen = prog; w.t_prog = now; }
      else if (now - w.t_prog > q.timeout_ns) { set_error(q, DERR_QUEUE_TIMEOUT, h); return POP_NONE; }
      if (q.nb_mask && (int32_t)(ld_volatile(&q.hdr->tails[b].v) - h) <= 0 && other_bucket_has_work(q, b)) {
        if (atomicCAS(slot, 0u, SLOT_CANCELLED) == 0u) return POP_RESCAN;
      }
    }
  }
}

// Pop, called by the whole warp; every lane gets the tile id or POP_NONE (queue drained, or error).
// FIFO: a ticket, then the popper waits on its own slot only (no shared hot line is polled).
// Bucketed: one load per bucket across the lanes finds the lowest bucket with work and the ticket is taken
// there; with no work anywhere the ticket is taken in the base bucket, whose pushes feed waiting poppers
// first.  Either way the popper then waits on its own slot.
__device__ __forceinline__ uint32_t queue_pop(const Queue& q) {
  const int lane = threadIdx.x & 31;
  PopWatch w{globaltimer(), 0u};
  if (lane == 0) w.seen = ld_volatile(&q.hdr->progress.v);
  for (;;) {
    uint32_t base = 0, m = 0;
    if (q.nb_mask) {
      if (lane == 0) base = ld_volatile(&q.hdr->base.v);
      base = __shfl_sync(~0u, base, 0);
      const uint32_t bl = (base + (uint32_t)lane) & q.nb_mask;
      bool avail = false;
      if ((uint32_t)lane <= q.nb_mask)
        avail = (int32_t)(ld_volatile(&q.hdr->tails[bl].v) - ld_volatile(&q.hdr->heads[bl].v)) > 0;
      m = __ballot_sync(~0u, avail);
    }
    uint32_t res = POP_NONE;
    if (lane == 0) {
      uint32_t b = base & q.nb_mask;
      if (m) {
        const uint32_t f = (uint32_t)(__ffs(m) - 1);
        if (f > 0) atomicCAS(&q.hdr->base.v, base, base + f);  // the lower buckets are empty: move the hint up
        b = (base + f) & q.nb_mask;
      }
      const uint32_t h = atomicAdd(&q.hdr->heads[b].v, 1u);
      // No fence and no checks between the ticket and the slot: with work queued the item is usually in the
      // slot already, and the end of the queue (done, an error, nothing pending) is noticed by slot_take's
      // periodic checks within POLL_CHECK_NS even when the ticket came after signal_done_warp read the heads.
      res = slot_take(q, b, h, w);
    }
    res = __shfl_sync(~0u, res, 0);
    if (res != POP_RESCAN) return res;
  }
}

// Non-blocking pop (whole warp) for staging a warp's next tile ahead: takes a ticket only in the lowest bucket
// whose next item a pusher has already reserved (tail ahead of head, by CAS on the head, so no popper waits
// there), so the wait for the slot write that follows is short and never for work that does not exist.
// Returns the tile id, or POP_NONE when no reserved item was found (the caller then pops blocking later).
__device__ __forceinline__ uint32_t queue_try_pop(const Queue& q) {
  const int lane = threadIdx.x & 31;
  uint32_t base = 0;
  if (q.nb_mask) {
    if (lane == 0) base = ld_volatile(&q.hdr->base.v);
    base = __shfl_sync(~0u, base, 0);
  }
  const uint32_t bl = (base + (uint32_t)lane) & q.nb_mask;
  uint32_t h = 0;
  bool avail = false;
  if ((uint32_t)lane <= q.nb_mask) {
    h = ld_volatile(&q.hdr->heads[bl].v);
    avail = (int32_t)(ld_volatile(&q.hdr->tails[bl].v) - h) > 0;
  }
  const uint32_t m = __ballot_sync(~0u, avail);
  if (!m) return POP_NONE;
  const int f = __ffs(m) - 1;
  const uint32_t hf = __shfl_sync(~0u, h, f);
  uint32_t res = POP_NONE;
  if (lane == 0) {
    const uint32_t b = (base + (uint32_t)f) & q.nb_mask;
    if (atomicCAS(&q.hdr->heads[b].v, hf, hf + 1u) == hf) {
      PopWatch w{globaltimer(), ld_volatile(&q.hdr->progress.v)};
      res = slot_take(q, b, hf, w);  // tail > hf: the item is on its way, slot_take never gives the ticket back
      if (res == POP_RESCAN) res = POP_NONE;
    }
  }
  return __shfl_sync(~0u, res, 0);
}

// ------------------------------------------------------------------------------------------------------
// Edge weights
// ------------------------------------------------------------------------------------------------------
// ns-mode: w = sqrt(1 + g2 * dI2), dI2 = sum_c (I_c(p) - I_c(q))^2.  Pixels are packed little-endian in a
// u32 (gray: byte 0; rgb8: bytes 0..2), unused bytes zero.  dI2 <= 3 * 255^2 is exact in fp32; each of the
// three float operations is rounded separately (no contraction), the square root correctly rounded.
__device__ __forceinline__ float ns_weight_sq(uint32_t dI2, float g2) {
  return __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(g2, __uint2float_rn(dI2))));
}
__device__ __forceinline__ float ns_weight(uint32_t pa, uint32_t pb, float g2) {
  const uint32_t ad = __vabsdiffu4(pa, pb);
  return ns_weight_sq(__dp4a(ad, ad, 0u), g2);
}

// ref-mode relaxation of one edge, reference dt/src/dt_block_passes.cuh:45-46:
//   D(q) + l_eucl * local_dist2d[k] + l_grad * |I(p) - I(q)|
template <bool FMA>
__device__ __forceinline__ float ref_relax(float dq, float eucl_d, float l_eucl, float l_grad, float absdi) {
  if (FMA) return __fmaf_rn(l_grad, absdi, __fmaf_rn(l_eucl, eucl_d, dq));
  return __fadd_rn(__fadd_rn(dq, __fmul_rn(l_eucl, eucl_d)), __fmul_rn(l_grad, absdi));
}

// ------------------------------------------------------------------------------------------------------
// One phase of the warp's tile in either layout.  Lane l holds a line of 32 pixels d[0..31] (a row in the
// row layout, a column in the column layout); lanes l-1 / l+1 hold the neighbouring lines.
//   chain edges  wc[k]: between positions k-1 and k of the own line (wc[0]: lo -> d[0], wc[32]: d[31] -> hi,
//                where lo / hi are the halo pixels before and after the line);
//   cross edges  wx[k]: between position k of line l-1 and position k of line l.
// A forward chain walks k = 0..31 and a backward chain k = 31..0, interleaved (two independent dependency
// chains).  At each step the chain pixel is first relaxed along the line (from its predecessor on the
// chain), then across the lines from both neighbouring lanes, whose values at the same position are
// exchanged by warp shuffles.  Every step is a set of single-edge relaxations fl(D + w): no two edge weights
// are ever added before meeting a distance, so the result is the exact fixpoint whatever the order.  A chain
// therefore follows any staircase path that moves at most one line per position, in both cross directions,
// so one phase covers every monotone path of slope <= 1 along its axis.  Every internal edge of the tile is
// relaxed in both directions during a phase: a phase that changes nothing proves the tile internally
// converged.  The halo lines of the cross direction are not read here (lane 0 / 31 shuffle with themselves,
// which never lowers a value); they are the chain halo of the other layout's phase.
// ------------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool sweep_phase(float (&d)[TILE], const float (&wc)[TILE + 1], const float (&wx)[TILE], float lo,
                                            float hi) {
  bool ch = false;
  float f = lo, b = hi;
#pragma unroll
  for (int k = 0; k < TILE; ++k) {
    const int i = k, j = TILE - 1 - k;
    const float di = d[i];
    const float a = fminf(di, __fadd_rn(f, wc[i]));
    const float from_prev = __shfl_up_sync(~0u, a, 1);
    const float from_next = __shfl_down_sync(~0u, __fadd_rn(a, wx[i]), 1);
    const float c = fminf(a, fminf(__fadd_rn(from_prev, wx[i]), from_next));
    ch |= c < di;
    d[i] = c;
    f = c;
    const float dj = d[j];
    const float e = fminf(dj, __fadd_rn(b, wc[j + 1]));
    const float from_prev2 = __shfl_up_sync(~0u, e, 1);
    const float from_next2 = __shfl_down_sync(~0u, __fadd_rn(e, wx[j]), 1);
    const float g = fminf(e, fminf(__fadd_rn(from_prev2, wx[j]), from_next2));
    ch |= g < dj;
    d[j] = g;
    b = g;
  }
  return ch;
}

}  // namespace dtb
