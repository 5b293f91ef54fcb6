// dtb_kernels.cuh -- the GGDT tile visit (warp per 32x32 tile) and the kernels built from it.
//
// Kernels
//   ggdt_scan        seed-tile scan: reads every mask tile once, writes the tile states and queues the tiles
//                    that hold seeds (replaces initialize_generalised_distance_map + initialize_task_queue,
//                    reference dt/src/utils.cu:5-18, and the priority set-up of dt/src/block_priority.cu).
//   ggdt_persistent  cooperative persistent kernel: every warp pops tiles from the shared queue, visits them
//                    and re-activates neighbours whose halo it can still lower (replaces the task variant,
//                    reference dt/src/generalised_distance_transform_task.cu:129-150).  No grid barrier:
//                    termination is "queue empty and nothing in flight".
//   ggdt_round       one host-driven round over the active tiles (the plain per-image path; the round
//                    structure of reference dt/src/generalised_distance_transform_blocks.cu:156-163).
//   ggdt_finalize    writes v into tiles that were never reached (their memory was never initialised).
#pragma once

#include "dtb_device.cuh"

namespace dtb {

constexpr int PHASE_LIMIT = 4096;
constexpr uint64_t TMA_TIMEOUT_NS = 2000000000ull;  // 2 s

// ------------------------------------------------------------------------------------------------------
// Schedulers: what "activate a neighbour" and "finish a visit" mean.
// ------------------------------------------------------------------------------------------------------
// Per-warp counters, flushed to the queue header in batches (the header lines are shared by all warps).
struct WarpStats {
  uint32_t visits = 0, phases = 0, activations = 0, unflushed = 0;
};

struct QueueSched {
  Queue q;
  uint32_t* states;
  // Optional: the warp's word for a tile it keeps.  Of the tiles a visit queues, one in the lowest bucket
  // (the one the workers take from: its activation value is among the smallest queued) is not pushed; the warp
  // visits it next, which saves the ring's push and pop (two to five L2 round trips) and reuses the halo just
  // written.  It stays counted in `pending` like a queued tile.  nullptr: every tile goes through the ring.
  uint32_t* keep_out = nullptr;
  // Warp-level end of a visit.  Lanes with `want` ask for a re-run of neighbour `item`, bringing activation
  // value `key` (distance units; bucket width 1 / inv_width): idle -> queued; running -> running with a re-run
  // requested; queued -> unchanged.  Lane 31 clears RUNNING of the own tile (and sets / clears the xor_bits);
  // a re-run requested meanwhile re-queues it at the smallest value its activators left in keys[].  `pending`
  // moves by (pushes - 1) in one atomic performed before any push is visible; the visit that brings it to 0
  // ends the queue.
  // The own-tile update comes first and, when it sets VISITED, is fenced before the activations: a woken
  // neighbour takes this tile's distances as halo only if it sees VISITED, and otherwise reads v in their
  // place.  Seeing the activation without the bit would consume the wake-up without the new distances.
  __device__ __forceinline__ void complete(uint32_t tile, uint32_t xor_bits, bool want, uint32_t want_item,
                                           float key = 0.0f, float inv_width = 0.0f) const {
    const int lane = threadIdx.x & 31;
    bool push = false;
    uint32_t item = 0;
    float pkey = key;
    if (lane == 31) {
      const uint32_t old = atomicXor(&states[tile], xor_bits | ST_RUNNING);
      push = (old & ST_PENDING) != 0u;
      item = tile;
      if (push && q.keys) {
        const uint32_t kb = ld_volatile(&q.keys[tile]);
        pkey = kb == KEY_NONE ? 0.0f : __uint_as_float(kb);
      }
      if (xor_bits & ST_VISITED) fence_acq_rel();
    }
    __syncwarp();
    if (want) {
      if (want_item >= q.total_tiles) {
        set_error(q, DERR_BAD_TILE, want_item);
      } else {
        if (q.keys) {
          const uint32_t prev = atomicMin(&q.keys[want_item], __float_as_uint(key));
          pkey = fminf(key, __uint_as_float(prev == KEY_NONE ? __float_as_uint(key) : prev));
        }
        const uint32_t old = atomicOr(&states[want_item], ST_PENDING);
        push = !(old & (ST_PENDING | ST_RUNNING));
        item = want_item;
      }
    }
    const uint32_t m = __ballot_sync(~0u, push);
    const uint32_t k = __popc(m);
    uint32_t last = 0;
    if (lane == 0) {
      if (k == 0) {
        last = atomicSub(&q.hdr->pending.v, 1u) == 1u ? 1u : 0u;
      } else if (k > 1) {
        atomicAdd(&q.hdr->pending.v, k - 1u);
      }
      fence_acq_rel();
    }
    __syncwarp();
    uint32_t base = 0;
    if (q.nb_mask) base = ld_volatile(&q.hdr->base.v);
    const uint32_t b = push ? bucket_at(q, pkey, inv_width, base) : 0u;
    int kept = -1;
    if (keep_out) {
      // The own tile first (lane 31 re-queues it when its halo dropped during the visit): its re-run reuses the
      // weights and distances in this warp's shared memory.  Else the smallest activation value.
      const bool elig = push && b == (base & q.nb_mask);
      const uint32_t em = __ballot_sync(~0u, elig);
      if (__ballot_sync(~0u, push) >> 31) {  // the own tile, whatever its bucket: its re-run is cheap
        kept = 31;
      } else {
        const uint32_t kmin = __reduce_min_sync(~0u, elig ? __float_as_uint(pkey) : 0xFFFFFFFFu);
        const uint32_t cand = __ballot_sync(~0u, elig && __float_as_uint(pkey) == kmin);
        if (cand) kept = __ffs(cand) - 1;
      }
      if (lane == kept) *keep_out = item;
    }
    if (push && lane != kept) slot_write(q, b, atomicAdd(&q.hdr->tails[b].v, 1u), item);
    __syncwarp();
    if (__shfl_sync(~0u, last, 0)) signal_done_warp(q);
  }
};

struct RoundSched {
  Queue q;  // only the counters and error word are used
  uint32_t* states;
  uint8_t* next_active;
  uint32_t* changed;
  __device__ __forceinline__ void complete(uint32_t tile, uint32_t xor_bits, bool want, uint32_t want_item,
                                           float = 0.0f, float = 0.0f) const {
    if (want) {
      if (want_item >= q.total_tiles) {
        set_error(q, DERR_BAD_TILE, want_item);
      } else {
        next_active[want_item] = 1;
        *(volatile uint32_t*)changed = 1u;
      }
    }
    if ((threadIdx.x & 31) == 31 && xor_bits) atomicXor(&states[tile], xor_bits);
  }
};

// Adds a finished visit to the warp's counters; flushes `progress` every 16 visits (the watchdog and the
// visit cap only need it approximately).
__device__ __forceinline__ void count_visit(WarpStats& ws, const Queue& q, uint32_t nphase, uint32_t nact) {
  ws.visits += 1;
  ws.phases += nphase;
  ws.activations += nact;
  if (++ws.unflushed == 16) {
    if ((threadIdx.x & 31) == 0) atomicAdd(&q.hdr->progress.v, ws.unflushed);
    ws.unflushed = 0;
  }
}

__device__ __forceinline__ void flush_stats(WarpStats& ws, const Queue& q) {
  if ((threadIdx.x & 31) == 0) {
    if (ws.unflushed) atomicAdd(&q.hdr->progress.v, ws.unflushed);
    if (ws.phases) atomicAdd(&q.hdr->phases.v, ws.phases);
    if (ws.activations) atomicAdd(&q.hdr->activations.v, ws.activations);
  }
  ws = WarpStats{};
}

__device__ __forceinline__ float f_inf() { return __int_as_float(0x7f800000); }

__device__ __forceinline__ float* dist_row(const ImgDesc& dd, int y) {
  return reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(dd.dist) + (int64_t)y * dd.dist_pitch);
}

// Distance read of a pixel that another warp (on any SM) may have written during this launch: L2 only, so no
// line an SM cached earlier can be returned.
__device__ __forceinline__ float ld_dist(const ImgDesc& dd, int y, int x) { return __ldcg(dist_row(dd, y) + x); }

// Address of column x of row y0 of the distance map, passed through an empty asm that also takes `dep`.  A
// visit's tile loads and its write-back each take their row addresses from such a base, with different `dep`:
// the compiler then cannot keep the 32 row addresses of the loads live across the whole visit to reuse them in
// the write-back (64 registers).
__device__ __forceinline__ uint8_t* dist_base(const ImgDesc& dd, int y0, int x, uint32_t dep) {
  uint8_t* p = reinterpret_cast<uint8_t*>(dist_row(dd, y0) + x);
  asm("" : "+l"(p) : "r"(dep));
  return p;
}
__device__ __forceinline__ float ld_dist_at(const uint8_t* base, int64_t pitch, int y) {
  return __ldcg(reinterpret_cast<const float*>(base + (int64_t)y * pitch));
}

// Waits for the TMA transactions on `bar`; its phase parity is bit `pmask` of `pbits`.  Bounded: after
// TMA_TIMEOUT_NS the error word is set and the wait goes on for as long again, to give a slow copy the chance
// to land before the warp leaves; after that the wait gives up, and a copy may then still be pending.  The
// error word ends the launch: every later pop returns POP_NONE, so the warp issues no further copy and never
// waits on this barrier again.
__device__ __forceinline__ bool tma_wait(uint64_t* bar, uint32_t& pbits, uint32_t pmask, const Queue& q, uint32_t tile) {
  const uint32_t parity = (pbits & pmask) ? 1u : 0u;
  const uint64_t t0 = globaltimer();
  bool ok = true;
  while (!mbar_try_wait(bar, parity)) {
    const uint64_t dt = globaltimer() - t0;
    if (ok && dt > TMA_TIMEOUT_NS) { set_error(q, DERR_TMA_TIMEOUT, tile); ok = false; }
    if (dt > 2 * TMA_TIMEOUT_NS) break;
  }
  pbits ^= pmask;
  return ok;
}

// Shared memory of one visit.  A self-staging visit loads its image box and seed-mask box on `bar`; a visit
// staged ahead finds its image box issued on `bar` already and loads the mask box (seed visits only) on `mbar`.
struct VisitBufs {
  uint8_t* box;       // image box (TMA destination), the tile buffer B once the weights are computed
  float* Wh;
  float* Wv;          // its first 1 KB receives the seed-mask box before the weights
  uint64_t* bar;
  uint64_t* mbar;
  uint32_t pmask;     // bit of *pbits holding bar's phase parity
  uint32_t mmask;     // bit of *pbits holding mbar's phase parity
  uint32_t* pbits;
};

__device__ __forceinline__ VisitBufs visit_bufs(WarpSmem& sm, uint32_t& pbits) {
  return VisitBufs{sm.img, sm.Wh, sm.Wv, &sm.bar, &sm.bar, 1u, 1u, &pbits};
}

// Issues one 2-D TMA box into this warp's shared memory on `bar` (whole warp; lane 0 issues).  Orders this
// warp's earlier generic accesses of the destination before the async-proxy writes.
__device__ __forceinline__ void stage_box(void* dst, uint64_t* bar, const CUtensorMap* tm, uint32_t bytes, int x, int y) {
  fence_proxy_async_smem();
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    tmap_acquire(tm);
    mbar_arrive_expect_tx(bar, bytes);
    tma_load_2d(dst, tm, x, y, bar);
  }
}

// The image box of a tile (1-pixel halo; x starts 16 bytes left of the halo so that it stays 16-byte aligned).
__device__ __forceinline__ void stage_image_box(uint8_t* box, uint64_t* bar, const CUtensorMap* tm_img, bool rgb, int x0,
                                                int y0) {
  stage_box(box, bar, tm_img, (rgb ? IMG_BOX_RGB : IMG_BOX_GRAY) * IMG_BOX_ROWS, rgb ? 3 * x0 - 16 : x0 - 16, y0 - 1);
}

// Issues the image box of a warp's next tile ahead of its visit (the image index bits of a tile state never
// change, so reading them before the tile is claimed is safe).
__device__ __forceinline__ void stage_ahead(const ImgDesc* __restrict__ descs, const CUtensorMap* __restrict__ tmaps,
                                            const uint32_t* states, uint32_t tile, uint8_t* box, uint64_t* bar) {
  uint32_t st = 0;
  if ((threadIdx.x & 31) == 0) st = ld_volatile(&states[tile]);
  const uint32_t img = __shfl_sync(~0u, st, 0) >> ST_IMG_SHIFT;
  const ImgDesc& dd = descs[img];
  const uint32_t local = tile - dd.tile_base;
  const uint32_t tx = local % (uint32_t)dd.tiles_x, ty = local / (uint32_t)dd.tiles_x;
  stage_image_box(box, bar, tmaps + 2 * img, dd.channels == 3, (int)tx * TILE, (int)ty * TILE);
}

// Stages the image box (with 1-pixel halo) and, if needed, the seed-mask tile of a tile into shared memory,
// both on vb.bar.
__device__ __forceinline__ void stage_tile(const VisitBufs& vb, const CUtensorMap* tm_img, const CUtensorMap* tm_mask,
                                           bool rgb, bool with_mask, int x0, int y0) {
  // Order this warp's earlier generic reads of the slot before the async-proxy writes below.
  fence_proxy_async_smem();
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    tmap_acquire(tm_img);
    if (with_mask) tmap_acquire(tm_mask);
    const uint32_t bytes = (rgb ? IMG_BOX_RGB : IMG_BOX_GRAY) * IMG_BOX_ROWS + (with_mask ? TILE * TILE : 0);
    mbar_arrive_expect_tx(vb.bar, bytes);
    tma_load_2d(vb.box, tm_img, rgb ? 3 * x0 - 16 : x0 - 16, y0 - 1, vb.bar);
    if (with_mask) tma_load_2d(vb.Wv, tm_mask, x0, y0, vb.bar);
  }
}

// Packed pixel of the staged image box: box row r (tile row r - 1), tile column c in [-1, 32].
__device__ __forceinline__ uint32_t box_pix(const uint8_t* box, bool rgb, int r, int c) {
  if (!rgb) return box[r * IMG_BOX_GRAY + 16 + c];
  const int off = r * IMG_BOX_RGB + 16 + 3 * c;
  const uint32_t* wp = reinterpret_cast<const uint32_t*>(box + (off & ~3));
  return __funnelshift_r(wp[0], wp[1], (off & 3) * 8) & 0xFFFFFFu;
}

// A lane's row of 32 floats of a W_STRIDE buffer (16-byte aligned), as 8 vector loads / stores.
__device__ __forceinline__ void load_row(float (&d)[TILE], const float* row) {
  const float4* p = reinterpret_cast<const float4*>(row);
#pragma unroll
  for (int j = 0; j < TILE / 4; ++j) {
    const float4 v4 = p[j];
    d[4 * j] = v4.x; d[4 * j + 1] = v4.y; d[4 * j + 2] = v4.z; d[4 * j + 3] = v4.w;
  }
}
__device__ __forceinline__ void store_row(float* row, const float (&d)[TILE]) {
  float4* p = reinterpret_cast<float4*>(row);
#pragma unroll
  for (int j = 0; j < TILE / 4; ++j) p[j] = make_float4(d[4 * j], d[4 * j + 1], d[4 * j + 2], d[4 * j + 3]);
}

// ------------------------------------------------------------------------------------------------------
// ns-mode visit (C4, w = sqrt(1 + g2 * dI2)), gray or rgb8.
//
// Layouts: "column" (lane = x, d[y]) and "row" (lane = y, d[x]).  Each phase (sweep_phase) relaxes every
// internal edge of the tile and the halo edges of its own axis; the halo edges of the other axis were relaxed
// by an earlier phase and stay satisfied, because tile values only decrease while the halo is fixed.  So the
// visit stops at the first phase that changes nothing once both layouts have run: every edge of the tile and
// its halo is then satisfied.  The halo is an upper bound of the neighbours' values (values only decrease;
// never-visited neighbours read as v), so the visit never undershoots the fixpoint.  A neighbour is
// re-activated only if some border pixel plus its edge weight is below the halo value it was compared with.
//
// One code path serves both layouts (the phase loop is small enough to stay in the instruction cache): the
// weights live in shared memory as Wh / Wv (stride 36: scalar lane-per-column reads and 16-byte lane-per-row
// reads are conflict-free) and are loaded into registers for the phase's layout; the tile changes layout through
// B.  Element k of lane l is at [k * 36 + l] of the row-major arrays in the column layout (scalar loads), at
// [l * 36 + k] in the row layout (16-byte vectors).
// Returns the number of phases and activations through *nph / *nact.
//
// rerun: the warp visits again the tile it has just visited (its halo dropped while it ran, and the visit kept
// it).  The warp's shared memory still holds that tile's edge weights (Wh / Wv) and its final distances (the
// tile buffer B, equal to the tile in global memory: no other warp can have visited it in between), so the
// re-run reloads only the neighbour states and halos: no bulk copy, no weights, no tile loads.
// ------------------------------------------------------------------------------------------------------
template <bool PRESTAGED, class Sched>
__device__ __forceinline__ void visit_ns(const ImgDesc& dd, const CUtensorMap* tm_img, const CUtensorMap* tm_mask,
                                         uint32_t tile, uint32_t old_state, const VisitBufs& vb, const Sched& sch,
                                         uint32_t* nph_out, uint32_t* nact_out, bool rerun = false) {
  const int lane = threadIdx.x & 31;
  const float INF = f_inf();
  const uint32_t local = tile - dd.tile_base;
  const int tx = (int)(local % (uint32_t)dd.tiles_x), ty = (int)(local / (uint32_t)dd.tiles_x);
  const int x0 = tx * TILE, y0 = ty * TILE;
  const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
  const bool first = !(old_state & ST_VISITED);
  const bool seed = (old_state & ST_SEED) != 0;
  const bool rgb = dd.channels == 3;
  const float v = dd.v;
  *nph_out = 0;
  *nact_out = 0;

  if (rerun) {
  } else if (!PRESTAGED) {
    stage_tile(vb, tm_img, tm_mask, rgb, seed, x0, y0);
  } else if (seed) {
    stage_box(vb.Wv, vb.mbar, tm_mask, TILE * TILE, x0, y0);
  }

  // Neighbour states: lane 0 left, 1 right, 2 top, 3 bottom.
  const uint32_t nexist = (tx > 0 ? 1u : 0u) | (tx + 1 < dd.tiles_x ? 2u : 0u) | (ty > 0 ? 4u : 0u) |
                          (ty + 1 < dd.tiles_y ? 8u : 0u);
  const int nbx = tx + (lane == 0 ? -1 : lane == 1 ? 1 : 0);
  const int nby = ty + (lane == 2 ? -1 : lane == 3 ? 1 : 0);
  const uint32_t nb_tile = dd.tile_base + (uint32_t)(nby * dd.tiles_x + nbx);  // meaningful for lanes < 4
  uint32_t nvis;
  {
    bool vis = false;
    if (lane < 4 && ((nexist >> lane) & 1u)) vis = (ld_volatile(&sch.states[nb_tile]) & ST_VISITED) != 0;
    nvis = __ballot_sync(~0u, vis);
  }
  fence_acq_rel();  // acquire: distances were written before the VISITED bits / the activation we saw

  // Halo: column layout for top/bottom (lane = x), row layout for left/right (lane = y).
  float top = INF, bot = INF, lft = INF, rgt = INF;
  if (lane < vw) {
    if (nexist & 4u) top = (nvis & 4u) ? ld_dist(dd, y0 - 1, x0 + lane) : v;
    if (nexist & 8u) bot = (nvis & 8u) ? ld_dist(dd, y0 + TILE, x0 + lane) : v;
  }
  if (lane < vh) {
    if (nexist & 1u) lft = (nvis & 1u) ? ld_dist(dd, y0 + lane, x0 - 1) : v;
    if (nexist & 2u) rgt = (nvis & 2u) ? ld_dist(dd, y0 + lane, x0 + TILE) : v;
  }

  // Tile distances in column layout.
  float d[TILE];
  if (rerun) {
    const float* pb = reinterpret_cast<const float*>(vb.box) + lane;  // B[y * 36 + x]
#pragma unroll
    for (int y = 0; y < TILE; ++y) d[y] = pb[y * W_STRIDE];
  } else if (!first) {
    const uint8_t* lb = dist_base(dd, y0, x0 + lane, 0u);
#pragma unroll
    for (int y = 0; y < TILE; ++y) d[y] = (lane < vw && y < vh) ? ld_dist_at(lb, dd.dist_pitch, y) : INF;
  }

  if (!rerun && !tma_wait(vb.bar, *vb.pbits, vb.pmask, sch.q, tile)) return;
  if (PRESTAGED && seed && !tma_wait(vb.mbar, *vb.pbits, vb.mmask, sch.q, tile)) return;
  const uint8_t* mbox = reinterpret_cast<const uint8_t*>(vb.Wv);

  // Seeds first: the mask box shares memory with Wv.
  if (first) {
#pragma unroll
    for (int y = 0; y < TILE; ++y) {
      const bool in = lane < vw && y < vh;
      const bool s = seed && mbox[y * TILE + lane] != 0;
      d[y] = in ? (s ? 0.0f : v) : INF;
    }
  } else if (seed) {
#pragma unroll
    for (int y = 0; y < TILE; ++y)
      if (lane < vw && y < vh && mbox[y * TILE + lane] != 0) d[y] = 0.0f;
  }
  __syncwarp();

  // Edge weights into Wh / Wv (computed in column layout, lane = x).  Edges touching a pixel outside the image
  // are INF.  A re-run has them from its previous visit.
  if (!rerun) {
    const float g2 = dd.g2;
    const uint8_t* box = vb.box;
    if (!rgb) {
      // Gray: the weight depends on |dI| in [0, 255] only.  A 256-entry table of the same expression (so the
      // same bits) costs 8 square roots per lane instead of 65; it sits in the part of the image box that the
      // 64-byte gray rows leave unused.
      float* lut = reinterpret_cast<float*>(vb.box + GRAY_LUT_OFFSET);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t a = (uint32_t)(lane + 32 * k);
        lut[a] = ns_weight_sq(a * a, g2);
      }
      __syncwarp();
      const uint8_t* col = box + 16 + lane;  // column `lane` of the box, row r at col[r * IMG_BOX_GRAY]
      int pprev = col[0];
      // Unrolled 2: the 1024-image batch ran 0.7 % faster than with 4 (8 was 2.4 % slower).
#pragma unroll 2
      for (int y = 0; y <= TILE; ++y) {  // edge (y-1, y); y == 32 is the bottom halo edge
        const int pcur = col[(y + 1) * IMG_BOX_GRAY];
        float w = lut[abs(pcur - pprev)];
        if (lane >= vw || (y < TILE ? y >= vh : TILE - 1 >= vh)) w = INF;
        vb.Wv[y * W_STRIDE + lane] = w;
        if (y < TILE) {
          float wx = lut[abs(pcur - (int)col[(y + 1) * IMG_BOX_GRAY - 1])];
          if (lane >= vw || y >= vh) wx = INF;
          vb.Wh[y * W_STRIDE + lane] = wx;
        }
        pprev = pcur;
      }
      const uint8_t* row = box + (lane + 1) * IMG_BOX_GRAY + 16;
      float er = lut[abs((int)row[TILE - 1] - (int)row[TILE])];
      if (lane >= vh || TILE - 1 >= vw) er = INF;
      vb.Wh[lane * W_STRIDE + TILE] = er;
    } else {
      uint32_t pprev = box_pix(box, rgb, 0, lane);
#pragma unroll 1
      for (int y = 0; y <= TILE; ++y) {  // edge (y-1, y); y == 32 is the bottom halo edge
        const uint32_t pcur = box_pix(box, rgb, y + 1, lane);
        float w = ns_weight(pprev, pcur, g2);
        if (lane >= vw || (y < TILE ? y >= vh : TILE - 1 >= vh)) w = INF;
        vb.Wv[y * W_STRIDE + lane] = w;
        if (y < TILE) {
          float wx = ns_weight(box_pix(box, rgb, y + 1, lane - 1), pcur, g2);
          if (lane >= vw || y >= vh) wx = INF;
          vb.Wh[y * W_STRIDE + lane] = wx;
        }
        pprev = pcur;
      }
      // Edge (x = 31, x = 32) of row `lane`.
      float er = ns_weight(box_pix(box, rgb, lane + 1, TILE - 1), box_pix(box, rgb, lane + 1, TILE), g2);
      if (lane >= vh || TILE - 1 >= vw) er = INF;
      vb.Wh[lane * W_STRIDE + TILE] = er;
    }
  }
  __syncwarp();

  // Bucket width of this image: one tile-width of path cost, 32 x the mean internal edge weight seen so far by
  // first visits (each first visit adds its column edges).
  const uint32_t img_idx = old_state >> ST_IMG_SHIFT;
  float inv_width = 0.0f;
  if (sch.q.wacc) {
    float* wa = sch.q.wacc + 2 * img_idx;
    if (first) {
      float wsum = 0.0f, wcnt = 0.0f;
#pragma unroll 4
      for (int y = 1; y < TILE; ++y) {
        const float w = vb.Wv[y * W_STRIDE + lane];
        if (w < INF) { wsum += w; wcnt += 1.0f; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        wsum += __shfl_xor_sync(~0u, wsum, o);
        wcnt += __shfl_xor_sync(~0u, wcnt, o);
      }
      if (lane == 0 && wcnt > 0.0f) {
        atomicAdd(&wa[0], wsum);
        atomicAdd(&wa[1], wcnt);
      }
    }
    const float s_ = *(volatile float*)&wa[0], c_ = *(volatile float*)&wa[1];
    const float bt = sch.q.bucket_tiles;
    inv_width = (c_ > 0.0f && s_ > 0.0f) ? c_ / (bt * (float)TILE * s_) : 1.0f / (bt * (float)TILE);
  }

  // Local fixpoint.  B overlays the image box, which is no longer needed.
  float* B = reinterpret_cast<float*>(vb.box);
  // Start in the layout whose chains begin at the halo sides that can lower the tile now: a column phase
  // never reads the left / right halo, so a tile reached only from the side would spend its first column
  // phase without any effect.
  bool col = true;
  // hside / vside: whether the left / right (top / bottom) halo can lower the tile as it stands.  A phase that
  // changes nothing proves every internal edge and its own axis's halo edges satisfied; if the first phase
  // changes nothing and the other axis's halo could not lower the unchanged tile, the tile is at its fixpoint
  // and the visit ends after that one phase (a false-positive activation costs one phase, not two).
  bool hside, vside;
  {
    float* pb = B + lane;
#pragma unroll
    for (int k = 0; k < TILE; ++k) pb[k * W_STRIDE] = d[k];
    __syncwarp();
    const float dl = B[lane * W_STRIDE], dr = B[lane * W_STRIDE + TILE - 1];
    hside = __any_sync(~0u, __fadd_rn(lft, vb.Wh[lane * W_STRIDE]) < dl ||
                                 __fadd_rn(rgt, vb.Wh[lane * W_STRIDE + TILE]) < dr);
    vside = __any_sync(~0u, __fadd_rn(top, vb.Wv[lane]) < d[0] ||
                                 __fadd_rn(bot, vb.Wv[TILE * W_STRIDE + lane]) < d[TILE - 1]);
    if (hside && !vside) {
      col = false;
      load_row(d, B + lane * W_STRIDE);
    }
    __syncwarp();
  }
  bool any = false, ran_col = false, ran_row = false;
  uint32_t nph = 0;
  for (;;) {
    float wc[TILE + 1], wx[TILE];
    if (col) {  // element k of lane x: [k * 36 + x]
      const float* pc = vb.Wv + lane;
      const float* px = vb.Wh + lane;
#pragma unroll
      for (int k = 0; k <= TILE; ++k) wc[k] = pc[k * W_STRIDE];
#pragma unroll
      for (int k = 0; k < TILE; ++k) wx[k] = px[k * W_STRIDE];
    } else {    // element k of lane y: [y * 36 + k], as 16-byte vectors
      const float4* pc = reinterpret_cast<const float4*>(vb.Wh + lane * W_STRIDE);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float4 v4 = pc[j];
        wc[4 * j] = v4.x; wc[4 * j + 1] = v4.y; wc[4 * j + 2] = v4.z; wc[4 * j + 3] = v4.w;
      }
      wc[TILE] = pc[8].x;
      load_row(wx, vb.Wv + lane * W_STRIDE);
    }
    bool ch = sweep_phase(d, wc, wx, col ? top : lft, col ? bot : rgt);
    ch = __any_sync(~0u, ch);
    any |= ch;
    ran_col |= col;
    ran_row |= !col;
    ++nph;
    const bool stop = (!ch && ((ran_col && ran_row) || (nph == 1 && !(col ? hside : vside)))) ||
                      nph >= (uint32_t)PHASE_LIMIT;
    if (col) {
      float* pb = B + lane;
#pragma unroll
      for (int k = 0; k < TILE; ++k) pb[k * W_STRIDE] = d[k];
      __syncwarp();
      if (stop) break;
      load_row(d, B + lane * W_STRIDE);
    } else {
      store_row(B + lane * W_STRIDE, d);
      __syncwarp();
      if (stop) break;
      const float* qb = B + lane;
#pragma unroll
      for (int k = 0; k < TILE; ++k) d[k] = qb[k * W_STRIDE];
    }
    col = !col;
    __syncwarp();
  }
  if (nph >= (uint32_t)PHASE_LIMIT && lane == 0) set_error(sch.q, DERR_PHASE_LIMIT, tile);

  // Neighbours that can still decrease (bit 0 left, 1 right, 2 top, 3 bottom).
  uint32_t act = 0;
  float act_key = 0.0f;
  if (any || seed) {
    const float dt = B[lane], db = B[(TILE - 1) * W_STRIDE + lane];               // column layout
    const float dl = B[lane * W_STRIDE], dr = B[lane * W_STRIDE + TILE - 1];      // row layout
    const float wt = vb.Wv[lane], wb = vb.Wv[TILE * W_STRIDE + lane];
    const float wl = vb.Wh[lane * W_STRIDE], wr = vb.Wh[lane * W_STRIDE + TILE];
    // The activation value of a side: the smallest border value it can bring (its priority in the queue).
    const float vl = __fadd_rn(dl, wl), vr = __fadd_rn(dr, wr), vt = __fadd_rn(dt, wt), vb = __fadd_rn(db, wb);
    const uint32_t kl = __reduce_min_sync(~0u, vl < lft ? __float_as_uint(vl) : KEY_NONE);
    const uint32_t kr = __reduce_min_sync(~0u, vr < rgt ? __float_as_uint(vr) : KEY_NONE);
    const uint32_t kt = __reduce_min_sync(~0u, vt < top ? __float_as_uint(vt) : KEY_NONE);
    const uint32_t kbm = __reduce_min_sync(~0u, vb < bot ? __float_as_uint(vb) : KEY_NONE);
    act = (kl != KEY_NONE ? 1u : 0u) | (kr != KEY_NONE ? 2u : 0u) | (kt != KEY_NONE ? 4u : 0u) |
          (kbm != KEY_NONE ? 8u : 0u);
    // A missing neighbour has an INF halo, and fl(d + w) < INF holds for any finite d: mask by existence.
    act &= nexist;
    act_key = __uint_as_float(lane == 0 ? kl : lane == 1 ? kr : lane == 2 ? kt : kbm);
  }

  // Write back (column layout: each row is one coalesced 128-byte store).
  if (any || first) {
    if (lane < vw) {
      uint8_t* wb = dist_base(dd, y0, x0 + lane, nph);
#pragma unroll 4
      for (int y = 0; y < TILE; ++y)
        if (y < vh) *reinterpret_cast<float*>(wb + (int64_t)y * dd.dist_pitch) = B[y * W_STRIDE + lane];
    }
  }
  fence_acq_rel();  // release: distances before activations and before the VISITED bit
  __syncwarp();
  sch.complete(tile, (first ? ST_VISITED : 0u) | (seed ? ST_SEED : 0u), lane < 4 && ((act >> lane) & 1u), nb_tile,
               act_key, inv_width);
  *nph_out = nph;
  *nact_out = (uint32_t)__popc(act);
}

// ------------------------------------------------------------------------------------------------------
// ref-mode visit (C8, reference weight), gray only.
//
// Mirrors the reference's in-tile passes (dt/src/dt_block_passes.cuh:12-127): a row phase relaxes every
// pixel from its three predecessors in the previous column (forward and backward chains interleaved), a
// column phase from the three predecessors in the previous row.  The three rows (columns) move in lockstep,
// so the predecessors of lane l come from lanes l-1 / l+1 by shuffle, or from the halo for the edge lanes.
// Each relaxation is a single edge with the reference's arithmetic (ref_relax).  Neighbours (8 of them)
// are re-activated when a border pixel facing them decreased, as in dt_block_passes.cuh:50-63, and on
// visits that applied seeds.
// ------------------------------------------------------------------------------------------------------
constexpr int PIMG_STRIDE = 36;  // padded image copies: 34 lines x 36 bytes (9 words a line, odd word stride)

// Pixel at position pos (-1..32) of an image line packed 4 per word (byte (pos + 1) & 3 of word (pos + 1) >> 2)
// as a float.  pos is a constant after unrolling, so this is one bit-field extract and one conversion.
__device__ __forceinline__ float line_px(const uint32_t (&w)[9], int pos) {
  const int i = pos + 1;
  return (float)((w[i >> 2] >> ((i & 3) * 8)) & 0xFFu);
}

template <bool FMA>
__device__ __forceinline__ float ref_min3(float cur, float da, float db, float dc, float le, float lg, float sq2,
                                          float ia, float ib, float ic, bool diag_a, bool diag_c) {
  // a and c are the diagonal predecessors, b the axial one
  const float ra = ref_relax<FMA>(da, diag_a ? sq2 : 1.0f, le, lg, ia);
  const float rb = ref_relax<FMA>(db, 1.0f, le, lg, ib);
  const float rc = ref_relax<FMA>(dc, diag_c ? sq2 : 1.0f, le, lg, ic);
  return fminf(cur, fminf(rb, fminf(ra, rc)));
}

template <bool FMA, class Sched>
__device__ __forceinline__ void visit_ref(const ImgDesc& dd, const CUtensorMap* tm_img, const CUtensorMap* tm_mask,
                                          uint32_t tile, uint32_t old_state, WarpSmem& sm, uint32_t& parity,
                                          const Sched& sch, uint32_t* nph_out, uint32_t* nact_out,
                                          bool rerun = false) {
  // rerun: as in visit_ns -- the padded image lines (pimg / pimgT) and the tile values (T) of this tile's previous
  // visit are still in the warp's shared memory; only the neighbour states and halos are read again.
  *nph_out = 0;
  *nact_out = 0;
  const int lane = threadIdx.x & 31;
  const float INF = f_inf();
  const uint32_t local = tile - dd.tile_base;
  const int tx = (int)(local % (uint32_t)dd.tiles_x), ty = (int)(local / (uint32_t)dd.tiles_x);
  const int x0 = tx * TILE, y0 = ty * TILE;
  const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
  const bool first = !(old_state & ST_VISITED);
  const bool seed = (old_state & ST_SEED) != 0;
  const float v = dd.v, le = dd.l_eucl, lg = dd.l_grad;
  const float sq2 = 1.41421354f;  // sqrtf(2.f), reference generalised_distance_transform.cu:111

  const VisitBufs vb = visit_bufs(sm, parity);
  if (!rerun) stage_tile(vb, tm_img, tm_mask, false, seed, x0, y0);

  // Neighbour k = lane (0..7): (dx, dy) = L, R, T, B, TL, TR, BL, BR.
  // Offsets of neighbour k = lane, the tables {-1,1,0,0,-1,1,-1,1} and {0,0,-1,1,-1,-1,1,1} as bit masks (an
  // array indexed by the lane would live in local memory).
  const int ndx_l = (0xF3u >> lane) & 1u ? ((0xA2u >> lane) & 1u ? 1 : -1) : 0;
  const int ndy_l = (0xFCu >> lane) & 1u ? ((0xC8u >> lane) & 1u ? 1 : -1) : 0;
  uint32_t nvis, nexist;
  {
    bool vis = false, ex = false;
    if (lane < 8) {
      const int nx = tx + ndx_l, ny = ty + ndy_l;
      ex = nx >= 0 && ny >= 0 && nx < dd.tiles_x && ny < dd.tiles_y;
      if (ex) vis = (ld_volatile(&sch.states[dd.tile_base + (uint32_t)(ny * dd.tiles_x + nx)]) & ST_VISITED) != 0;
    }
    nvis = __ballot_sync(~0u, vis);
    nexist = __ballot_sync(~0u, ex);
  }
  fence_acq_rel();

  // Halo rows / columns in shared memory, index = coordinate + 1 (corners appear in both).
  float* ht = sm.Wh;                // top row   (y0 - 1), x = -1..32
  float* hb = sm.Wh + 40;           // bottom row (y0 + 32)
  float* hl = sm.Wv + 256;          // left column (x0 - 1), y = -1..32 (after the 1 KB seed-mask box)
  float* hr = sm.Wv + 300;          // right column (x0 + 32)
  auto halo_val = [&](int k, int gx, int gy) -> float {  // neighbour k's pixel (gx, gy)
    if (!((nexist >> k) & 1u)) return INF;
    if (gx >= dd.width || gy >= dd.height) return INF;
    return ((nvis >> k) & 1u) ? ld_dist(dd, gy, gx) : v;
  };
  ht[lane + 1] = (lane < vw) ? halo_val(2, x0 + lane, y0 - 1) : INF;
  hb[lane + 1] = (lane < vw) ? halo_val(3, x0 + lane, y0 + TILE) : INF;
  hl[lane + 1] = (lane < vh) ? halo_val(0, x0 - 1, y0 + lane) : INF;
  hr[lane + 1] = (lane < vh) ? halo_val(1, x0 + TILE, y0 + lane) : INF;
  if (lane == 0) {
    const float tl = halo_val(4, x0 - 1, y0 - 1), tr = halo_val(5, x0 + TILE, y0 - 1);
    const float bl = halo_val(6, x0 - 1, y0 + TILE), br = halo_val(7, x0 + TILE, y0 + TILE);
    ht[0] = tl; hl[0] = tl;
    ht[TILE + 1] = tr; hr[0] = tr;
    hb[0] = bl; hl[TILE + 1] = bl;
    hb[TILE + 1] = br; hr[TILE + 1] = br;
  }

  // Tile values live in T (column-layout transposes) = sm.img region after staging is consumed.
  float* T = reinterpret_cast<float*>(sm.img);  // 32 x 33 floats = 4224 bytes <= 4352
  float d[TILE];
  if (rerun) {
#pragma unroll
    for (int y = 0; y < TILE; ++y) d[y] = T[y * S_STRIDE + lane];
  } else if (!first) {
    const uint8_t* lb = dist_base(dd, y0, x0 + lane, 0u);
#pragma unroll
    for (int y = 0; y < TILE; ++y) d[y] = (lane < vw && y < vh) ? ld_dist_at(lb, dd.dist_pitch, y) : INF;
  }

  if (!rerun && !tma_wait(&sm.bar, parity, 1u, sch.q, tile)) return;

  // Padded copies of the image box, one line per tile row and one per tile column (position -1..32 at byte
  // pos + 1): pimg line r = box row r (tile row r - 1), pimgT line c = tile column c - 1.  In either layout
  // lane l needs lines l, l + 1, l + 2 (its own line and the two beside it) of one of them.  A re-run has them.
  uint8_t* pimg = reinterpret_cast<uint8_t*>(sm.Wh + 96);    // 34 * 36 = 1224 bytes after the halo rows
  uint8_t* pimgT = reinterpret_cast<uint8_t*>(sm.Wh + 416);  // 1224 bytes after pimg
  for (int i = lane; !rerun && i < IMG_BOX_ROWS * PIMG_STRIDE; i += 32) {
    const int r = i / PIMG_STRIDE, c = i % PIMG_STRIDE;
    const uint8_t px = (c < TILE + 2) ? sm.img[r * IMG_BOX_GRAY + 15 + c] : 0;
    pimg[i] = px;
    if (c < TILE + 2) pimgT[c * PIMG_STRIDE + r] = px;
  }

  if (first) {
#pragma unroll
    for (int y = 0; y < TILE; ++y) {
      const bool in = lane < vw && y < vh;
      d[y] = in ? ((seed && mask_box(sm)[y * TILE + lane] != 0) ? 0.0f : v) : INF;
    }
  } else if (seed) {
#pragma unroll
    for (int y = 0; y < TILE; ++y)
      if (lane < vw && y < vh && mask_box(sm)[y * TILE + lane] != 0) d[y] = 0.0f;
  }
  __syncwarp();

  // From here on the image is needed through pimg only; T holds the tile.
  // Initial border values for the change test, kept in shared memory through the phases (registers are the
  // scarce resource there): top, bottom, left, right at border0[32 * side + lane].
  float* border0 = sm.Wv + 352;  // after the halo columns
  border0[lane] = d[0];
  border0[32 + lane] = d[TILE - 1];
#pragma unroll
  for (int y = 0; y < TILE; ++y) T[y * S_STRIDE + lane] = d[y];
  __syncwarp();
  border0[64 + lane] = T[lane * S_STRIDE];
  border0[96 + lane] = T[lane * S_STRIDE + TILE - 1];
  __syncwarp();

  auto P = [&](int r, int c) -> float {  // pixel at tile (c, r) as float, r, c in [-1, 32]
    return (float)pimg[(r + 1) * PIMG_STRIDE + c + 1];
  };
  auto absd = [](float a, float b) { return fabsf(a - b); };  // exact for integers in [0, 255]

  // Bucket width of this image (priority queue): half a tile-width of the mean axial edge cost
  // l_eucl + l_grad * |dI| seen by first visits (vertical edges of the tile).
  float inv_width = 0.0f;
  if (sch.q.wacc) {
    float* wa = sch.q.wacc + 2 * (old_state >> ST_IMG_SHIFT);
    if (first) {
      float wsum = 0.0f, wcnt = 0.0f;
      if (lane < vw) {
#pragma unroll 1
        for (int y = 1; y < vh; ++y) {
          wsum += le + lg * absd(P(y, lane), P(y - 1, lane));
          wcnt += 1.0f;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        wsum += __shfl_xor_sync(~0u, wsum, o);
        wcnt += __shfl_xor_sync(~0u, wcnt, o);
      }
      if (lane == 0 && wcnt > 0.0f) {
        atomicAdd(&wa[0], wsum);
        atomicAdd(&wa[1], wcnt);
      }
    }
    const float s_ = *(volatile float*)&wa[0], c_ = *(volatile float*)&wa[1];
    const float bt = sch.q.bucket_tiles;
    inv_width = (c_ > 0.0f && s_ > 0.0f) ? c_ / (bt * (float)TILE * s_) : 1.0f / (bt * (float)TILE);
  }

  bool any = false;
  uint32_t nph = 0;
  bool col = true;
  for (;;) {
    bool ch = false;
    // One code path for both layouts.  Column phase (lane = x, position k = y): forward over y from the three
    // predecessors (x-1..x+1, y-1), backward from (x-1..x+1, y+1).  Row phase (lane = y, k = x): forward over x
    // from (x-1, y-1..y+1), backward from (x+1, y-1..y+1).  Lanes l-1 / l+1 hold the diagonal predecessors (by
    // shuffle); the edge lanes take them from the halo beside the tile (`side_lo` / `side_hi`), and position
    // -1 / 32 from the halo across the chain (`lo` / `hi`).  The lane's image lines (its own and the two beside
    // it) are loaded once per phase.  The forward and the backward chain are interleaved (two independent
    // dependency chains per warp); every step is the same single-edge relaxation as in the reference passes,
    // so the order does not change the fixpoint.
    const float* lo = col ? ht : hl;
    const float* hi = col ? hb : hr;
    const float* side_lo = col ? hl : ht;
    const float* side_hi = col ? hr : hb;
    const bool lane_in = lane < (col ? vw : vh);
    const int kmax = col ? vh : vw;
    uint32_t L0[9], L1[9], L2[9];
    {
      const uint32_t* w = reinterpret_cast<const uint32_t*>((col ? pimgT : pimg) + lane * PIMG_STRIDE);
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        L0[j] = w[j];
        L1[j] = w[9 + j];
        L2[j] = w[18 + j];
      }
    }
#pragma unroll
    for (int k = 0; k < TILE; ++k) {
      {
        float pa, pb, pc;
        if (k == 0) { pa = lo[lane]; pb = lo[lane + 1]; pc = lo[lane + 2]; }
        else {
          pb = d[k - 1];
          pa = __shfl_up_sync(~0u, pb, 1);
          pc = __shfl_down_sync(~0u, pb, 1);
          if (lane == 0) pa = side_lo[k];
          if (lane == TILE - 1) pc = side_hi[k];
        }
        const float c = line_px(L1, k);
        const float nd = ref_min3<FMA>(d[k], pa, pb, pc, le, lg, sq2, absd(c, line_px(L0, k - 1)),
                                       absd(c, line_px(L1, k - 1)), absd(c, line_px(L2, k - 1)), true, true);
        const bool upd = lane_in && k < kmax && nd < d[k];
        ch |= upd;
        d[k] = upd ? nd : d[k];
      }
      {
        const int j = TILE - 1 - k;
        float pa, pb, pc;
        if (j == TILE - 1) { pa = hi[lane]; pb = hi[lane + 1]; pc = hi[lane + 2]; }
        else {
          pb = d[j + 1];
          pa = __shfl_up_sync(~0u, pb, 1);
          pc = __shfl_down_sync(~0u, pb, 1);
          if (lane == 0) pa = side_lo[j + 2];
          if (lane == TILE - 1) pc = side_hi[j + 2];
        }
        const float c = line_px(L1, j);
        const float nd = ref_min3<FMA>(d[j], pa, pb, pc, le, lg, sq2, absd(c, line_px(L0, j + 1)),
                                       absd(c, line_px(L1, j + 1)), absd(c, line_px(L2, j + 1)), true, true);
        const bool upd = lane_in && j < kmax && nd < d[j];
        ch |= upd;
        d[j] = upd ? nd : d[j];
      }
    }
    ch = __any_sync(~0u, ch);
    any |= ch;
    ++nph;
    if (col) {
#pragma unroll
      for (int y = 0; y < TILE; ++y) T[y * S_STRIDE + lane] = d[y];
    } else {
#pragma unroll
      for (int x = 0; x < TILE; ++x) T[lane * S_STRIDE + x] = d[x];
    }
    __syncwarp();
    if ((!ch && nph >= 2) || nph >= (uint32_t)PHASE_LIMIT) break;
    if (col) {
#pragma unroll
      for (int x = 0; x < TILE; ++x) d[x] = T[lane * S_STRIDE + x];
    } else {
#pragma unroll
      for (int y = 0; y < TILE; ++y) d[y] = T[y * S_STRIDE + lane];
    }
    col = !col;
    __syncwarp();
  }
  if (nph >= (uint32_t)PHASE_LIMIT && lane == 0) set_error(sch.q, DERR_PHASE_LIMIT, tile);

  // Border changes -> neighbours (bit k = neighbour k as in ndx_l / ndy_l), as the reference activates blocks
  // (dt_block_passes.cuh:50-63).  An exact "can this border lower the neighbour's halo" test (as in ns-mode)
  // removed only a tenth of the visits here and cost more than it saved: most re-visits in ref-mode carry
  // last-bit improvements of equally long paths summed in another order, which that test also lets through.
  // The activation's priority is the smallest border value facing the neighbour.
  uint32_t act = 0;
  float key = 0.0f;
  if (any || seed) {
    const bool force = seed;
    const float bt = T[lane], bb = T[(TILE - 1) * S_STRIDE + lane];
    const float bl = T[lane * S_STRIDE], br = T[lane * S_STRIDE + TILE - 1];
    const uint32_t ct = __ballot_sync(~0u, force || bt != border0[lane]);
    const uint32_t cb = __ballot_sync(~0u, force || bb != border0[32 + lane]);
    const uint32_t cl = __ballot_sync(~0u, force || bl != border0[64 + lane]);
    const uint32_t cr = __ballot_sync(~0u, force || br != border0[96 + lane]);
    act |= cl ? 1u : 0u;
    act |= cr ? 2u : 0u;
    act |= ct ? 4u : 0u;
    act |= cb ? 8u : 0u;
    act |= (ct & 1u) ? 16u : 0u;
    act |= (ct >> (TILE - 1)) & 1u ? 32u : 0u;
    act |= (cb & 1u) ? 64u : 0u;
    act |= (cb >> (TILE - 1)) & 1u ? 128u : 0u;
    act &= nexist;
    if (act) {
      const uint32_t kl = __reduce_min_sync(~0u, __float_as_uint(bl));
      const uint32_t kr = __reduce_min_sync(~0u, __float_as_uint(br));
      const uint32_t kt = __reduce_min_sync(~0u, __float_as_uint(bt));
      const uint32_t kb = __reduce_min_sync(~0u, __float_as_uint(bb));
      const float corner = lane == 4 ? T[0] : lane == 5 ? T[TILE - 1] : lane == 6 ? T[(TILE - 1) * S_STRIDE]
                                                                                    : T[(TILE - 1) * S_STRIDE + TILE - 1];
      key = lane == 0 ? __uint_as_float(kl) : lane == 1 ? __uint_as_float(kr) : lane == 2 ? __uint_as_float(kt)
          : lane == 3 ? __uint_as_float(kb) : corner;
    }
  }

  if (any || first) {
    if (lane < vw) {
      uint8_t* wb = dist_base(dd, y0, x0 + lane, nph);
#pragma unroll
      for (int y = 0; y < TILE; ++y)
        if (y < vh) *reinterpret_cast<float*>(wb + (int64_t)y * dd.dist_pitch) = T[y * S_STRIDE + lane];
    }
  }
  fence_acq_rel();
  __syncwarp();
  const bool want = lane < 8 && ((act >> lane) & 1u);
  const uint32_t item = want ? dd.tile_base + (uint32_t)((ty + ndy_l) * dd.tiles_x + tx + ndx_l) : 0u;
  sch.complete(tile, (first ? ST_VISITED : 0u) | (seed ? ST_SEED : 0u), want, item, key, inv_width);
  *nph_out = nph;
  *nact_out = (uint32_t)__popc(act);
}

// MODE is fixed per kernel instantiation: a launch covers images of one weight mode (and, in ref-mode, one
// rounding) only, so no kernel's register allocation is inflated by another mode's code.
template <int MODE, class Sched>
__device__ __forceinline__ void visit_tile(const ImgDesc& dd, const CUtensorMap* tmaps, uint32_t img, uint32_t tile,
                                           uint32_t old_state, WarpSmem& sm, uint32_t& parity, const Sched& sch,
                                           WarpStats& ws, bool rerun = false) {
  const CUtensorMap* tm_img = tmaps + 2 * img;
  const CUtensorMap* tm_mask = tmaps + 2 * img + 1;
  uint32_t nph, nact;
  if (MODE == MODE_NS)
    visit_ns<false>(dd, tm_img, tm_mask, tile, old_state, visit_bufs(sm, parity), sch, &nph, &nact, rerun);
  else if (MODE == MODE_REF)
    visit_ref<true>(dd, tm_img, tm_mask, tile, old_state, sm, parity, sch, &nph, &nact, rerun);
  else
    visit_ref<false>(dd, tm_img, tm_mask, tile, old_state, sm, parity, sch, &nph, &nact, rerun);
  count_visit(ws, sch.q, nph, nact);
}

__device__ __forceinline__ WarpSmem& warp_slot(uint8_t* smem_raw) {
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  return reinterpret_cast<WarpSmem*>(base)[threadIdx.x >> 5];
}

__device__ __forceinline__ void warp_slot_init(WarpSmem& sm) {
  if ((threadIdx.x & 31) == 0) {
    mbar_init(&sm.bar, 1);
    fence_mbar_init();
  }
  __syncwarp();
}

__device__ __forceinline__ WarpSmemP& warp_slot_p(uint8_t* smem_raw) {
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  return reinterpret_cast<WarpSmemP*>(base)[threadIdx.x >> 5];
}

__device__ __forceinline__ void warp_slot_init(WarpSmemP& sm) {
  if ((threadIdx.x & 31) == 0) {
    mbar_init(&sm.bar[0], 1);
    mbar_init(&sm.bar[1], 1);
    mbar_init(&sm.mbar, 1);
    fence_mbar_init();
  }
  __syncwarp();
}

// Image of a global tile id: binary search over the prefix array tile_base[0..n].
__device__ __forceinline__ uint32_t image_of_tile(const uint32_t* tile_base, int n, uint32_t t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_base[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return (uint32_t)lo;
}

}  // namespace dtb
