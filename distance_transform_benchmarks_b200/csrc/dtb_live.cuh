// dtb_live.cuh -- the live tile kernel of the serving engine: requests join the tile queue of a kernel that is
// already running.
//
// The wave engine (dtb_serve.cu) runs one persistent launch per wave, so a request that arrives while a wave
// runs waits for that launch to end.  Here one persistent kernel stays resident while requests flow: the host
// publishes each request into a device ring (its image, mask, descriptor and tensor maps are copied in first,
// on the same stream, so a published entry's data is complete), idle warps of the running kernel notice the
// published counter move, one of them claims the entry and turns it into work in the same tile queue the other
// requests' tiles are in:
//   new image   set-up jobs, each a band of whole tile rows (about LIVE_JOB_TILES tiles): pass 1 moves rows
//               the host staged packed into their pitched planes and writes the tile states (image slot, SEED
//               from a scan of the mask tile), pass 2 -- once every pass-1 job of the image has ended, so that no
//               activation can meet an uninitialised state and no visit a plane row not yet in place -- queues
//               the seed tiles;
//   seed edit   the claiming warp draws the disks into the resident mask and queues the tiles they touch; the
//               tiles keep VISITED and their map, which is the warm start (added seeds only lower distances).
// Each image slot counts its request's queued and running items; the warp whose completion brings the count to
// zero writes v into the tiles never reached and then the entry's completion word into host-mapped memory,
// which the host polls before it copies the map out.  So requests are admitted while others run, and their
// tiles share the warps tile by tile.
//
// Queue: one FIFO ring (the bucketed rings' ticket give-backs would move heads ahead of tails for as long as
// the kernel lives); a waiting warp keeps its ticket while it admits an entry.  Termination: the kernel ends
// when nothing is queued or running and the host asked it to stop, no request was claimed or completed for
// `idle_us`, or it has run for `life_us` (after which it claims nothing new and drains); ending is one CAS of
// the pending word from 0 to LIVE_EXIT, which an admission checks before it claims, so no entry is claimed by
// a kernel that is ending.  Unclaimed entries are claimed by the next launch.  Every wait is bounded: a
// no-progress watchdog (while work is pending) ends the kernel with an error code.
#pragma once

#include "dtb_kernels.cuh"

namespace dtb {

constexpr uint32_t LIVE_RING = 4096;          // request entries (power of two); at most LIVE_RING / 2 in flight
constexpr uint32_t LIVE_JOB_TILES = 64;       // tiles per set-up job (whole tile rows, at least one)
constexpr uint32_t LIVE_JOB = 1u << 30;       // queue item: a set-up job (tile ids stay below 2^29)
constexpr uint32_t LIVE_JOB_PASS2 = 1u << 29; // set-up job, second pass (queue the seed tiles)
constexpr int LIVE_CHUNK_BITS = 15;           // set-up jobs per pass < 32768 (tile rows < 32768)
constexpr int LIVE_SLOT_BITS = 14;            // image slots < 16384
constexpr uint32_t LIVE_MAX_SLOTS = 1u << LIVE_SLOT_BITS;
constexpr uint32_t LIVE_MAX_TILES = 1u << 29; // tile ids of the live tile space
constexpr uint32_t LIVE_EXIT = 0x80000000u;   // pending word of a kernel that is ending
constexpr uint32_t LIVE_ADMIT = 0xFFFFFFFCu;  // pop result: a published entry waits to be claimed
constexpr uint32_t LIVE_END = 0xFFFFFFFBu;    // pop result (one lane): this warp ended the kernel
constexpr uint32_t DERR_LIVE_ENTRY = 7;       // a claimed entry named a slot or image outside the server's tables

enum : uint32_t { LIVE_NEW = 0u, LIVE_EDIT = 1u };

// One request as the host publishes it.
struct alignas(32) LiveEntry {
  uint32_t kind;     // LIVE_NEW / LIVE_EDIT
  uint32_t slot;     // image slot: descriptor, tensor maps and counters
  uint32_t n_disks;  // edit: disks (cx, cy, r, 0: 16-byte records) at disks[4 * disk_idx ..]
  uint32_t disk_idx;
  uint32_t stage;    // new image: LIVE_STAGE_* flags
  uint32_t pad[3];
};

// Host <-> kernel words in device memory, kept across launches (the queue header is reset per launch).
struct LiveHdr {
  Line published;   // entries published (host copy after the entry's data)
  Line claimed;     // entries claimed
  Line stop;        // host: end once idle
  Line inject;      // failure self-test: the next claimed request counts one item that never runs
  Line last_busy;   // low 32 bits of the globaltimer (us) of the last claim or completion
  Line watch_ms;    // no-progress limit of the watchdog (ms)
  Line end_reason;  // why the last launch ended: LIVE_END_STOP / _IDLE / _LIFE (0: an error, or still running)
};
constexpr uint32_t LIVE_END_STOP = 1u, LIVE_END_IDLE = 2u, LIVE_END_LIFE = 3u;

// Per image slot.
struct LiveSlot {
  uint32_t pending;     // set-up jobs and tiles of the slot's request queued or running, + 1 while admitting
  uint32_t entry;       // entry index of that request
  uint32_t setup_left;  // pass-1 set-up jobs not yet ended
  uint32_t stage;       // new image: LIVE_STAGE_* planes staged packed in its distance plane
};

// A new image's planes whose rows need a new pitch are copied in packed, into the image's own distance plane
// (not written before the set-up ends; at least (channels + 1) bytes a pixel): the image at its start, the mask
// after it, 16-byte aligned.  Pass-1 set-up jobs move the rows into place.
constexpr uint32_t LIVE_STAGE_IMG = 1u, LIVE_STAGE_MASK = 2u;
constexpr uint64_t LIVE_STAGE_SLACK = 64;  // bytes the staging leaves free at the end of the distance plane
__host__ __device__ __forceinline__ uint64_t live_stage_mask_offset(uint32_t rb, uint32_t h) {
  return ((uint64_t)rb * h + 15u) & ~uint64_t(15);
}

struct LiveArgs {
  Queue q;                    // one FIFO ring; total_tiles = size of the tile space
  uint32_t* states;           // per tile of the tile space
  const ImgDesc* descs;       // per slot (tile_base = the image's first tile id)
  const CUtensorMap* tmaps;   // 2 per slot
  LiveHdr* lh;
  LiveSlot* slots;
  const LiveEntry* entries;   // LIVE_RING
  const int32_t* disks;
  uint32_t* host_done;        // mapped host memory, LIVE_RING words: entry index + 1 once its map is final
  uint32_t nslots;
  uint32_t disk_cap;          // disks in the pool
  uint32_t idle_us, life_us;
};

__device__ __forceinline__ uint32_t now_us() { return (uint32_t)(globaltimer() / 1000ull); }

// Descriptor of a slot, read through L2: the host rewrites a slot's descriptor while the kernel runs, so a
// stale L1 line of the slot's previous image must never be used.
__device__ __forceinline__ ImgDesc load_desc(const ImgDesc* p) {
  ImgDesc d;
  const uint4* s = reinterpret_cast<const uint4*>(p);
  uint4* o = reinterpret_cast<uint4*>(&d);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(ImgDesc) / 16); ++k) o[k] = __ldcg(s + k);
  return d;
}

// Tile rows of one set-up job: whole tile rows, about LIVE_JOB_TILES tiles.
__device__ __forceinline__ uint32_t live_band(const ImgDesc& dd) {
  return max(1u, LIVE_JOB_TILES / (uint32_t)max(dd.tiles_x, 1));
}

// Item pushes of the live kernel: the caller has already counted them in `pending` (global and slot).
__device__ __forceinline__ void live_push(const Queue& q, uint32_t item) {
  slot_write(q, 0u, atomicAdd(&q.hdr->tails[0].v, 1u), item);
}

// Request end (whole warp): v into the tiles never reached, then the completion word for the host.
__device__ void live_finish(const LiveArgs& a, uint32_t slot) {
  const int lane = threadIdx.x & 31;
  __threadfence();  // acquire: the visits and set-up jobs counted down before us
  const ImgDesc dd = load_desc(a.descs + slot);
  const uint32_t tiles = (uint32_t)dd.tiles_x * (uint32_t)dd.tiles_y;
  for (uint32_t t0 = 0; t0 < tiles; t0 += 32) {
    const uint32_t t = t0 + (uint32_t)lane;
    bool unreached = false;
    if (t < tiles) unreached = !(ld_volatile(&a.states[dd.tile_base + t]) & ST_VISITED);
    uint32_t m = __ballot_sync(~0u, unreached);
    while (m) {
      const uint32_t local = t0 + (uint32_t)(__ffs(m) - 1);
      m &= m - 1u;
      const int x0 = (int)(local % (uint32_t)dd.tiles_x) * TILE, y0 = (int)(local / (uint32_t)dd.tiles_x) * TILE;
      const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
      if (lane < vw)
        for (int y = 0; y < vh; ++y) dist_row(dd, y0 + y)[x0 + lane] = dd.v;
    }
  }
  __threadfence_system();  // the map before the completion word the host acts on
  __syncwarp();
  if (lane == 0) {
    const uint32_t e = ld_volatile(&a.slots[slot].entry);
    atomicExch(&a.lh->last_busy.v, now_us());
    *(volatile uint32_t*)&a.host_done[e & (LIVE_RING - 1u)] = e + 1u;
  }
  __syncwarp();
}

// Ends one queued or running item of a slot's request (lane 0 only); true if it was the request's last.
__device__ __forceinline__ bool live_item_done(const LiveArgs& a, uint32_t slot) {
  atomicSub(&a.q.hdr->pending.v, 1u);
  return atomicSub(&a.slots[slot].pending, 1u) == 1u;
}

// The scheduler of the tile visit: as QueueSched::complete, plus the slot's count of its request's items.
struct LiveSched {
  Queue q;
  uint32_t* states;
  const LiveArgs* a;
  // The warp's word for its own tile when its halo dropped during the visit: the warp re-runs it next from the
  // weights and distances in its shared memory (neighbour tiles always go through the ring, so that warps come
  // back to the queue, where new requests are claimed).
  uint32_t* keep_out;
  __device__ __forceinline__ void complete(uint32_t tile, uint32_t xor_bits, bool want, uint32_t want_item,
                                           float = 0.0f, float = 0.0f) const {
    const int lane = threadIdx.x & 31;
    bool push = false;
    uint32_t item = 0, slot = 0;
    if (lane == 31) {
      const uint32_t old = atomicXor(&states[tile], xor_bits | ST_RUNNING);
      push = (old & ST_PENDING) != 0u;
      item = tile;
      slot = old >> ST_IMG_SHIFT;
      if (xor_bits & ST_VISITED) __threadfence();
    }
    slot = __shfl_sync(~0u, slot, 31);
    __syncwarp();
    if (want) {
      if (want_item >= q.total_tiles) {
        set_error(q, DERR_BAD_TILE, want_item);
      } else {
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
        last = live_item_done(*a, slot) ? 1u : 0u;
      } else if (k > 1) {
        atomicAdd(&q.hdr->pending.v, k - 1u);
        atomicAdd(&a->slots[slot].pending, k - 1u);
      }
      __threadfence();
    }
    __syncwarp();
    const bool keep_own = (m >> 31) != 0u;  // lane 31 re-queues the own tile (activations are lanes 0-3)
    if (lane == 31 && keep_own) *keep_out = item;
    if (push && !(lane == 31 && keep_own)) live_push(q, item);
    __syncwarp();
    if (__shfl_sync(~0u, last, 0)) live_finish(*a, slot);
  }
};

// Whether this kernel may still claim entries (not stopping, no error, within its lifetime).
__device__ __forceinline__ bool live_may_claim(const LiveArgs& a, uint32_t t_start) {
  return (ld_volatile(&a.lh->stop.v) | ld_volatile(&a.q.hdr->error.v)) == 0u && now_us() - t_start < a.life_us;
}

// Claims one published entry and queues its work (whole warp).  Returns whether an entry was claimed.
__device__ bool live_admit(const LiveArgs& a, uint32_t t_start) {
  const int lane = threadIdx.x & 31;
  const Queue& q = a.q;
  uint32_t e = 0, ok = 0;
  if (lane == 0 && live_may_claim(a, t_start)) {
    const uint32_t c = ld_volatile(&a.lh->claimed.v);
    if (c != ld_volatile(&a.lh->published.v)) {
      // Count this admission in `pending` before claiming: a kernel that is ending has set LIVE_EXIT there.
      const uint32_t old = atomicAdd(&q.hdr->pending.v, 1u);
      if (!(old & LIVE_EXIT)) {
        if (atomicCAS(&a.lh->claimed.v, c, c + 1u) == c) {
          ok = 1;
          e = c;
        } else {
          atomicSub(&q.hdr->pending.v, 1u);
        }
      }
    }
  }
  ok = __shfl_sync(~0u, ok, 0);
  if (!ok) return false;
  e = __shfl_sync(~0u, e, 0);
  __threadfence();  // acquire: the entry and its data were copied in before the published counter
  const LiveEntry* pe = a.entries + (e & (LIVE_RING - 1u));
  const uint4 w0 = __ldcg(reinterpret_cast<const uint4*>(pe));
  const uint32_t kind = w0.x, slot = w0.y, nd = w0.z, di = w0.w;
  if (slot >= a.nslots || (kind == LIVE_EDIT && ((uint64_t)di + nd > a.disk_cap))) {
    if (lane == 0) {
      set_error(q, DERR_LIVE_ENTRY, e);
      atomicSub(&q.hdr->pending.v, 1u);
    }
    return true;
  }
  const ImgDesc dd = load_desc(a.descs + slot);
  LiveSlot* ls = a.slots + slot;
  uint32_t phantom = 0;
  if (lane == 0) {
    ls->entry = e;
    ls->pending = 1u;  // held by this admission until its items are queued
    atomicExch(&a.lh->last_busy.v, now_us());
    phantom = atomicExch(&a.lh->inject.v, 0u);
    if (phantom) {  // failure self-test: one item of this request never runs
      atomicAdd(&q.hdr->pending.v, 1u);
      atomicAdd(&ls->pending, 1u);
    }
  }
  const uint32_t tiles = (uint32_t)dd.tiles_x * (uint32_t)dd.tiles_y;
  if (kind == LIVE_NEW) {
    const uint32_t band = live_band(dd);
    const uint32_t njobs = tiles ? ((uint32_t)dd.tiles_y + band - 1u) / band : 0u;
    if (lane == 0 && njobs) {
      ls->stage = __ldcg(&pe->stage);
      ls->setup_left = njobs;
      if (q.wacc) { q.wacc[2 * slot] = 0.0f; q.wacc[2 * slot + 1] = 0.0f; }
      atomicAdd(&q.hdr->pending.v, njobs);
      atomicAdd(&ls->pending, njobs);
      __threadfence();
    }
    __syncwarp();
    for (uint32_t j = (uint32_t)lane; j < njobs; j += 32u) live_push(q, LIVE_JOB | (slot << LIVE_CHUNK_BITS) | j);
  } else {
    // Draw the disks into the resident mask (the same pixels as serve_draw_disks).
    uint8_t* mask = const_cast<uint8_t*>(dd.mask);
    for (uint32_t k = 0; k < nd; ++k) {
      const int4 dk = __ldcg(reinterpret_cast<const int4*>(a.disks) + (di + k));
      const int cx = dk.x, cy = dk.y, r = dk.z;
      const int xa = max(0, cx - r), xb = min(dd.width - 1, cx + r), ya = max(0, cy - r), yb = min(dd.height - 1, cy + r);
      if (xa > xb || ya > yb) continue;
      const int bw = xb - xa + 1, cnt = bw * (yb - ya + 1);
      for (int i = lane; i < cnt; i += 32) {
        const int x = xa + i % bw, y = ya + i / bw, ddx = x - cx, ddy = y - cy;
        if (ddx * ddx + ddy * ddy <= r * r) mask[(int64_t)y * dd.mask_pitch + x] = 1;
      }
    }
    // The mask bytes before the tiles that read them by bulk copy (async proxy) are queued.
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __threadfence();
    __syncwarp();
    // Queue the tiles the disks touch (as serve_seed_tiles); the image has no other request in flight, so every
    // tile is idle: VISITED with its map, or never reached, holding v, where its first visit starts from v too.
    for (uint32_t k = 0; k < nd; ++k) {
      const int4 dk = __ldcg(reinterpret_cast<const int4*>(a.disks) + (di + k));
      const int cx = dk.x, cy = dk.y, r = dk.z;
      const int xa = max(0, cx - r), xb = min(dd.width - 1, cx + r), ya = max(0, cy - r), yb = min(dd.height - 1, cy + r);
      if (xa > xb || ya > yb) continue;
      const int txa = xa / TILE, txb = xb / TILE, tya = ya / TILE, tyb = yb / TILE;
      const int ntx = txb - txa + 1, cnt = ntx * (tyb - tya + 1);
      for (int i0 = 0; i0 < cnt; i0 += 32) {
        const int i = i0 + lane;
        bool push = false;
        uint32_t t = 0;
        if (i < cnt) {
          t = dd.tile_base + (uint32_t)((tya + i / ntx) * dd.tiles_x + txa + i % ntx);
          const uint32_t old = atomicOr(&a.states[t], ST_SEED | ST_PENDING);
          push = !(old & (ST_PENDING | ST_RUNNING));
        }
        const uint32_t n = __popc(__ballot_sync(~0u, push));
        if (lane == 0 && n) {
          atomicAdd(&q.hdr->pending.v, n);
          atomicAdd(&ls->pending, n);
          __threadfence();
        }
        __syncwarp();
        if (push) live_push(q, t);
      }
    }
  }
  // Release the admission's hold on the slot and its own count in `pending`.
  uint32_t last = 0;
  if (lane == 0) last = live_item_done(a, slot) ? 1u : 0u;
  if (__shfl_sync(~0u, last, 0)) live_finish(a, slot);
  (void)phantom;
  return true;
}

// Rows [y0, y1) of a plane copied packed (row r at src + r * rb) into its pitched place (row r at dst + r *
// pitch), as 16-byte chunks of the destination: the destination rows are 128-byte aligned, the packed source
// rows only byte aligned, so a chunk is five aligned 4-byte source words funnel-shifted by the row's byte
// offset (the same for every chunk of a row).  Each lane keeps four chunks' loads in flight.  A row's last
// chunk may carry up to 15 bytes past the row into the pitch padding, and the loads may read up to 19 bytes past
// the packed data: the host leaves LIVE_STAGE_SLACK bytes free.  The source was written by a host copy into
// memory whose earlier contents this SM may have cached, so the loads go through L2.
__device__ __forceinline__ void live_repitch(const uint8_t* src, uint8_t* dst, int64_t pitch, uint32_t rb, int y0, int y1) {
  const int lane = threadIdx.x & 31;
  const uint32_t chunks = (rb + 15u) / 16u;
  for (int y = y0; y < y1; ++y) {
    const uintptr_t sa = reinterpret_cast<uintptr_t>(src) + (uintptr_t)y * rb;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(sa & ~uintptr_t(3));
    const uint32_t sh = (uint32_t)(sa & 3u) * 8u;
    uint4* d = reinterpret_cast<uint4*>(dst + (int64_t)y * pitch);
    for (uint32_t c0 = (uint32_t)lane; c0 < chunks; c0 += 32u * 4u) {
      uint32_t v[4][5];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t c = c0 + 32u * (uint32_t)u;
#pragma unroll
        for (int j = 0; j < 5; ++j) v[u][j] = c < chunks ? __ldcg(w + 4u * c + (uint32_t)j) : 0u;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t c = c0 + 32u * (uint32_t)u;
        if (c < chunks)
          d[c] = make_uint4(__funnelshift_r(v[u][0], v[u][1], sh), __funnelshift_r(v[u][1], v[u][2], sh),
                            __funnelshift_r(v[u][2], v[u][3], sh), __funnelshift_r(v[u][3], v[u][4], sh));
      }
    }
  }
}

// One set-up job of a new image (whole warp): a band of whole tile rows.
__device__ void live_job(const LiveArgs& a, uint32_t item) {
  const int lane = threadIdx.x & 31;
  const Queue& q = a.q;
  const uint32_t slot = (item >> LIVE_CHUNK_BITS) & (LIVE_MAX_SLOTS - 1u);
  const uint32_t chunk = item & ((1u << LIVE_CHUNK_BITS) - 1u);
  const bool pass2 = (item & LIVE_JOB_PASS2) != 0u;
  const ImgDesc dd = load_desc(a.descs + slot);
  const uint32_t band = live_band(dd);
  const uint32_t ty0 = chunk * band, ty1 = min(ty0 + band, (uint32_t)dd.tiles_y);
  const uint32_t t0 = ty0 * (uint32_t)dd.tiles_x, t1 = ty1 * (uint32_t)dd.tiles_x;
  LiveSlot* ls = a.slots + slot;
  if (!pass2) {
    // Rows of the band staged packed in the distance plane move into their pitched planes first (the host
    // copied them as one 1-D copy each: a copy that changes the pitch runs at a fraction of the link's rate).
    const uint32_t stage = ld_volatile(&ls->stage);
    if (stage) {
      const int y0 = (int)ty0 * TILE, y1 = min((int)ty1 * TILE, dd.height);
      const uint32_t rb = (uint32_t)dd.width * (uint32_t)dd.channels;
      const uint8_t* st = reinterpret_cast<const uint8_t*>(dd.dist);
      if (stage & LIVE_STAGE_IMG) live_repitch(st, const_cast<uint8_t*>(dd.img), dd.img_pitch, rb, y0, y1);
      if (stage & LIVE_STAGE_MASK)
        live_repitch(st + ((stage & LIVE_STAGE_IMG) ? live_stage_mask_offset(rb, (uint32_t)dd.height) : 0),
                     const_cast<uint8_t*>(dd.mask), dd.mask_pitch, (uint32_t)dd.width, y0, y1);
      // The planes are read by bulk copies (async proxy) in the visits.
      asm volatile("fence.proxy.async.global;" ::: "memory");
      __threadfence();
      __syncwarp();
    }
    // States of the band: the slot, and SEED where the mask tile holds a seed (lane = row of the tile; four
    // tiles' loads in flight at once).
    for (uint32_t tb = t0; tb < t1; tb += 4u) {
      bool nz[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t t = tb + (uint32_t)u;
        nz[u] = false;
        if (t < t1) {
          const int x0 = (int)(t % (uint32_t)dd.tiles_x) * TILE, y0 = (int)(t / (uint32_t)dd.tiles_x) * TILE;
          const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
          if (lane < vh) {
            const uint8_t* row = dd.mask + (int64_t)(y0 + lane) * dd.mask_pitch + x0;
            if (vw == TILE && (reinterpret_cast<uintptr_t>(row) & 15u) == 0) {
              const uint4 p = __ldcg(reinterpret_cast<const uint4*>(row));
              const uint4 r = __ldcg(reinterpret_cast<const uint4*>(row) + 1);
              nz[u] = (p.x | p.y | p.z | p.w | r.x | r.y | r.z | r.w) != 0u;
            } else {
              for (int c = 0; c < vw; ++c) nz[u] |= __ldcg(row + c) != 0;
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool any = __any_sync(~0u, nz[u]);
        if (lane == 0 && tb + (uint32_t)u < t1) a.states[dd.tile_base + tb + u] = (slot << ST_IMG_SHIFT) | (any ? ST_SEED : 0u);
      }
    }
    __threadfence();
    __syncwarp();
    uint32_t all = 0;
    if (lane == 0) all = atomicSub(&ls->setup_left, 1u) == 1u ? 1u : 0u;
    if (__shfl_sync(~0u, all, 0)) {
      // Every state and plane row of the image is written: queue the second pass.
      const uint32_t njobs = ((uint32_t)dd.tiles_y + band - 1u) / band;
      if (lane == 0) {
        atomicAdd(&q.hdr->pending.v, njobs);
        atomicAdd(&ls->pending, njobs);
        __threadfence();
      }
      __syncwarp();
      for (uint32_t j = (uint32_t)lane; j < njobs; j += 32u)
        live_push(q, LIVE_JOB | LIVE_JOB_PASS2 | (slot << LIVE_CHUNK_BITS) | j);
    }
  } else {
    // Queue the seed tiles of the band.  A tile an activation has queued or visited meanwhile is left alone
    // (its visit applies or applied the seeds); a visited one queued again only costs a converged visit.
    for (uint32_t tb = t0; tb < t1; tb += 32u) {
      const uint32_t t = tb + (uint32_t)lane;
      bool push = false;
      if (t < t1 && (ld_volatile(&a.states[dd.tile_base + t]) & ST_SEED)) {
        const uint32_t old = atomicOr(&a.states[dd.tile_base + t], ST_PENDING);
        push = !(old & (ST_PENDING | ST_RUNNING));
      }
      const uint32_t n = __popc(__ballot_sync(~0u, push));
      if (lane == 0 && n) {
        atomicAdd(&q.hdr->pending.v, n);
        atomicAdd(&ls->pending, n);
        __threadfence();
      }
      __syncwarp();
      if (push) live_push(q, dd.tile_base + t);
    }
  }
  uint32_t last = 0;
  if (lane == 0) last = live_item_done(a, slot) ? 1u : 0u;
  if (__shfl_sync(~0u, last, 0)) live_finish(a, slot);
}

// Waits for the item of ticket h (lane 0).  Returns the item, POP_NONE (the kernel ends), LIVE_ADMIT (an entry
// waits to be claimed: the warp claims it and comes back to the same ticket) or LIVE_END (this lane ended the
// kernel; the warp wakes every waiter).
__device__ __forceinline__ uint32_t live_take(const LiveArgs& a, uint32_t h, PopWatch& w, uint32_t t_start) {
  const Queue& q = a.q;
  uint32_t* slot = ring_slot(q, 0u, h);
  uint32_t ns = 32;
  uint64_t t_check = globaltimer();
  for (;;) {
    const uint32_t cur = ld_volatile(slot);
    if (cur != 0u) {
      const uint32_t v = atomicExch(slot, 0u);
      if (v == SLOT_SENTINEL) return POP_NONE;
      if (v != 0u) return v - 1u;
    }
    __nanosleep(ns);
    ns = ns < 256 ? ns * 2 : ns;
    const uint64_t now = globaltimer();
    if (now - t_check > POLL_CHECK_NS) {
      t_check = now;
      if (ld_volatile(&q.hdr->done.v) | ld_volatile(&q.hdr->error.v)) return POP_NONE;
      if (ld_volatile(&a.lh->published.v) != ld_volatile(&a.lh->claimed.v) && live_may_claim(a, t_start)) return LIVE_ADMIT;
      const uint32_t pend = ld_volatile(&q.hdr->pending.v);
      if (pend == 0u) {
        w.t_prog = now;  // nothing to watch while idle
        const uint32_t tn = (uint32_t)(now / 1000ull);
        // Signed differences: another warp may have stamped last_busy after this warp read the clock.
        const bool idle = (int32_t)(tn - ld_volatile(&a.lh->last_busy.v)) > (int32_t)a.idle_us &&
                          (int32_t)(tn - t_start) > (int32_t)a.idle_us;
        const uint32_t why = ld_volatile(&a.lh->stop.v) ? LIVE_END_STOP
                             : idle                     ? LIVE_END_IDLE
                             : (int32_t)(tn - t_start) >= (int32_t)a.life_us ? LIVE_END_LIFE
                                                         : 0u;
        if (why && atomicCAS(&q.hdr->pending.v, 0u, LIVE_EXIT) == 0u) {
          atomicExch(&a.lh->end_reason.v, why);
          return LIVE_END;
        }
        continue;
      }
      // Progress: visits (flushed by the warps in batches) or a request claimed or completed.
      const uint32_t prog = ld_volatile(&q.hdr->progress.v) + ld_volatile(&a.lh->last_busy.v);
      if (prog != w.seen) { w.seen = prog; w.t_prog = now; }
      else if (now - w.t_prog > 1000000ull * ld_volatile(&a.lh->watch_ms.v)) { set_error(q, DERR_QUEUE_TIMEOUT, h); return POP_NONE; }
    }
  }
}

// Pop of the live kernel (whole warp): a tile id, a set-up job item, or POP_NONE when the kernel ends.
// Published entries are claimed first (before a ticket is taken, and by waiters that keep their ticket).
__device__ __forceinline__ uint32_t live_pop(const LiveArgs& a, uint32_t t_start) {
  const int lane = threadIdx.x & 31;
  const Queue& q = a.q;
  for (;;) {  // claim what is published before waiting
    uint32_t more = 0;
    if (lane == 0) more = ld_volatile(&a.lh->published.v) != ld_volatile(&a.lh->claimed.v) && live_may_claim(a, t_start);
    if (!__shfl_sync(~0u, more, 0)) break;
    if (!live_admit(a, t_start)) break;
  }
  PopWatch w{globaltimer(), 0u};
  uint32_t h = 0, res = POP_NONE;
  if (lane == 0) {
    w.seen = ld_volatile(&q.hdr->progress.v) + ld_volatile(&a.lh->last_busy.v);
    h = atomicAdd(&q.hdr->heads[0].v, 1u);
    __threadfence();
  }
  for (;;) {
    if (lane == 0) res = (ld_volatile(&q.hdr->done.v) | ld_volatile(&q.hdr->error.v)) ? POP_NONE : live_take(a, h, w, t_start);
    res = __shfl_sync(~0u, res, 0);
    if (res == LIVE_ADMIT) {
      live_admit(a, t_start);
      continue;
    }
    if (res == LIVE_END) {
      signal_done_warp(q);
      return POP_NONE;
    }
    return res;
  }
}

// The live tile kernel: every warp claims published entries, runs set-up jobs and visits tiles until the
// kernel ends (see the head of this file).
template <int WPC, int MINB>
__global__ void __launch_bounds__(WPC * 32, MINB) ggdt_live(LiveArgs a) {
  extern __shared__ uint8_t smem_raw[];
  WarpSmem& sm = warp_slot(smem_raw);
  warp_slot_init(sm);
  uint32_t parity = 0;
  const int lane = threadIdx.x & 31;
  uint32_t t_start = 0;
  if (lane == 0) t_start = now_us();
  t_start = __shfl_sync(~0u, t_start, 0);
  if (lane == 0) sm.keep = POP_NONE;
  __syncwarp();
  const LiveSched sch{a.q, a.states, &a, &sm.keep};
  WarpStats ws;
  for (;;) {
    uint32_t it = sm.keep;  // the own tile the last visit kept (a re-run), else the queue and admissions
    __syncwarp();
    const bool again = it != POP_NONE;
    if (!again) {
      it = live_pop(a, t_start);
      if (it == POP_NONE) break;
    } else if (lane == 0) {
      sm.keep = POP_NONE;
    }
    if (it & LIVE_JOB) {
      live_job(a, it);
      continue;
    }
    uint32_t old = 0;
    if (lane == 0) old = atomicXor(&a.states[it], ST_PENDING | ST_RUNNING);
    old = __shfl_sync(~0u, old, 0);
    const uint32_t slot = old >> ST_IMG_SHIFT;
    const ImgDesc dd = load_desc(a.descs + slot);
    // A first visit reads planes that a set-up job may have moved into place, and a seed visit a mask an edit
    // drew into, by generic stores; the visit reads them by bulk copy (async proxy).
    if ((old & ST_SEED) || !(old & ST_VISITED)) asm volatile("fence.proxy.async.global;" ::: "memory");
    uint32_t nph, nact;
    visit_ns<false>(dd, a.tmaps + 2 * slot, a.tmaps + 2 * slot + 1, it, old, visit_bufs(sm, parity), sch, &nph, &nact,
                    again && (old & ST_VISITED) && !(old & ST_SEED));
    count_visit(ws, a.q, nph, nact);
  }
  flush_stats(ws, a.q);
}

}  // namespace dtb
