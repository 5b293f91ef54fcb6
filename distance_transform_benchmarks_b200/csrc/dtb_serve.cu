// dtb_serve.cu -- serving engine: continuous batching of new-image and seed-edit requests.
//
// A worker thread runs waves.  Each wave admits, in arrival order, the pending requests that fit the device
// memory budget (a new image needs its image, mask and distance planes; an edit needs a resident image not
// already in the wave), evicting least-recently-used idle resident images when room is needed.  All requests
// of a wave share one persistent launch over one tile queue, so their work overlaps on the device; requests
// that arrive while a wave runs join the next one.  Distance maps stay resident: a seed edit draws its disks
// into the resident mask and warm-starts from the previous map -- every tile starts as already computed and
// only the tiles the new disks touch are queued.  This is exact: added seeds only lower distances, and the
// relaxation from the previous fixpoint ends in the fixpoint of the union of the seeds.
//
// With dtb_serve_config.live the worker runs no waves: it publishes each request into the device ring of the
// live tile kernel (dtb_live.cuh), keeps that kernel launched while requests are in flight, watches the
// completion words the kernel writes into mapped host memory and copies each finished map out.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "dtb.h"
#include "dtb_internal.h"
#include "dtb_live.cuh"

namespace dtb {

struct DiskItem {
  int32_t img, cx, cy, r;
};

// Tile states of a wave: cold images scan their seed mask (as ggdt_scan); warm images start VISITED.
__global__ void __launch_bounds__(128) serve_wave_init(const ImgDesc* __restrict__ descs, const uint32_t* __restrict__ tile_base,
                                                       const uint8_t* __restrict__ warm, int n, uint32_t total,
                                                       uint32_t* __restrict__ states, Queue q) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < total; t += nw) {
    const uint32_t img = image_of_tile(tile_base, n, t);
    if (warm[img]) {
      if (lane == 0) states[t] = (img << ST_IMG_SHIFT) | ST_VISITED;
      continue;
    }
    const ImgDesc& dd = descs[img];
    const uint32_t local = t - dd.tile_base;
    const int tx = (int)(local % (uint32_t)dd.tiles_x), ty = (int)(local / (uint32_t)dd.tiles_x);
    const int x0 = tx * TILE, y0 = ty * TILE;
    const int vw = min(TILE, dd.width - x0), vh = min(TILE, dd.height - y0);
    bool nz = false;
    if (lane < vh) {
      const uint8_t* row = dd.mask + (int64_t)(y0 + lane) * dd.mask_pitch + x0;
      for (int c = 0; c < vw; ++c) nz |= row[c] != 0;
    }
    nz = __any_sync(~0u, nz);
    if (lane == 0) {
      states[t] = (img << ST_IMG_SHIFT) | (nz ? (ST_SEED | ST_PENDING) : 0u);
      if (nz) queue_push(q, t);
    }
  }
}

// Draws the new seed disks of edit requests into the resident masks.
__global__ void __launch_bounds__(256) serve_draw_disks(const ImgDesc* __restrict__ descs, const DiskItem* __restrict__ disks,
                                                        int nd) {
  for (int k = blockIdx.x; k < nd; k += gridDim.x) {
    const DiskItem dk = disks[k];
    const ImgDesc& dd = descs[dk.img];
    const int xa = max(0, dk.cx - dk.r), xb = min(dd.width - 1, dk.cx + dk.r);
    const int ya = max(0, dk.cy - dk.r), yb = min(dd.height - 1, dk.cy + dk.r);
    if (xa > xb || ya > yb) continue;
    const int bw = xb - xa + 1, cnt = bw * (yb - ya + 1);
    uint8_t* mask = const_cast<uint8_t*>(dd.mask);
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int x = xa + i % bw, y = ya + i / bw;
      const int ddx = x - dk.cx, ddy = y - dk.cy;
      if (ddx * ddx + ddy * ddy <= dk.r * dk.r) mask[(int64_t)y * dd.mask_pitch + x] = 1;
    }
  }
}

// Queues the tiles touched by the new disks (after serve_wave_init): SEED makes the visit apply the mask.
__global__ void __launch_bounds__(32) serve_seed_tiles(const ImgDesc* __restrict__ descs, const DiskItem* __restrict__ disks,
                                                       int nd, uint32_t* __restrict__ states, Queue q) {
  for (int k = blockIdx.x; k < nd; k += gridDim.x) {
    const DiskItem dk = disks[k];
    const ImgDesc& dd = descs[dk.img];
    const int xa = max(0, dk.cx - dk.r), xb = min(dd.width - 1, dk.cx + dk.r);
    const int ya = max(0, dk.cy - dk.r), yb = min(dd.height - 1, dk.cy + dk.r);
    if (xa > xb || ya > yb) continue;
    const int txa = xa / TILE, txb = xb / TILE, tya = ya / TILE, tyb = yb / TILE;
    const int ntx = txb - txa + 1, cnt = ntx * (tyb - tya + 1);
    for (int i = threadIdx.x; i < cnt; i += 32) {
      const uint32_t t = dd.tile_base + (uint32_t)((tya + i / ntx) * dd.tiles_x + txa + i % ntx);
      const uint32_t old = atomicOr(&states[t], ST_SEED | ST_PENDING);
      if (!(old & (ST_PENDING | ST_RUNNING))) queue_push(q, t);
    }
  }
}

}  // namespace dtb

using namespace dtb;
using Clock = std::chrono::steady_clock;

namespace {

// First-fit allocator over the device arena (offsets, 256-byte granules).
class Arena {
 public:
  void reset(size_t size) {
    free_.clear();
    if (size) free_[0] = size;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = align_up(std::max<size_t>(bytes, 1), 256);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, at = it->first + bytes;
        free_.erase(it);
        if (rest) free_[at] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = align_up(std::max<size_t>(bytes, 1), 256);
    auto it = free_.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }

 private:
  std::map<size_t, size_t> free_;
};

struct Resident {
  int W = 0, H = 0, C = 1;
  float g2 = 0.0f;
  size_t off = 0, bytes = 0;  // one arena block: image, mask, distances
  int64_t img_pitch = 0, mask_pitch = 0, dist_pitch = 0;
  size_t o_img = 0, o_mask = 0, o_dist = 0;  // within the block
  uint64_t last_use = 0;
  int64_t wave = -1;  // wave the image takes part in (busy while it runs); live engine: 0 while in flight
  int32_t slot = -1;  // live engine: image slot (descriptor, tensor maps, request counters)
  uint32_t tile_base = 0, tiles = 0;  // live engine: the image's range of the tile space
};

struct Request {
  int64_t rid = 0;
  dtb_serve_request r{};
  std::vector<int32_t> disks;
  Clock::time_point t_submit;
};

size_t plane_pitch(size_t row_bytes) { return row_bytes % 16 ? align_up(row_bytes, 128) : row_bytes; }

uint64_t tiles_of(int W, int H) { return (uint64_t)((W + 31) / 32) * (uint64_t)((H + 31) / 32); }

// Device staging a new image needs in a wave: its image and mask planes, where their rows need a new pitch.
size_t stage_need(int W, int H, int C) {
  size_t b = 0;
  if (plane_pitch((size_t)W * C) != (size_t)W * C) b += align_up((size_t)W * C * H, 256);
  if (plane_pitch((size_t)W) != (size_t)W) b += align_up((size_t)W * H, 256);
  return b;
}

}  // namespace

// Device and pinned host buffers of one wave in flight, allocated by dtb_serve_create for the per-wave limits;
// a slot is reused only after its previous wave ended.
struct WaveSlot {
  void* scratch = nullptr;  // queue, tile states, tables of the wave
  size_t scratch_size = 0;
  void* stage = nullptr;    // packed staging of new images whose rows need a pitch change
  size_t stage_size = 0;
  uint8_t* hpin = nullptr;  // pinned host copy of the wave's tables
  size_t hpin_size = 0;
  cudaEvent_t ev_in = nullptr, ev_comp = nullptr, ev_done = nullptr;
  // Timing of the wave's phases on their streams: copies in, tile run, copies out (start and end of each).
  cudaEvent_t t_in0 = nullptr, t_in1 = nullptr, t_run0 = nullptr, t_run1 = nullptr, t_out0 = nullptr, t_out1 = nullptr;
};

// Per-wave limits (dtb_serve_config defaults).
constexpr int SERVE_MAX_WAVE_REQUESTS = 4096;
constexpr uint32_t SERVE_MAX_WAVE_TILES = 1u << 20;
constexpr uint64_t SERVE_WAVE_STAGE_BYTES = 256ull << 20;
constexpr size_t SERVE_MAX_WAVE_DISKS = 65536;

struct LiveEngine;
void live_free_resident(LiveEngine* L, const Resident& r);

struct dtb_server_s {
  dtb_context ctx = nullptr;
  dtb_serve_config cfg{};
  uint8_t* arena_base = nullptr;
  Arena arena;
  std::map<int64_t, Resident> resident;
  std::mutex mu;
  std::condition_variable cv_sub, cv_done;
  std::deque<Request> pending;
  std::deque<dtb_serve_completion> done;
  std::thread worker;
  bool stop = false;
  int64_t next_rid = 1;
  uint64_t tick = 0;
  int64_t wave_no = 0;
  int64_t busy_from = 1;  // residents with wave >= busy_from belong to a wave in flight
  WaveSlot slot[2];
  cudaStream_t s_in = nullptr, s_run = nullptr, s_out = nullptr;  // copies in, tile runs, copies out
  dtb_serve_stats st{};
  // Per-wave limits, and the queue geometry every wave's scratch was sized for.
  int max_reqs = SERVE_MAX_WAVE_REQUESTS;
  uint32_t max_tiles = SERVE_MAX_WAVE_TILES;
  size_t stage_cap = SERVE_WAVE_STAGE_BYTES;
  uint32_t workers = 0;  // resident warps of the largest tile-kernel launch
  uint32_t nb = 1;       // priority buckets of the waves' tile queues
  LiveEngine* live = nullptr;  // live admission instead of waves
};

namespace {

void complete(dtb_server s, const Request& q, dtb_status status, Clock::time_point now) {
  dtb_serve_completion c{};
  c.request_id = q.rid;
  c.status = status;
  c.latency_ms = std::chrono::duration<double, std::milli>(now - q.t_submit).count();
  s->done.push_back(c);
  s->st.completed += 1;
  if (status != DTB_OK) s->st.failed += 1;
}

bool referenced(dtb_server s, int64_t id) {
  for (const Request& q : s->pending)
    if (q.r.image_id == id) return true;
  return false;
}

// Forgets a resident image: its arena block and, in the live engine, its slot and tile range.  Caller holds mu.
void drop_resident(dtb_server s, std::map<int64_t, Resident>::iterator it) {
  s->arena.release(it->second.off, it->second.bytes);
  if (s->live) live_free_resident(s->live, it->second);
  s->resident.erase(it);
}

// Least-recently-used idle resident, or resident.end().  Caller holds mu.
std::map<int64_t, Resident>::iterator lru_idle(dtb_server s) {
  auto victim = s->resident.end();
  uint64_t oldest = UINT64_MAX;
  for (auto it = s->resident.begin(); it != s->resident.end(); ++it) {
    if (it->second.wave >= s->busy_from || referenced(s, it->first)) continue;
    if (it->second.last_use < oldest) {
      oldest = it->second.last_use;
      victim = it;
    }
  }
  return victim;
}

// Makes room for `bytes` in the arena by evicting least-recently-used idle residents.  Caller holds mu.
bool make_room(dtb_server s, size_t bytes, size_t* off) {
  while (!s->arena.alloc(bytes, off)) {
    auto victim = lru_idle(s);
    if (victim == s->resident.end()) return false;
    drop_resident(s, victim);
    s->st.evictions += 1;
  }
  return true;
}

// Admission of one wave (caller holds mu).  Requests that cannot run now stay pending in order.  The wave is
// closed when the next request would take it past a per-wave limit (requests, tiles, staging, disks): the
// buffers of a wave slot were sized for those limits at create time.  *split reports such a close.
std::vector<Request> admit(dtb_server s, bool* split) {
  std::vector<Request> wave;
  std::deque<Request> keep;
  const auto now = Clock::now();
  bool blocked = false;  // a new image that did not fit keeps later new images waiting (arrival order)
  bool closed = false;   // a per-wave limit was reached: the rest waits for the next wave
  std::set<int64_t> kept_new;  // new images left pending: edits of them wait too
  uint64_t w_tiles = 0;
  size_t w_stage = 0, w_disks = 0;
  *split = false;
  while (!s->pending.empty()) {
    Request q = std::move(s->pending.front());
    s->pending.pop_front();
    if (closed || (int32_t)wave.size() >= s->max_reqs) {
      if (!closed) closed = *split = true;
      keep.push_back(std::move(q));
      continue;
    }
    auto it = s->resident.find(q.r.image_id);
    if (q.r.kind == DTB_REQ_EDIT) {
      if (it == s->resident.end() && kept_new.count(q.r.image_id)) {
        keep.push_back(std::move(q));  // its image's request waits: so does the edit
        continue;
      }
      if (it == s->resident.end()) {
        complete(s, q, DTB_ERR_INVALID_ARG, now);  // not resident (never submitted, released or evicted)
        continue;
      }
      if (it->second.wave >= s->busy_from) {
        keep.push_back(std::move(q));  // one wave in flight per image: its map may still be on its way out
        continue;
      }
      const uint64_t t = tiles_of(it->second.W, it->second.H);
      const size_t nd = q.disks.size() / 3;
      if (!wave.empty() && (w_tiles + t > s->max_tiles || w_disks + nd > SERVE_MAX_WAVE_DISKS)) {
        closed = *split = true;
        keep.push_back(std::move(q));
        continue;
      }
      w_tiles += t;
      w_disks += nd;
      it->second.wave = s->wave_no;
      it->second.last_use = ++s->tick;
      wave.push_back(std::move(q));
      continue;
    }
    // new image
    if (it != s->resident.end()) {
      complete(s, q, DTB_ERR_INVALID_ARG, now);  // id already resident
      continue;
    }
    if (blocked) {
      kept_new.insert(q.r.image_id);
      keep.push_back(std::move(q));
      continue;
    }
    const uint64_t t = tiles_of(q.r.img.width, q.r.img.height);
    const size_t sb = stage_need(q.r.img.width, q.r.img.height, q.r.img.elem_size);
    if (t > s->max_tiles || sb > s->stage_cap) {
      complete(s, q, DTB_ERR_CAPACITY, now);  // larger than a whole wave may be
      continue;
    }
    if (!wave.empty() && (w_tiles + t > s->max_tiles || w_stage + sb > s->stage_cap)) {
      closed = *split = true;
      keep.push_back(std::move(q));
      continue;
    }
    Resident r;
    r.W = q.r.img.width;
    r.H = q.r.img.height;
    r.C = q.r.img.elem_size;
    r.g2 = gamma_to_g2(q.r.gamma);
    r.img_pitch = (int64_t)plane_pitch((size_t)r.W * r.C);
    r.mask_pitch = (int64_t)plane_pitch((size_t)r.W);
    r.dist_pitch = (int64_t)align_up(4 * (size_t)std::max(r.W, 1), 128);
    r.o_img = 0;
    r.o_mask = align_up((size_t)r.img_pitch * r.H, 256);
    r.o_dist = r.o_mask + align_up((size_t)r.mask_pitch * r.H, 256);
    r.bytes = r.o_dist + align_up((size_t)r.dist_pitch * r.H, 256);
    if (r.bytes > s->cfg.hbm_budget_bytes) {
      complete(s, q, DTB_ERR_CAPACITY, now);
      continue;
    }
    size_t off = 0;
    if (!make_room(s, r.bytes, &off)) {
      blocked = true;
      kept_new.insert(q.r.image_id);
      keep.push_back(std::move(q));
      continue;
    }
    r.off = off;
    r.wave = s->wave_no;
    r.last_use = ++s->tick;
    s->resident[q.r.image_id] = r;
    w_tiles += t;
    w_stage += sb;
    wave.push_back(std::move(q));
  }
  s->pending = std::move(keep);
  return wave;
}

// Device scratch a wave of n requests and `total` tiles needs: its run layout plus warm flags, disks and
// repitch items; *o_* receive the offsets of the three extras.
size_t wave_scratch_bytes(const ScratchLayout& L, int n, size_t ndisks, size_t nitems, size_t* o_warm, size_t* o_disks,
                          size_t* o_items) {
  size_t off = L.bytes;
  *o_warm = off;
  off = align_up(off + (size_t)std::max(n, 1), 256);
  *o_disks = off;
  off = align_up(off + sizeof(DiskItem) * std::max<size_t>(ndisks, 1), 256);
  *o_items = off;
  off = align_up(off + sizeof(RepitchItem) * std::max<size_t>(nitems, 1), 256);
  return off;
}

// A wave in flight: its requests, slot and device queue header.
struct InFlight {
  std::vector<Request> reqs;
  int slot = 0;
  int64_t no = 0;
  uint32_t total = 0;
  const QueueHdr* hdr = nullptr;
  double prep_ms = 0.0;  // host time to admit and enqueue the wave
};

// Enqueues one wave: copies in and table upload on s_in, tile work on s_run, copies out on s_out; ev_done of
// the slot marks its end.  The caller holds the context's lock, as every API call on the context does (the
// helpers below record failures in the context's message).  Requests of the wave reference no image of another wave in flight (admit), so the
// waves' device work only shares the arena's free space and the tile-run stream.
dtb_status launch_wave(dtb_server s, InFlight& f) {
  const TraceRange trace("dtb serve wave");
  dtb_context ctx = s->ctx;
  cudaStream_t st = s->s_run;
  WaveSlot& ws = s->slot[f.slot];
  std::vector<Request>& wave = f.reqs;
  const int n = (int)wave.size();
  std::vector<Resident*> rs(n);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (int i = 0; i < n; ++i) rs[i] = &s->resident[wave[i].r.image_id];
  }
  // Jobs on the resident planes; packed staging for new images whose rows need a pitch change.
  std::vector<Job> jobs(n);
  std::vector<uint8_t> warm(n);
  std::vector<DiskItem> disks;
  std::vector<RepitchItem> items;
  uint32_t rows = 0;
  size_t stage_bytes = 0;
  std::vector<size_t> o_stage_img(n, SIZE_MAX), o_stage_mask(n, SIZE_MAX);
  for (int i = 0; i < n; ++i) {
    Resident& r = *rs[i];
    uint8_t* base = s->arena_base + r.off;
    Job& j = jobs[i];
    j.img = base + r.o_img;
    j.img_pitch = r.img_pitch;
    j.channels = r.C;
    j.mask = base + r.o_mask;
    j.mask_pitch = r.mask_pitch;
    j.dist = reinterpret_cast<float*>(base + r.o_dist);
    j.dist_pitch = r.dist_pitch;
    j.width = r.W;
    j.height = r.H;
    j.g2 = r.g2;
    j.v = s->cfg.v;
    j.mode = MODE_NS;
    warm[i] = wave[i].r.kind == DTB_REQ_EDIT;
    if (warm[i]) {
      for (size_t k = 0; k + 2 < wave[i].disks.size(); k += 3)
        disks.push_back({i, wave[i].disks[k], wave[i].disks[k + 1], wave[i].disks[k + 2]});
    } else {
      if ((size_t)r.img_pitch != (size_t)r.W * r.C) {
        o_stage_img[i] = stage_bytes;
        stage_bytes = align_up(stage_bytes + (size_t)r.W * r.C * r.H, 256);
      }
      if ((size_t)r.mask_pitch != (size_t)r.W) {
        o_stage_mask[i] = stage_bytes;
        stage_bytes = align_up(stage_bytes + (size_t)r.W * r.H, 256);
      }
    }
  }
  dtb_status s2 = DTB_OK;
  if (stage_bytes > ws.stage_size)  // admission keeps a wave within the slot's staging
    return fail(ctx, DTB_ERR_CAPACITY, "serve: wave staging %zu > %zu bytes", stage_bytes, ws.stage_size);
  uint8_t* stage = static_cast<uint8_t*>(ws.stage);
  DTB_CUDA(ctx, cudaEventRecord(ws.t_in0, s->s_in));
  // Host -> device: one 1-D copy per plane (into the resident plane, or into staging + repitch).
  for (int i = 0; i < n; ++i) {
    if (warm[i]) continue;
    const dtb_serve_request& q = wave[i].r;
    Resident& r = *rs[i];
    const size_t rb = (size_t)r.W * r.C;
    uint8_t* dimg = o_stage_img[i] == SIZE_MAX ? const_cast<uint8_t*>(jobs[i].img) : stage + o_stage_img[i];
    uint8_t* dmask = o_stage_mask[i] == SIZE_MAX ? const_cast<uint8_t*>(jobs[i].mask) : stage + o_stage_mask[i];
    if ((size_t)q.img.pitch == rb)
      DTB_CUDA(ctx, cudaMemcpyAsync(dimg, q.img.buffer, rb * r.H, cudaMemcpyHostToDevice, s->s_in));
    else
      DTB_CUDA(ctx, cudaMemcpy2DAsync(dimg, rb, q.img.buffer, q.img.pitch, rb, r.H, cudaMemcpyHostToDevice, s->s_in));
    if (q.mask.pitch == r.W)
      DTB_CUDA(ctx, cudaMemcpyAsync(dmask, q.mask.buffer, (size_t)r.W * r.H, cudaMemcpyHostToDevice, s->s_in));
    else
      DTB_CUDA(ctx, cudaMemcpy2DAsync(dmask, r.W, q.mask.buffer, q.mask.pitch, r.W, r.H, cudaMemcpyHostToDevice, s->s_in));
    if (o_stage_img[i] != SIZE_MAX) {
      items.push_back({dimg, const_cast<uint8_t*>(jobs[i].img), (uint32_t)rb, (uint32_t)r.H, (uint32_t)r.img_pitch, rows});
      rows += (uint32_t)r.H;
    }
    if (o_stage_mask[i] != SIZE_MAX) {
      items.push_back({dmask, const_cast<uint8_t*>(jobs[i].mask), (uint32_t)r.W, (uint32_t)r.H, (uint32_t)r.mask_pitch, rows});
      rows += (uint32_t)r.H;
    }
  }
  // Scratch: run layout + warm flags + disks + repitch items, one upload.
  uint32_t total = 0;
  if ((s2 = count_tiles(ctx, jobs, &total)) != DTB_OK) return s2;
  LaunchTuning tuning = ctx->tuning;
  tuning.buckets = (int)std::min<uint32_t>((uint32_t)tuning.buckets, s->nb);
  const ScratchLayout L = layout_for(n, total, s->workers, false, s->nb);
  size_t o_warm = 0, o_disks = 0, o_items = 0;
  const size_t off = wave_scratch_bytes(L, n, disks.size(), items.size(), &o_warm, &o_disks, &o_items);
  if (off > ws.scratch_size)  // admission keeps a wave within the slot's scratch
    return fail(ctx, DTB_ERR_CAPACITY, "serve: wave scratch %zu > %zu bytes", off, ws.scratch_size);
  uint8_t* sc = static_cast<uint8_t*>(ws.scratch);
  std::vector<uint8_t> tab;
  if ((s2 = build_tables(ctx, jobs, L, tab)) != DTB_OK) return s2;
  // Tables, warm flags, disks and repitch items: one upload from the slot's pinned buffer (free: the slot's
  // previous wave has ended), so that the copy does not wait for the other wave's work.
  const size_t hbytes = off - L.o_desc;
  if (ws.hpin_size < hbytes)
    return fail(ctx, DTB_ERR_CAPACITY, "serve: wave tables %zu > %zu bytes", hbytes, ws.hpin_size);
  uint8_t* host = ws.hpin;
  std::memset(host, 0, hbytes);
  std::copy(tab.begin(), tab.end(), host);
  std::copy(warm.begin(), warm.end(), host + (o_warm - L.o_desc));
  std::copy(reinterpret_cast<const uint8_t*>(disks.data()), reinterpret_cast<const uint8_t*>(disks.data() + disks.size()),
            host + (o_disks - L.o_desc));
  std::copy(reinterpret_cast<const uint8_t*>(items.data()), reinterpret_cast<const uint8_t*>(items.data() + items.size()),
            host + (o_items - L.o_desc));
  DTB_CUDA(ctx, cudaMemcpyAsync(sc + L.o_desc, host, hbytes, cudaMemcpyHostToDevice, s->s_in));
  DTB_CUDA(ctx, cudaEventRecord(ws.t_in1, s->s_in));
  DTB_CUDA(ctx, cudaEventRecord(ws.ev_in, s->s_in));
  DTB_CUDA(ctx, cudaStreamWaitEvent(st, ws.ev_in, 0));
  DTB_CUDA(ctx, cudaEventRecord(ws.t_run0, st));
  const dtb_status qs = reset_queue(ctx, sc, L, st);
  if (qs != DTB_OK) return qs;
  const ImgDesc* ddesc = reinterpret_cast<const ImgDesc*>(sc + L.o_desc);
  const CUtensorMap* dtm = reinterpret_cast<const CUtensorMap*>(sc + L.o_tmap);
  const uint32_t* dbase = reinterpret_cast<const uint32_t*>(sc + L.o_base);
  uint32_t* states = reinterpret_cast<uint32_t*>(sc + L.o_states);
  // dtb_debug_inject_queue_stall on the server's context applies to the next wave with tiles (one-shot; the
  // caller holds ctx->mu).
  uint64_t stall_ns = 0;
  if (total > 0) {
    stall_ns = ctx->inject_stall_ns;
    ctx->inject_stall_ns = 0;
  }
  Queue q = make_queue(sc, L, stall_ns ? stall_ns : DEFAULT_TIMEOUT_NS, &tuning);
  f.hdr = total > 0 ? reinterpret_cast<QueueHdr*>(sc + L.o_hdr) : nullptr;
  f.total = total;
  if (!items.empty()) {
    repitch_rows<<<std::min<uint32_t>((rows + 7) / 8, (uint32_t)ctx->num_sms * 8), 256, 0, st>>>(
        reinterpret_cast<const RepitchItem*>(sc + o_items), (int)items.size(), rows);
    DTB_CUDA(ctx, cudaGetLastError());
  }
  if (!disks.empty()) {
    serve_draw_disks<<<std::min<int>((int)disks.size(), 4096), 256, 0, st>>>(ddesc, reinterpret_cast<const DiskItem*>(sc + o_disks),
                                                                             (int)disks.size());
    DTB_CUDA(ctx, cudaGetLastError());
  }
  if (total > 0) {
    const uint32_t blocks = std::min<uint32_t>((total + 3) / 4, (uint32_t)ctx->num_sms * 16);
    serve_wave_init<<<blocks, 128, 0, st>>>(ddesc, dbase, sc + o_warm, n, total, states, q);
    DTB_CUDA(ctx, cudaGetLastError());
    if (!disks.empty()) {
      serve_seed_tiles<<<std::min<int>((int)disks.size(), 4096), 32, 0, st>>>(
          ddesc, reinterpret_cast<const DiskItem*>(sc + o_disks), (int)disks.size(), states, q);
      DTB_CUDA(ctx, cudaGetLastError());
    }
    if (stall_ns) {
      ggdt_phantom_pending<<<1, 1, 0, st>>>(q.hdr);
      DTB_CUDA(ctx, cudaGetLastError());
    }
    const dtb_status ls = launch_tile_kernel(ctx, MODE_NS, tuning, ddesc, dtm, states, q, st);
    if (ls != DTB_OK) return ls;
    ggdt_finalize<<<blocks, 128, 0, st>>>(ddesc, dbase, n, total, states, nullptr, nullptr);
    DTB_CUDA(ctx, cudaGetLastError());
  }
  DTB_CUDA(ctx, cudaEventRecord(ws.t_run1, st));
  DTB_CUDA(ctx, cudaEventRecord(ws.ev_comp, st));
  // Device -> host: each request's map into its output buffer.
  DTB_CUDA(ctx, cudaStreamWaitEvent(s->s_out, ws.ev_comp, 0));
  DTB_CUDA(ctx, cudaEventRecord(ws.t_out0, s->s_out));
  for (int i = 0; i < n; ++i) {
    const dtb_image& o = wave[i].r.out;
    if (o.width == 0 || o.height == 0) continue;
    DTB_CUDA(ctx, cudaMemcpy2DAsync(o.buffer, o.pitch, jobs[i].dist, jobs[i].dist_pitch, 4 * (size_t)o.width, o.height,
                                    cudaMemcpyDeviceToHost, s->s_out));
  }
  DTB_CUDA(ctx, cudaEventRecord(ws.t_out1, s->s_out));
  DTB_CUDA(ctx, cudaEventRecord(ws.ev_done, s->s_out));
  return DTB_OK;
}

// Adds the stream times of an ended wave's phases to the statistics (caller holds mu).
void add_wave_times(dtb_server s, const InFlight& f) {
  const WaveSlot& ws = s->slot[f.slot];
  float a = 0.0f, b = 0.0f, c = 0.0f;
  if (cudaEventElapsedTime(&a, ws.t_in0, ws.t_in1) != cudaSuccess) a = 0.0f;
  if (cudaEventElapsedTime(&b, ws.t_run0, ws.t_run1) != cudaSuccess) b = 0.0f;
  if (cudaEventElapsedTime(&c, ws.t_out0, ws.t_out1) != cudaSuccess) c = 0.0f;
  cudaGetLastError();
  s->st.copy_in_ms += a;
  s->st.kernel_ms += b;
  s->st.copy_out_ms += c;
  s->st.host_prep_ms += f.prep_ms;
}

// Completes the requests of a wave that has ended (or failed to enqueue): a failed new image is dropped, since
// its map is not valid.  Caller holds mu.
void retire_wave(dtb_server s, InFlight& f, dtb_status status) {
  const auto now = Clock::now();
  s->st.waves += 1;
  for (const Request& q : f.reqs) {
    if (status != DTB_OK && q.r.kind == DTB_REQ_IMAGE) {
      auto it = s->resident.find(q.r.image_id);
      if (it != s->resident.end()) drop_resident(s, it);
    }
    complete(s, q, status, now);
  }
}

// The worker keeps up to two waves in flight: while one runs, the next is admitted and enqueued, so its copies
// in and host preparation overlap the running tile kernel, and its tile kernel overlaps the previous wave's
// copies out.  A request whose image belongs to a wave in flight waits for that wave's end (admit).
void worker_main(dtb_server s) {
  cudaSetDevice(s->ctx->device);
  std::deque<InFlight> inflight;
  int64_t blocked_at = -1;  // submissions counted when an admission found nothing to run beside a wave in flight
  auto set_busy_from = [&] { s->busy_from = inflight.empty() ? s->wave_no + 1 : inflight.front().no; };
  for (;;) {
    InFlight f;
    Clock::time_point t_prep;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (inflight.empty()) s->cv_sub.wait(lk, [&] { return s->stop || !s->pending.empty(); });
      if (inflight.empty() && s->stop && s->pending.empty()) break;
      if (inflight.size() < 2 && !s->pending.empty() && s->st.submitted != blocked_at) {
        f.no = ++s->wave_no;
        s->busy_from = inflight.empty() ? f.no : inflight.front().no;  // during admission and while f runs
        bool split = false;
        t_prep = Clock::now();
        f.reqs = admit(s, &split);
        if (split) s->st.waves_split += 1;
        for (const Request& q : f.reqs) {
          const double w = std::chrono::duration<double, std::milli>(t_prep - q.t_submit).count();
          s->st.queue_wait_ms += w;
          s->st.queue_wait_max_ms = std::max(s->st.queue_wait_max_ms, w);
        }
        if (f.reqs.empty()) {
          set_busy_from();
          s->cv_done.notify_all();  // admission may have completed invalid requests
          if (inflight.empty()) {
            // nothing fits and nothing runs: the head request can never fit
            if (!s->pending.empty()) {
              complete(s, s->pending.front(), DTB_ERR_CAPACITY, Clock::now());
              s->pending.pop_front();
            }
            continue;
          }
          blocked_at = s->st.submitted;  // retry after the oldest wave ends or a request arrives
        }
      }
    }
    if (!f.reqs.empty()) {
      f.slot = inflight.empty() ? 0 : (inflight.front().slot ^ 1);  // at most one wave is in flight here
      dtb_status ls;
      {
        std::lock_guard<std::mutex> ctx_lock(s->ctx->mu);
        ls = launch_wave(s, f);
      }
      f.prep_ms = std::chrono::duration<double, std::milli>(Clock::now() - t_prep).count();
      if (ls != DTB_OK) {
        // Nothing of this wave may still run when its requests complete.
        cudaStreamSynchronize(s->s_in);
        cudaStreamSynchronize(s->s_run);
        cudaStreamSynchronize(s->s_out);
        std::lock_guard<std::mutex> lk(s->mu);
        retire_wave(s, f, ls);
        set_busy_from();
        s->cv_done.notify_all();
        continue;
      }
      inflight.push_back(std::move(f));
      continue;
    }
    // Nothing to enqueue now: wait for the oldest wave's end or, with a slot free, for a new request.
    InFlight& old = inflight.front();
    cudaEvent_t ev = s->slot[old.slot].ev_done;
    if (inflight.size() < 2) {
      bool ended = false;
      for (;;) {
        if (cudaEventQuery(ev) != cudaErrorNotReady) {
          ended = true;
          break;
        }
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->st.submitted != blocked_at && !s->pending.empty()) break;
        s->cv_sub.wait_for(lk, std::chrono::microseconds(50));
      }
      if (!ended) continue;
    }
    dtb_status status = cudaEventSynchronize(ev) == cudaSuccess ? DTB_OK : DTB_ERR_CUDA;
    dtb_stats ds{};
    if (status == DTB_OK && old.hdr) {
      std::lock_guard<std::mutex> ctx_lock(s->ctx->mu);
      status = read_device_status(s->ctx, old.hdr, &ds);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.tile_visits += ds.tile_visits;
    s->st.tiles += old.total;
    add_wave_times(s, old);
    retire_wave(s, old, status);
    inflight.pop_front();
    set_busy_from();
    blocked_at = -1;
    s->cv_done.notify_all();
  }
}

}  // namespace

// ======================================================================================================
// Live engine (dtb_serve_config.live): requests join the tile queue of one running kernel (dtb_live.cuh).
// ======================================================================================================

// Pinned staging of one entry: its descriptor and tensor maps, the entry and the published count, copied in
// on s_in in that order.  Entry e's staging is reused by entry e + LIVE_RING, published only after e ended.
constexpr size_t LIVE_STAGE = 512;
constexpr size_t LST_DESC = 0, LST_TMAP = 128, LST_ENTRY = 384, LST_PUB = 448;
static_assert(LST_TMAP + 2 * sizeof(CUtensorMap) <= LST_ENTRY && LST_ENTRY + sizeof(LiveEntry) <= LST_PUB &&
                  sizeof(ImgDesc) <= LST_TMAP, "live staging layout");
constexpr uint32_t LIVE_WATCH_MS = 2000;       // no-progress limit of the live kernel's watchdog
constexpr uint32_t LIVE_LIFE_US = 4000000;     // a launch claims new requests for this long, then drains and ends
constexpr uint32_t LIVE_IDLE_US = 20000;       // default idle time after which a launch ends
constexpr uint32_t LIVE_DISK_CAP = 1u << 20;   // disks of edits in flight
constexpr size_t LIVE_DISK_BYTES = 16;         // a disk record (cx, cy, r, 0) in the pool
constexpr int LIVE_CTAS = 3;                   // CTAs of PERSIST_WPC warps per SM (the 168-register launch)

// A published request.
struct LiveFlight {
  Request q;
  uint32_t entry = 0;
  int stage = 0;               // 0: published; 1: its map is being copied out
  Clock::time_point t_pub, t_seen;
  cudaEvent_t ev = nullptr;    // end of the copy out
  size_t disk_off = SIZE_MAX;  // bytes of the disk pool held by an edit
  size_t disk_bytes = 0;
};

struct LiveEngine {
  uint8_t* dmem = nullptr;     // one device block: queue header, live header, ring, states, tables, entries, disks
  QueueHdr* qhdr = nullptr;
  LiveHdr* lh = nullptr;
  uint32_t* ring = nullptr;
  uint32_t ring_cap = 0;
  uint32_t* states = nullptr;
  ImgDesc* descs = nullptr;
  CUtensorMap* tmaps = nullptr;
  LiveSlot* slots = nullptr;
  LiveEntry* entries = nullptr;
  int32_t* disks = nullptr;
  uint32_t tile_cap = 0, nslots = 0;
  uint32_t* hdone = nullptr;   // mapped pinned host memory (LIVE_RING words), written by the kernel
  uint32_t* ddone = nullptr;   // its device address
  uint8_t* hstage = nullptr;   // pinned: LIVE_RING entry stagings, then the disk pool mirror, then constant words
  int32_t* hdisks = nullptr;
  uint32_t* hwords = nullptr;  // [0] = 1, [1] = LIVE_WATCH_MS, [2] = injected limit (ms)
  Arena tiles, diskpool;       // tile-space ranges (4 bytes a tile), disk-pool bytes
  std::vector<int32_t> free_slots;
  uint32_t next_entry = 0;
  std::deque<LiveFlight> flights;  // in publish order
  uint64_t flight_tiles = 0;
  std::vector<cudaEvent_t> ev_free;
  bool running = false;
  cudaEvent_t ev_kernel = nullptr;
  uint32_t idle_us = LIVE_IDLE_US;
  uint32_t grid = 0;
  uint32_t claimed_seen = 0;   // `claimed` as read after the last launch ended
};

void live_free_resident(LiveEngine* L, const Resident& r) {
  if (r.slot >= 0) L->free_slots.push_back(r.slot);
  if (r.tiles) L->tiles.release(4ull * r.tile_base, 4ull * r.tiles);
}

namespace {

// Device and pinned allocations of the live engine (dtb_serve_create).
dtb_status live_create(dtb_server s, uint32_t idle_us) {
  dtb_context ctx = s->ctx;
  LiveEngine* L = new (std::nothrow) LiveEngine();
  if (!L) return DTB_ERR_OUT_OF_MEMORY;
  s->live = L;
  s->busy_from = 0;  // a resident is busy while wave == 0
  L->idle_us = idle_us ? idle_us : LIVE_IDLE_US;
  // Tile space: every gray pixel the budget can hold, plus 64 tiles of rounding per slot; slots: at most
  // LIVE_MAX_SLOTS, at least enough for 64 KiB per image.
  const uint64_t budget = s->cfg.hbm_budget_bytes;
  L->nslots = (uint32_t)std::min<uint64_t>(LIVE_MAX_SLOTS, std::max<uint64_t>(64, budget / 65536));
  const uint64_t tiles = budget / (9ull * 1024ull) + 64ull * L->nslots + 64;
  L->tile_cap = (uint32_t)std::min<uint64_t>(LIVE_MAX_TILES, align_up(tiles, 64));
  // The live kernel's launch: LIVE_CTAS CTAs per SM, or fewer if fewer fit (the launch is cooperative).
  const void* fn = (const void*)ggdt_live<PERSIST_WPC, LIVE_CTAS>;
  int per_sm = 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PERSIST_SMEM) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PERSIST_WPC * 32, PERSIST_SMEM) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    return fail(ctx, DTB_ERR_CUDA, "serve (live): the live tile kernel cannot be resident");
  }
  L->grid = (uint32_t)ctx->num_sms * (uint32_t)std::min(per_sm, LIVE_CTAS);
  const uint32_t workers = L->grid * PERSIST_WPC;
  // Ring: items in flight (tiles of the requests in flight, their set-up jobs) plus waiting workers.
  const uint64_t items = (uint64_t)s->max_tiles + 2ull * (s->max_tiles + (uint64_t)s->max_reqs) +
                         workers + 64;
  uint32_t cap = 1;
  while (cap < 2 * items && cap < (1u << 30)) cap <<= 1;
  L->ring_cap = cap;
  size_t off = 0;
  const size_t o_q = off;       off = align_up(off + sizeof(QueueHdr), 256);
  const size_t o_lh = off;      off = align_up(off + sizeof(LiveHdr), 256);
  const size_t o_ring = off;    off = align_up(off + 4ull * cap, 256);
  const size_t o_states = off;  off = align_up(off + 4ull * L->tile_cap, 256);
  const size_t o_desc = off;    off = align_up(off + sizeof(ImgDesc) * L->nslots, 256);
  const size_t o_tmap = off;    off = align_up(off + 2 * sizeof(CUtensorMap) * L->nslots, 256);
  const size_t o_slots = off;   off = align_up(off + sizeof(LiveSlot) * L->nslots, 256);
  const size_t o_ent = off;     off = align_up(off + sizeof(LiveEntry) * LIVE_RING, 256);
  const size_t o_disks = off;   off = align_up(off + LIVE_DISK_BYTES * LIVE_DISK_CAP, 256);
  if (cudaMalloc((void**)&L->dmem, off) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, DTB_ERR_OUT_OF_MEMORY, "serve (live): cudaMalloc of %zu bytes failed", off);
  }
  L->qhdr = reinterpret_cast<QueueHdr*>(L->dmem + o_q);
  L->lh = reinterpret_cast<LiveHdr*>(L->dmem + o_lh);
  L->ring = reinterpret_cast<uint32_t*>(L->dmem + o_ring);
  L->states = reinterpret_cast<uint32_t*>(L->dmem + o_states);
  L->descs = reinterpret_cast<ImgDesc*>(L->dmem + o_desc);
  L->tmaps = reinterpret_cast<CUtensorMap*>(L->dmem + o_tmap);
  L->slots = reinterpret_cast<LiveSlot*>(L->dmem + o_slots);
  L->entries = reinterpret_cast<LiveEntry*>(L->dmem + o_ent);
  L->disks = reinterpret_cast<int32_t*>(L->dmem + o_disks);
  const size_t hbytes = LIVE_STAGE * LIVE_RING + LIVE_DISK_BYTES * LIVE_DISK_CAP + 256;
  if (cudaHostAlloc((void**)&L->hstage, hbytes, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void**)&L->hdone, 4ull * LIVE_RING, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void**)&L->ddone, L->hdone, 0) != cudaSuccess ||
      cudaEventCreateWithFlags(&L->ev_kernel, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, DTB_ERR_OUT_OF_MEMORY, "serve (live): pinned host buffers");
  }
  std::memset(L->hstage, 0, hbytes);
  std::memset(L->hdone, 0, 4ull * LIVE_RING);
  L->hdisks = reinterpret_cast<int32_t*>(L->hstage + LIVE_STAGE * LIVE_RING);
  L->hwords = reinterpret_cast<uint32_t*>(L->hstage + LIVE_STAGE * LIVE_RING + LIVE_DISK_BYTES * LIVE_DISK_CAP);
  L->hwords[0] = 1u;
  L->hwords[1] = LIVE_WATCH_MS;
  L->tiles.reset(4ull * L->tile_cap);
  L->diskpool.reset(LIVE_DISK_BYTES * LIVE_DISK_CAP);
  for (int32_t k = (int32_t)L->nslots - 1; k >= 0; --k) L->free_slots.push_back(k);
  // Everything starts at zero (states, counters, entries); the watchdog limit is set once.
  DTB_CUDA(ctx, cudaMemsetAsync(L->dmem, 0, off, s->s_run));
  DTB_CUDA(ctx, cudaMemcpyAsync(&L->lh->watch_ms.v, &L->hwords[1], 4, cudaMemcpyHostToDevice, s->s_run));
  DTB_CUDA(ctx, cudaStreamSynchronize(s->s_run));
  return DTB_OK;
}

void live_destroy(LiveEngine* L) {
  if (!L) return;
  for (cudaEvent_t e : L->ev_free) cudaEventDestroy(e);
  for (LiveFlight& f : L->flights)
    if (f.ev) cudaEventDestroy(f.ev);
  if (L->ev_kernel) cudaEventDestroy(L->ev_kernel);
  if (L->dmem) cudaFree(L->dmem);
  if (L->hstage) cudaFreeHost(L->hstage);
  if (L->hdone) cudaFreeHost(L->hdone);
  delete L;
}

// A free slot and a tile range for a new image of `tiles` tiles, evicting least-recently-used idle images when
// needed.  Caller holds mu.
bool live_place(dtb_server s, uint32_t tiles, int32_t* slot, uint32_t* tile_base) {
  LiveEngine* L = s->live;
  size_t toff = 0;
  for (;;) {
    const bool have_slot = !L->free_slots.empty();
    const bool have_tiles = tiles == 0 || L->tiles.alloc(4ull * tiles, &toff);
    if (have_slot && have_tiles) break;
    if (have_tiles && tiles) L->tiles.release(toff, 4ull * tiles);
    auto victim = lru_idle(s);
    if (victim == s->resident.end()) return false;
    drop_resident(s, victim);
    s->st.evictions += 1;
  }
  *slot = L->free_slots.back();
  L->free_slots.pop_back();
  *tile_base = tiles ? (uint32_t)(toff / 4) : 0u;
  return true;
}

// Admission of the live engine (caller holds mu): pending requests in arrival order while the requests and tiles
// in flight stay within the limits, the disk pool has room and (new images) the arena, a slot and a tile range
// can be found.  An edit of an image in flight waits; a new image that does not fit keeps later new images
// waiting.
std::vector<LiveFlight> live_admit_host(dtb_server s) {
  LiveEngine* L = s->live;
  std::vector<LiveFlight> out;
  std::deque<Request> keep;
  const auto now = Clock::now();
  bool blocked = false;
  std::set<int64_t> kept_new;  // new images left pending: edits of them wait too
  const size_t max_flights = std::min<size_t>((size_t)s->max_reqs, LIVE_RING / 2);
  while (!s->pending.empty()) {
    Request q = std::move(s->pending.front());
    s->pending.pop_front();
    if (L->flights.size() + out.size() >= max_flights) {
      keep.push_back(std::move(q));
      continue;
    }
    auto it = s->resident.find(q.r.image_id);
    if (q.r.kind == DTB_REQ_EDIT) {
      if (it == s->resident.end() && kept_new.count(q.r.image_id)) {
        keep.push_back(std::move(q));  // its image's request waits: so does the edit
        continue;
      }
      if (it == s->resident.end()) {
        complete(s, q, DTB_ERR_INVALID_ARG, now);
        continue;
      }
      if (it->second.wave >= s->busy_from) {
        keep.push_back(std::move(q));
        continue;
      }
      LiveFlight f;
      f.disk_bytes = LIVE_DISK_BYTES * (q.disks.size() / 3);
      if (f.disk_bytes) {
        size_t doff = 0;
        if (!L->diskpool.alloc(f.disk_bytes, &doff)) {
          keep.push_back(std::move(q));
          continue;
        }
        f.disk_off = doff;
      }
      it->second.wave = 0;
      it->second.last_use = ++s->tick;
      L->flight_tiles += it->second.tiles;
      f.q = std::move(q);
      out.push_back(std::move(f));
      continue;
    }
    if (it != s->resident.end()) {
      complete(s, q, DTB_ERR_INVALID_ARG, now);
      continue;
    }
    if (blocked) {
      kept_new.insert(q.r.image_id);
      keep.push_back(std::move(q));
      continue;
    }
    const uint64_t t = tiles_of(q.r.img.width, q.r.img.height);
    if (t > s->max_tiles || (uint64_t)(q.r.img.height + 31) / 32 >= (1ull << LIVE_CHUNK_BITS)) {
      complete(s, q, DTB_ERR_CAPACITY, now);
      continue;
    }
    if (L->flight_tiles + t > s->max_tiles) {
      blocked = true;
      kept_new.insert(q.r.image_id);
      keep.push_back(std::move(q));
      continue;
    }
    Resident r;
    r.W = q.r.img.width;
    r.H = q.r.img.height;
    r.C = q.r.img.elem_size;
    r.g2 = gamma_to_g2(q.r.gamma);
    r.img_pitch = (int64_t)plane_pitch((size_t)r.W * r.C);
    r.mask_pitch = (int64_t)plane_pitch((size_t)r.W);
    r.dist_pitch = (int64_t)align_up(4 * (size_t)std::max(r.W, 1), 128);
    r.o_img = 0;
    r.o_mask = align_up((size_t)r.img_pitch * r.H, 256);
    r.o_dist = r.o_mask + align_up((size_t)r.mask_pitch * r.H, 256);
    r.bytes = r.o_dist + align_up((size_t)r.dist_pitch * r.H, 256);
    if (r.bytes > s->cfg.hbm_budget_bytes || t > L->tile_cap) {
      complete(s, q, DTB_ERR_CAPACITY, now);
      continue;
    }
    size_t off = 0;
    if (!make_room(s, r.bytes, &off)) {
      blocked = true;
      kept_new.insert(q.r.image_id);
      keep.push_back(std::move(q));
      continue;
    }
    r.off = off;
    if (!live_place(s, (uint32_t)t, &r.slot, &r.tile_base)) {
      s->arena.release(off, r.bytes);
      blocked = true;
      kept_new.insert(q.r.image_id);
      keep.push_back(std::move(q));
      continue;
    }
    r.tiles = (uint32_t)t;
    r.wave = 0;
    r.last_use = ++s->tick;
    s->resident[q.r.image_id] = r;
    L->flight_tiles += t;
    LiveFlight f;
    f.q = std::move(q);
    out.push_back(std::move(f));
  }
  s->pending = std::move(keep);
  return out;
}

// Copies one admitted request in and publishes it (s_in, in order: data, descriptor + maps, entry, count).  The
// caller holds the context's lock.
dtb_status live_publish(dtb_server s, LiveFlight& f, const Resident& r) {
  const TraceRange trace("dtb live publish");
  dtb_context ctx = s->ctx;
  LiveEngine* L = s->live;
  cudaStream_t st = s->s_in;
  const uint32_t e = L->next_entry;
  uint8_t* stg = L->hstage + LIVE_STAGE * (e & (LIVE_RING - 1u));
  LiveEntry* ent = reinterpret_cast<LiveEntry*>(stg + LST_ENTRY);
  std::memset(ent, 0, sizeof(LiveEntry));
  ent->slot = (uint32_t)r.slot;
  uint8_t* base = s->arena_base + r.off;
  const dtb_serve_request& q = f.q.r;
  if (q.kind == DTB_REQ_IMAGE) {
    ent->kind = LIVE_NEW;
    const size_t rb = (size_t)r.W * r.C;
    if (r.W > 0 && r.H > 0) {
      // Planes whose rows need a new pitch go in packed, as one 1-D copy, into the image's distance plane, and the
      // kernel's set-up jobs move the rows into place (a 2-D copy that changes the pitch runs at 12-30 GB/s
      // against 47-54 GB/s for a 1-D copy); if the host rows are padded themselves, or the staging does not fit,
      // a 2-D copy goes straight into place.
      bool st_img = (size_t)r.img_pitch != rb && (size_t)q.img.pitch == rb;
      bool st_mask = r.mask_pitch != r.W && q.mask.pitch == r.W;
      const uint64_t o_mask_st = st_img ? live_stage_mask_offset((uint32_t)rb, (uint32_t)r.H) : 0;
      const uint64_t need = o_mask_st + (st_mask ? (uint64_t)r.W * r.H : 0) + LIVE_STAGE_SLACK;
      if (need > (uint64_t)r.dist_pitch * r.H) st_img = st_mask = false;
      uint8_t* stage = base + r.o_dist;
      ent->stage = (st_img ? LIVE_STAGE_IMG : 0u) | (st_mask ? LIVE_STAGE_MASK : 0u);
      if (st_img)
        DTB_CUDA(ctx, cudaMemcpyAsync(stage, q.img.buffer, rb * r.H, cudaMemcpyHostToDevice, st));
      else if ((size_t)q.img.pitch == rb && (size_t)r.img_pitch == rb)
        DTB_CUDA(ctx, cudaMemcpyAsync(base + r.o_img, q.img.buffer, rb * r.H, cudaMemcpyHostToDevice, st));
      else
        DTB_CUDA(ctx, cudaMemcpy2DAsync(base + r.o_img, r.img_pitch, q.img.buffer, q.img.pitch, rb, r.H,
                                        cudaMemcpyHostToDevice, st));
      if (st_mask)
        DTB_CUDA(ctx, cudaMemcpyAsync(stage + (st_img ? o_mask_st : 0), q.mask.buffer, (size_t)r.W * r.H,
                                      cudaMemcpyHostToDevice, st));
      else if (q.mask.pitch == r.W && r.mask_pitch == r.W)
        DTB_CUDA(ctx, cudaMemcpyAsync(base + r.o_mask, q.mask.buffer, (size_t)r.W * r.H, cudaMemcpyHostToDevice, st));
      else
        DTB_CUDA(ctx, cudaMemcpy2DAsync(base + r.o_mask, r.mask_pitch, q.mask.buffer, q.mask.pitch, r.W, r.H,
                                        cudaMemcpyHostToDevice, st));
    }
    Job j;
    j.img = base + r.o_img;
    j.img_pitch = r.img_pitch;
    j.channels = r.C;
    j.mask = base + r.o_mask;
    j.mask_pitch = r.mask_pitch;
    j.dist = reinterpret_cast<float*>(base + r.o_dist);
    j.dist_pitch = r.dist_pitch;
    j.width = r.W;
    j.height = r.H;
    j.g2 = r.g2;
    j.v = s->cfg.v;
    j.mode = MODE_NS;
    ImgDesc* d = reinterpret_cast<ImgDesc*>(stg + LST_DESC);
    CUtensorMap* tm = reinterpret_cast<CUtensorMap*>(stg + LST_TMAP);
    std::memset(stg, 0, LST_ENTRY);
    dtb_status ds = fill_desc(ctx, j, r.tile_base, 0, d, tm);
    if (ds != DTB_OK) return ds;
    DTB_CUDA(ctx, cudaMemcpyAsync(L->descs + r.slot, d, sizeof(ImgDesc), cudaMemcpyHostToDevice, st));
    DTB_CUDA(ctx, cudaMemcpyAsync(L->tmaps + 2 * r.slot, tm, 2 * sizeof(CUtensorMap), cudaMemcpyHostToDevice, st));
  } else {
    ent->kind = LIVE_EDIT;
    const size_t nd = f.q.disks.size() / 3;
    ent->n_disks = (uint32_t)nd;
    if (nd) {
      // 16-byte records: pool offsets (multiples of the arena's 256-byte granule) are whole records.
      ent->disk_idx = (uint32_t)(f.disk_off / LIVE_DISK_BYTES);
      int32_t* hd = L->hdisks + f.disk_off / 4;
      for (size_t k = 0; k < nd; ++k) {
        hd[4 * k] = f.q.disks[3 * k];
        hd[4 * k + 1] = f.q.disks[3 * k + 1];
        hd[4 * k + 2] = f.q.disks[3 * k + 2];
        hd[4 * k + 3] = 0;
      }
      DTB_CUDA(ctx, cudaMemcpyAsync(reinterpret_cast<uint8_t*>(L->disks) + f.disk_off, hd, LIVE_DISK_BYTES * nd,
                                    cudaMemcpyHostToDevice, st));
    }
  }
  // dtb_debug_inject_queue_stall on the server's context: the next request the kernel claims counts one item
  // that never runs, under the injected no-progress limit (the caller holds ctx->mu).
  if (ctx->inject_stall_ns) {
    L->hwords[2] = (uint32_t)std::max<uint64_t>(1, ctx->inject_stall_ns / 1000000ull);
    ctx->inject_stall_ns = 0;
    DTB_CUDA(ctx, cudaMemcpyAsync(&L->lh->watch_ms.v, &L->hwords[2], 4, cudaMemcpyHostToDevice, st));
    DTB_CUDA(ctx, cudaMemcpyAsync(&L->lh->inject.v, &L->hwords[0], 4, cudaMemcpyHostToDevice, st));
  }
  DTB_CUDA(ctx, cudaMemcpyAsync(L->entries + (e & (LIVE_RING - 1u)), ent, sizeof(LiveEntry), cudaMemcpyHostToDevice, st));
  uint32_t* pub = reinterpret_cast<uint32_t*>(stg + LST_PUB);
  *pub = e + 1u;
  DTB_CUDA(ctx, cudaMemcpyAsync(&L->lh->published.v, pub, 4, cudaMemcpyHostToDevice, st));
  f.entry = e;
  L->next_entry = e + 1u;
  return DTB_OK;
}

// Launches the live kernel (queue header and ring reset first, on the tile-run stream).
dtb_status live_launch(dtb_server s) {
  const TraceRange trace("dtb live launch");
  dtb_context ctx = s->ctx;
  LiveEngine* L = s->live;
  cudaStream_t st = s->s_run;
  DTB_CUDA(ctx, cudaMemsetAsync(L->qhdr, 0, sizeof(QueueHdr), st));
  DTB_CUDA(ctx, cudaMemsetAsync(L->ring, 0, 4ull * L->ring_cap, st));
  DTB_CUDA(ctx, cudaMemsetAsync(&L->lh->end_reason.v, 0, 4, st));
  LiveArgs a{};
  a.q.hdr = L->qhdr;
  a.q.ring = L->ring;
  a.q.mask = L->ring_cap - 1u;
  a.q.timeout_ns = (uint64_t)LIVE_WATCH_MS * 1000000ull;
  a.q.max_visits = 0xF0000000u;
  a.q.total_tiles = L->tile_cap;
  a.states = L->states;
  a.descs = L->descs;
  a.tmaps = L->tmaps;
  a.lh = L->lh;
  a.slots = L->slots;
  a.entries = L->entries;
  a.disks = L->disks;
  a.host_done = L->ddone;
  a.nslots = L->nslots;
  a.disk_cap = LIVE_DISK_CAP;
  a.idle_us = L->idle_us;
  a.life_us = LIVE_LIFE_US;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(L->grid);
  cfg.blockDim = dim3(PERSIST_WPC * 32);
  cfg.dynamicSmemBytes = PERSIST_SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;  // co-residency of all workers (the slot waits need it)
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[1] = {(void*)&a};
  DTB_CUDA(ctx, cudaLaunchKernelExC(&cfg, (const void*)ggdt_live<PERSIST_WPC, LIVE_CTAS>, args));
  DTB_CUDA(ctx, cudaEventRecord(L->ev_kernel, st));
  L->running = true;
  return DTB_OK;
}

// A launch has ended: its error (if any) fails the requests it claimed and did not finish (their images are
// dropped: their tile states are not trustworthy); unclaimed requests stay for the next launch.
void live_after_kernel(dtb_server s) {
  dtb_context ctx = s->ctx;
  LiveEngine* L = s->live;
  L->running = false;
  QueueHdr h{};
  LiveHdr lhh{};
  dtb_status status = DTB_OK;
  if (cudaEventSynchronize(L->ev_kernel) != cudaSuccess ||
      cudaMemcpy(&h, L->qhdr, sizeof(QueueHdr), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&lhh, L->lh, sizeof(LiveHdr), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    status = DTB_ERR_CUDA;
  } else if (h.error.v) {
    status = h.error.v == DERR_QUEUE_TIMEOUT || h.error.v == DERR_TMA_TIMEOUT || h.error.v == DERR_RING_FULL
                 ? DTB_ERR_TIMEOUT
                 : DTB_ERR_DEVICE;
    std::lock_guard<std::mutex> ctx_lock(ctx->mu);
    fail(ctx, status, "serve (live): device error %u (detail %u)", h.error.v, h.err_info.v);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->st.tile_visits += h.progress.v;
  L->claimed_seen = lhh.claimed.v;
  if (status != DTB_OK) s->st.live_ended_error += 1;
  else if (lhh.end_reason.v == LIVE_END_IDLE) s->st.live_ended_idle += 1;
  else if (lhh.end_reason.v == LIVE_END_LIFE) s->st.live_ended_lifetime += 1;
  else if (lhh.end_reason.v == LIVE_END_STOP) s->st.live_ended_stop += 1;
  if (status == DTB_OK) return;
  // Requests claimed by the failed launch (entries below `claimed`) whose completion word is not written fail.
  const auto now = Clock::now();
  for (auto it = L->flights.begin(); it != L->flights.end();) {
    LiveFlight& f = *it;
    const bool claimed = status == DTB_ERR_CUDA || (int32_t)(lhh.claimed.v - f.entry) > 0;
    const bool finished = L->hdone[f.entry & (LIVE_RING - 1u)] == f.entry + 1u;
    if (f.stage != 0 || !claimed || finished) {
      ++it;
      continue;
    }
    auto r = s->resident.find(f.q.r.image_id);
    if (r != s->resident.end()) {
      L->flight_tiles -= r->second.tiles;
      drop_resident(s, r);
    }
    if (f.disk_off != SIZE_MAX) L->diskpool.release(f.disk_off, f.disk_bytes);
    complete(s, f.q, status, now);
    it = L->flights.erase(it);
  }
  // The next launch starts from the default watchdog limit.
  if (cudaMemcpyAsync(&L->lh->watch_ms.v, &L->hwords[1], 4, cudaMemcpyHostToDevice, s->s_run) != cudaSuccess)
    cudaGetLastError();
  s->cv_done.notify_all();
}

void live_worker_main(dtb_server s) {
  cudaSetDevice(s->ctx->device);
  LiveEngine* L = s->live;
  for (;;) {
    std::vector<LiveFlight> adm;
    std::vector<Resident> rs;
    Clock::time_point t0 = Clock::now();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->stop && s->pending.empty() && L->flights.empty()) break;
      adm = live_admit_host(s);
      for (LiveFlight& f : adm) {
        rs.push_back(s->resident[f.q.r.image_id]);
        const double w = std::chrono::duration<double, std::milli>(t0 - f.q.t_submit).count();
        s->st.queue_wait_ms += w;
        s->st.queue_wait_max_ms = std::max(s->st.queue_wait_max_ms, w);
      }
      if (!adm.empty()) s->cv_done.notify_all();  // admission may have completed invalid requests
    }
    bool progress = !adm.empty();
    // Publish the admitted requests.
    for (size_t i = 0; i < adm.size(); ++i) {
      dtb_status ps;
      {
        std::lock_guard<std::mutex> ctx_lock(s->ctx->mu);
        ps = live_publish(s, adm[i], rs[i]);
      }
      adm[i].t_pub = Clock::now();
      std::lock_guard<std::mutex> lk(s->mu);
      s->st.host_prep_ms += std::chrono::duration<double, std::milli>(adm[i].t_pub - t0).count() / (double)adm.size();
      if (ps != DTB_OK) {
        // Nothing was published for it (the count is copied last); its copies in may still run: wait for them.
        cudaStreamSynchronize(s->s_in);
        auto r = s->resident.find(adm[i].q.r.image_id);
        if (r != s->resident.end()) {
          L->flight_tiles -= r->second.tiles;
          if (adm[i].q.r.kind == DTB_REQ_IMAGE) drop_resident(s, r);
          else r->second.wave = -1;
        }
        if (adm[i].disk_off != SIZE_MAX) L->diskpool.release(adm[i].disk_off, adm[i].disk_bytes);
        complete(s, adm[i].q, ps, Clock::now());
        s->cv_done.notify_all();
        continue;
      }
      L->flights.push_back(std::move(adm[i]));
    }
    // The kernel: notice its end; launch it while published requests wait.
    if (L->running && cudaEventQuery(L->ev_kernel) != cudaErrorNotReady) {
      live_after_kernel(s);
      progress = true;
    }
    if (!L->running) {
      bool waiting = false;
      for (const LiveFlight& f : L->flights)
        if (f.stage == 0 && L->hdone[f.entry & (LIVE_RING - 1u)] != f.entry + 1u) waiting = true;
      if (waiting) {
        dtb_status ls;
        {
          std::lock_guard<std::mutex> ctx_lock(s->ctx->mu);
          ls = live_launch(s);
        }
        if (ls == DTB_OK) {
          std::lock_guard<std::mutex> lk(s->mu);
          s->st.waves += 1;  // launches of the live kernel
        } else {
          // Could not launch: fail the requests that wait for it.
          cudaStreamSynchronize(s->s_in);
          std::lock_guard<std::mutex> lk(s->mu);
          for (auto it = L->flights.begin(); it != L->flights.end();) {
            if (it->stage != 0) { ++it; continue; }
            auto r = s->resident.find(it->q.r.image_id);
            if (r != s->resident.end()) {
              L->flight_tiles -= r->second.tiles;
              drop_resident(s, r);
            }
            if (it->disk_off != SIZE_MAX) L->diskpool.release(it->disk_off, it->disk_bytes);
            complete(s, it->q, ls, Clock::now());
            it = L->flights.erase(it);
          }
          s->cv_done.notify_all();
        }
        progress = true;
      }
    }
    // Finished maps: copy out.
    for (LiveFlight& f : L->flights) {
      if (f.stage != 0 || L->hdone[f.entry & (LIVE_RING - 1u)] != f.entry + 1u) continue;
      f.t_seen = Clock::now();
      std::lock_guard<std::mutex> lk(s->mu);
      const Resident& r = s->resident[f.q.r.image_id];
      const dtb_image& o = f.q.r.out;
      if (L->ev_free.empty()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) cudaGetLastError();
        L->ev_free.push_back(e);
      }
      f.ev = L->ev_free.back();
      L->ev_free.pop_back();
      bool ok = f.ev != nullptr;
      if (ok && o.width > 0 && o.height > 0)
        ok = cudaMemcpy2DAsync(o.buffer, o.pitch, s->arena_base + r.off + r.o_dist, r.dist_pitch, 4 * (size_t)o.width,
                               o.height, cudaMemcpyDeviceToHost, s->s_out) == cudaSuccess;
      ok = ok && cudaEventRecord(f.ev, s->s_out) == cudaSuccess;
      if (!ok) {
        cudaGetLastError();
        if (f.ev) L->ev_free.push_back(f.ev);
        f.ev = nullptr;
      }
      f.stage = 1;
      progress = true;
    }
    // Copies out that ended: the request completes and its image is free for the next request.
    for (auto it = L->flights.begin(); it != L->flights.end();) {
      LiveFlight& f = *it;
      if (f.stage != 1) { ++it; continue; }
      dtb_status status = DTB_OK;
      if (f.ev) {
        const cudaError_t q = cudaEventQuery(f.ev);
        if (q == cudaErrorNotReady) { ++it; continue; }
        if (q != cudaSuccess) { cudaGetLastError(); status = DTB_ERR_CUDA; }
        L->ev_free.push_back(f.ev);
      } else {
        status = DTB_ERR_CUDA;
      }
      const auto now = Clock::now();
      std::lock_guard<std::mutex> lk(s->mu);
      auto r = s->resident.find(f.q.r.image_id);
      if (r != s->resident.end()) {
        L->flight_tiles -= r->second.tiles;
        s->st.tiles += r->second.tiles;
        r->second.wave = -1;
        if (status != DTB_OK && f.q.r.kind == DTB_REQ_IMAGE) drop_resident(s, r);
      }
      if (f.disk_off != SIZE_MAX) L->diskpool.release(f.disk_off, f.disk_bytes);
      s->st.kernel_ms += std::chrono::duration<double, std::milli>(f.t_seen - f.t_pub).count();
      s->st.copy_out_ms += std::chrono::duration<double, std::milli>(now - f.t_seen).count();
      complete(s, f.q, status, now);
      s->cv_done.notify_all();
      it = L->flights.erase(it);
      progress = true;
    }
    if (!progress) {
      std::unique_lock<std::mutex> lk(s->mu);
      const bool idle = L->flights.empty() && !L->running;
      if (idle) s->cv_sub.wait(lk, [&] { return s->stop || !s->pending.empty(); });
      else s->cv_sub.wait_for(lk, std::chrono::microseconds(20));
    }
  }
  // Ask a running kernel to end, and wait for it (bounded by its idle time).
  if (L->running) {
    if (cudaMemcpyAsync(&L->lh->stop.v, &L->hwords[0], 4, cudaMemcpyHostToDevice, s->s_in) != cudaSuccess) cudaGetLastError();
    live_after_kernel(s);
  }
}

}  // namespace

namespace {

// Frees the server's device and host resources (no wave in flight).
void release_server(dtb_server s) {
  for (WaveSlot& w : s->slot) {
    if (w.scratch) cudaFree(w.scratch);
    if (w.stage) cudaFree(w.stage);
    if (w.hpin) cudaFreeHost(w.hpin);
    for (cudaEvent_t e : {w.ev_in, w.ev_comp, w.ev_done, w.t_in0, w.t_in1, w.t_run0, w.t_run1, w.t_out0, w.t_out1})
      if (e) cudaEventDestroy(e);
  }
  live_destroy(s->live);
  for (cudaStream_t t : {s->s_in, s->s_run, s->s_out})
    if (t) cudaStreamDestroy(t);
  if (s->arena_base) cudaFree(s->arena_base);
  delete s;
}

}  // namespace

extern "C" {

DTB_API dtb_status dtb_serve_create(dtb_context ctx, const dtb_serve_config* cfg, dtb_server* out) {
  if (!ctx || !cfg || !out || cfg->hbm_budget_bytes == 0 || !(cfg->v >= 0.0f) || cfg->max_wave_requests < 0 ||
      cfg->max_wave_tiles > (1u << 26) || (cfg->live != 0 && cfg->live != 1))
    return DTB_ERR_INVALID_ARG;
  *out = nullptr;
  dtb_server s = new (std::nothrow) dtb_server_s();
  if (!s) return DTB_ERR_OUT_OF_MEMORY;
  s->ctx = ctx;
  s->cfg = *cfg;
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    delete s;
    return DTB_ERR_CUDA;
  }
  if (cudaMalloc((void**)&s->arena_base, cfg->hbm_budget_bytes) != cudaSuccess) {
    delete s;
    return DTB_ERR_OUT_OF_MEMORY;
  }
  s->arena.reset(cfg->hbm_budget_bytes);
  bool ok = cudaStreamCreateWithFlags(&s->s_in, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&s->s_run, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&s->s_out, cudaStreamNonBlocking) == cudaSuccess;
  for (WaveSlot& w : s->slot) {
    ok = ok && cudaEventCreateWithFlags(&w.ev_in, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&w.ev_comp, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&w.ev_done, cudaEventDisableTiming) == cudaSuccess;
    for (cudaEvent_t* e : {&w.t_in0, &w.t_in1, &w.t_run0, &w.t_run1, &w.t_out0, &w.t_out1})
      ok = ok && cudaEventCreate(e) == cudaSuccess;
  }
  if (!ok) {
    release_server(s);
    return DTB_ERR_CUDA;
  }
  // Per-wave buffers for the largest wave the limits admit: scratch (run layout for max_reqs images and
  // max_tiles tiles with every launch variant's workers, plus warm flags, disks and repitch items), staging and
  // the pinned tables.
  s->max_reqs = cfg->max_wave_requests > 0 ? cfg->max_wave_requests : SERVE_MAX_WAVE_REQUESTS;
  s->max_tiles = cfg->max_wave_tiles > 0 ? cfg->max_wave_tiles : SERVE_MAX_WAVE_TILES;
  s->stage_cap = cfg->wave_stage_bytes > 0 ? (size_t)cfg->wave_stage_bytes : (size_t)SERVE_WAVE_STAGE_BYTES;
  if (cfg->live) {
    // Live admission: the live kernel's tables, ring and pinned buffers instead of per-wave slots.
    const dtb_status ls = live_create(s, cfg->live_idle_us);
    if (ls != DTB_OK) {
      release_server(s);
      return ls;
    }
    s->worker = std::thread(live_worker_main, s);
    *out = s;
    return DTB_OK;
  }
  for (int k = 0; k < NS_VARIANTS; ++k) {
    LaunchTuning t = ctx->tuning;
    t.variant = k;
    t.grid_percent = 100;
    s->workers = std::max(s->workers, resident_workers(ctx, MODE_NS, t));
  }
  s->nb = (uint32_t)ctx->tuning.buckets;
  const ScratchLayout Lmax = layout_for(s->max_reqs, s->max_tiles, s->workers, false, s->nb);
  size_t o_warm = 0, o_disks = 0, o_items = 0;
  const size_t scratch = wave_scratch_bytes(Lmax, s->max_reqs, SERVE_MAX_WAVE_DISKS, 2 * (size_t)s->max_reqs, &o_warm,
                                            &o_disks, &o_items);
  for (WaveSlot& w : s->slot) {
    ok = ok && cudaMalloc(&w.scratch, scratch) == cudaSuccess && cudaMalloc(&w.stage, s->stage_cap) == cudaSuccess &&
         cudaHostAlloc((void**)&w.hpin, scratch - Lmax.o_desc, cudaHostAllocDefault) == cudaSuccess;
    if (!ok) break;
    w.scratch_size = scratch;
    w.stage_size = s->stage_cap;
    w.hpin_size = scratch - Lmax.o_desc;
  }
  if (!ok) {
    cudaGetLastError();
    release_server(s);
    return DTB_ERR_OUT_OF_MEMORY;
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return DTB_OK;
}

DTB_API dtb_status dtb_serve_submit(dtb_server s, const dtb_serve_request* r, int64_t* request_id) {
  if (!s || !r) return DTB_ERR_INVALID_ARG;
  if (r->kind != DTB_REQ_IMAGE && r->kind != DTB_REQ_EDIT) return DTB_ERR_INVALID_ARG;
  const dtb_image& o = r->out;
  if (o.elem_size != 4 || o.memory_kind != DTB_CPU || (o.width > 0 && o.height > 0 && (!o.buffer || o.pitch < 4 * o.width)))
    return DTB_ERR_INVALID_ARG;
  if (r->kind == DTB_REQ_IMAGE) {
    const dtb_image& i = r->img;
    const dtb_image& m = r->mask;
    if ((i.elem_size != 1 && i.elem_size != 3) || m.elem_size != 1 || i.memory_kind != DTB_CPU || m.memory_kind != DTB_CPU)
      return DTB_ERR_INVALID_ARG;
    if (i.width < 0 || i.height < 0 || i.width != m.width || i.height != m.height || i.width != o.width ||
        i.height != o.height)
      return DTB_ERR_INVALID_ARG;
    if (i.width > 0 && i.height > 0 &&
        (!i.buffer || !m.buffer || i.pitch < i.width * i.elem_size || m.pitch < m.width))
      return DTB_ERR_INVALID_ARG;
    if (!(r->gamma >= 0.0f) || std::isinf(r->gamma)) return DTB_ERR_INVALID_ARG;
  } else {
    if (r->n_disks < 0 || (r->n_disks > 0 && !r->disks)) return DTB_ERR_INVALID_ARG;
    if ((size_t)r->n_disks > SERVE_MAX_WAVE_DISKS) return DTB_ERR_CAPACITY;
  }
  Request q;
  q.r = *r;
  if (r->kind == DTB_REQ_EDIT) q.disks.assign(r->disks, r->disks + 3 * (size_t)r->n_disks);
  q.r.disks = nullptr;
  q.t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return DTB_ERR_INVALID_ARG;
    q.rid = s->next_rid++;
    if (request_id) *request_id = q.rid;
    s->pending.push_back(std::move(q));
    s->st.submitted += 1;
  }
  s->cv_sub.notify_one();
  return DTB_OK;
}

DTB_API int32_t dtb_serve_poll(dtb_server s, dtb_serve_completion* out, int32_t max, int32_t wait_ms) {
  if (!s || !out || max <= 0) return 0;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && wait_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
  int32_t k = 0;
  while (k < max && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  return k;
}

DTB_API dtb_status dtb_serve_release(dtb_server s, int64_t image_id) {
  if (!s) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->resident.find(image_id);
  if (it == s->resident.end() || it->second.wave >= s->busy_from || referenced(s, image_id)) return DTB_ERR_INVALID_ARG;
  drop_resident(s, it);
  return DTB_OK;
}

DTB_API dtb_status dtb_serve_get_stats(dtb_server s, dtb_serve_stats* out) {
  if (!s || !out) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident_images = (int64_t)s->resident.size();
  uint64_t b = 0;
  for (auto& kv : s->resident) b += kv.second.bytes;
  out->resident_bytes = b;
  out->pending = (int64_t)s->pending.size();
  return DTB_OK;
}

DTB_API void dtb_serve_destroy(dtb_server s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_sub.notify_all();
  if (s->worker.joinable()) s->worker.join();
  release_server(s);
}

}  // extern "C"
