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
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "dtb.h"
#include "dtb_internal.h"
#include "dtb_kernels.cuh"

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
  int64_t wave = -1;  // wave the image takes part in (busy while it runs)
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

// Makes room for `bytes` in the arena by evicting least-recently-used idle residents.  Caller holds mu.
bool make_room(dtb_server s, size_t bytes, size_t* off) {
  while (!s->arena.alloc(bytes, off)) {
    int64_t victim = 0;
    uint64_t oldest = UINT64_MAX;
    bool found = false;
    for (auto& kv : s->resident) {
      if (kv.second.wave >= s->busy_from || referenced(s, kv.first)) continue;
      if (kv.second.last_use < oldest) {
        oldest = kv.second.last_use;
        victim = kv.first;
        found = true;
      }
    }
    if (!found) return false;
    s->arena.release(s->resident[victim].off, s->resident[victim].bytes);
    s->resident.erase(victim);
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
      if (it != s->resident.end()) {
        s->arena.release(it->second.off, it->second.bytes);
        s->resident.erase(it);
      }
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

// Frees the server's device and host resources (no wave in flight).
void release_server(dtb_server s) {
  for (WaveSlot& w : s->slot) {
    if (w.scratch) cudaFree(w.scratch);
    if (w.stage) cudaFree(w.stage);
    if (w.hpin) cudaFreeHost(w.hpin);
    for (cudaEvent_t e : {w.ev_in, w.ev_comp, w.ev_done, w.t_in0, w.t_in1, w.t_run0, w.t_run1, w.t_out0, w.t_out1})
      if (e) cudaEventDestroy(e);
  }
  for (cudaStream_t t : {s->s_in, s->s_run, s->s_out})
    if (t) cudaStreamDestroy(t);
  if (s->arena_base) cudaFree(s->arena_base);
  delete s;
}

}  // namespace

extern "C" {

DTB_API dtb_status dtb_serve_create(dtb_context ctx, const dtb_serve_config* cfg, dtb_server* out) {
  if (!ctx || !cfg || !out || cfg->hbm_budget_bytes == 0 || !(cfg->v >= 0.0f) || cfg->max_wave_requests < 0 ||
      cfg->max_wave_tiles > (1u << 26))
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
  s->arena.release(it->second.off, it->second.bytes);
  s->resident.erase(it);
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
