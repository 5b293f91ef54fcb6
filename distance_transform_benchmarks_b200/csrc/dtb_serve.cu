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

}  // namespace

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
  void* wscratch = nullptr;
  size_t wscratch_size = 0;
  void* wstage = nullptr;
  size_t wstage_size = 0;
  std::vector<uint8_t> host;
  cudaStream_t stream = nullptr;
  dtb_serve_stats st{};
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
      if (kv.second.wave == s->wave_no || referenced(s, kv.first)) continue;
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

// Admission of one wave (caller holds mu).  Requests that cannot run now stay pending in order.
std::vector<Request> admit(dtb_server s) {
  std::vector<Request> wave;
  std::deque<Request> keep;
  const auto now = Clock::now();
  bool blocked = false;  // a new image that did not fit keeps later new images waiting (arrival order)
  while (!s->pending.empty()) {
    Request q = std::move(s->pending.front());
    s->pending.pop_front();
    if (s->cfg.max_wave_requests > 0 && (int32_t)wave.size() >= s->cfg.max_wave_requests) {
      keep.push_back(std::move(q));
      continue;
    }
    auto it = s->resident.find(q.r.image_id);
    if (q.r.kind == DTB_REQ_EDIT) {
      if (it == s->resident.end()) {
        complete(s, q, DTB_ERR_INVALID_ARG, now);  // not resident (never submitted, released or evicted)
        continue;
      }
      if (it->second.wave == s->wave_no) {
        keep.push_back(std::move(q));  // one request per image per wave
        continue;
      }
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
    wave.push_back(std::move(q));
  }
  s->pending = std::move(keep);
  return wave;
}

dtb_status run_wave(dtb_server s, std::vector<Request>& wave) {
  dtb_context ctx = s->ctx;
  cudaStream_t st = s->stream;
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
  dtb_status s2 = grow(ctx, &s->wstage, &s->wstage_size, std::max<size_t>(stage_bytes, 256));
  if (s2 != DTB_OK) return s2;
  uint8_t* stage = static_cast<uint8_t*>(s->wstage);
  // Host -> device: one 1-D copy per plane (into the resident plane, or into staging + repitch).
  for (int i = 0; i < n; ++i) {
    if (warm[i]) continue;
    const dtb_serve_request& q = wave[i].r;
    Resident& r = *rs[i];
    const size_t rb = (size_t)r.W * r.C;
    uint8_t* dimg = o_stage_img[i] == SIZE_MAX ? const_cast<uint8_t*>(jobs[i].img) : stage + o_stage_img[i];
    uint8_t* dmask = o_stage_mask[i] == SIZE_MAX ? const_cast<uint8_t*>(jobs[i].mask) : stage + o_stage_mask[i];
    if ((size_t)q.img.pitch == rb)
      DTB_CUDA(ctx, cudaMemcpyAsync(dimg, q.img.buffer, rb * r.H, cudaMemcpyHostToDevice, st));
    else
      DTB_CUDA(ctx, cudaMemcpy2DAsync(dimg, rb, q.img.buffer, q.img.pitch, rb, r.H, cudaMemcpyHostToDevice, st));
    if (q.mask.pitch == r.W)
      DTB_CUDA(ctx, cudaMemcpyAsync(dmask, q.mask.buffer, (size_t)r.W * r.H, cudaMemcpyHostToDevice, st));
    else
      DTB_CUDA(ctx, cudaMemcpy2DAsync(dmask, r.W, q.mask.buffer, q.mask.pitch, r.W, r.H, cudaMemcpyHostToDevice, st));
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
  const LaunchTuning tuning = ctx->tuning;
  const ScratchLayout L = layout_for(n, total, resident_workers(ctx, MODE_NS, tuning), false);
  size_t off = L.bytes;
  const size_t o_warm = off;
  off = align_up(off + (size_t)std::max(n, 1), 256);
  const size_t o_disks = off;
  off = align_up(off + sizeof(DiskItem) * std::max<size_t>(disks.size(), 1), 256);
  const size_t o_items = off;
  off = align_up(off + sizeof(RepitchItem) * std::max<size_t>(items.size(), 1), 256);
  if ((s2 = grow(ctx, &s->wscratch, &s->wscratch_size, off)) != DTB_OK) return s2;
  uint8_t* sc = static_cast<uint8_t*>(s->wscratch);
  std::vector<uint8_t> tab;
  if ((s2 = build_tables(ctx, jobs, L, tab)) != DTB_OK) return s2;
  s->host.assign(off - L.o_desc, 0);
  std::copy(tab.begin(), tab.end(), s->host.begin());
  std::copy(warm.begin(), warm.end(), s->host.begin() + (o_warm - L.o_desc));
  std::copy(reinterpret_cast<const uint8_t*>(disks.data()), reinterpret_cast<const uint8_t*>(disks.data() + disks.size()),
            s->host.begin() + (o_disks - L.o_desc));
  std::copy(reinterpret_cast<const uint8_t*>(items.data()), reinterpret_cast<const uint8_t*>(items.data() + items.size()),
            s->host.begin() + (o_items - L.o_desc));
  DTB_CUDA(ctx, cudaMemcpyAsync(sc + L.o_desc, s->host.data(), s->host.size(), cudaMemcpyHostToDevice, st));
  const dtb_status qs = reset_queue(ctx, sc, L, st);
  if (qs != DTB_OK) return qs;
  const ImgDesc* ddesc = reinterpret_cast<const ImgDesc*>(sc + L.o_desc);
  const CUtensorMap* dtm = reinterpret_cast<const CUtensorMap*>(sc + L.o_tmap);
  const uint32_t* dbase = reinterpret_cast<const uint32_t*>(sc + L.o_base);
  uint32_t* states = reinterpret_cast<uint32_t*>(sc + L.o_states);
  Queue q = make_queue(sc, L);
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
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(resident_workers(ctx, MODE_NS, tuning) / PERSIST_WPC);
    cfg.blockDim = dim3(PERSIST_WPC * 32);
    cfg.dynamicSmemBytes = PERSIST_SMEM;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[4] = {(void*)&ddesc, (void*)&dtm, (void*)&states, (void*)&q};
    DTB_CUDA(ctx, cudaLaunchKernelExC(&cfg, ctx->ns_fn[tuning.variant], args));
    ggdt_finalize<<<blocks, 128, 0, st>>>(ddesc, dbase, n, total, states);
    DTB_CUDA(ctx, cudaGetLastError());
  }
  // Device -> host: each request's map into its output buffer.
  for (int i = 0; i < n; ++i) {
    const dtb_image& o = wave[i].r.out;
    if (o.width == 0 || o.height == 0) continue;
    DTB_CUDA(ctx, cudaMemcpy2DAsync(o.buffer, o.pitch, jobs[i].dist, jobs[i].dist_pitch, 4 * (size_t)o.width, o.height,
                                    cudaMemcpyDeviceToHost, st));
  }
  DTB_CUDA(ctx, cudaStreamSynchronize(st));
  dtb_stats ds{};
  const dtb_status status = read_device_status(ctx, reinterpret_cast<QueueHdr*>(sc + L.o_hdr), &ds);
  s->st.tile_visits += ds.tile_visits;
  s->st.tiles += total;
  return status;
}

void worker_main(dtb_server s) {
  cudaSetDevice(s->ctx->device);
  for (;;) {
    std::vector<Request> wave;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_sub.wait(lk, [&] { return s->stop || !s->pending.empty(); });
      if (s->stop && s->pending.empty()) break;
      ++s->wave_no;
      wave = admit(s);
      if (wave.empty()) {
        s->cv_done.notify_all();
        if (!s->pending.empty()) {
          // nothing fits right now and nothing runs: the head request can never fit
          complete(s, s->pending.front(), DTB_ERR_CAPACITY, Clock::now());
          s->pending.pop_front();
        }
        continue;
      }
    }
    const dtb_status status = run_wave(s, wave);
    const auto now = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.waves += 1;
    for (const Request& q : wave) {
      if (status != DTB_OK && q.r.kind == DTB_REQ_IMAGE) {
        auto it = s->resident.find(q.r.image_id);  // its map is not valid: drop the image
        if (it != s->resident.end()) {
          s->arena.release(it->second.off, it->second.bytes);
          s->resident.erase(it);
        }
      }
      complete(s, q, status, now);
    }
    s->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

DTB_API dtb_status dtb_serve_create(dtb_context ctx, const dtb_serve_config* cfg, dtb_server* out) {
  if (!ctx || !cfg || !out || cfg->hbm_budget_bytes == 0 || !(cfg->v >= 0.0f) || cfg->max_wave_requests < 0)
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
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(s->arena_base);
    delete s;
    return DTB_ERR_CUDA;
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
  if (it == s->resident.end() || it->second.wave == s->wave_no || referenced(s, image_id)) return DTB_ERR_INVALID_ARG;
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
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->arena_base) cudaFree(s->arena_base);
  if (s->wscratch) cudaFree(s->wscratch);
  if (s->wstage) cudaFree(s->wstage);
  delete s;
}

}  // extern "C"
