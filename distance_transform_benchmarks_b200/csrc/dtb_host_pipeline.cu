// dtb_host_pipeline.cu -- batches whose images, masks and distance maps are all in host memory.
//
// Host-to-device copies with a pitch change crawl (the copy engines move one narrow row at a time), and many
// small copies in both directions overlap poorly, so the pipeline moves each run of planes that are packed and
// adjacent in host memory (a batch in one pinned arena is one run per plane kind) as ONE 1-D copy into device
// staging that mirrors the host bytes, moves rows into 128-byte pitches on the device only where the TMA needs
// it (rows or bases not on 16 bytes), and writes distances packed in the mirrored layout so that each run
// returns as one 1-D copy.  The batch is cut into chunks of about host_chunk_px pixels; the copies in (stream
// s_in), the tile runs and the copies out (stream s_out) of successive chunks overlap.  The tile runs alternate
// between two compute lanes (s_lane0, s_lane), each launched on half of the co-resident CTAs: a run's tail,
// where only the last tiles of its largest images are still active, then overlaps the next chunk's run instead
// of idling the GPU (one lane ran each chunk at about a third of the batch rate).  Successive calls use
// alternate sets of device staging and scratch, so a call's copies in run while the previous call's copies
// out finish (the two directions of the link overlap across calls as well as within one).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "dtb.h"
#include "dtb_internal.h"

namespace dtb {

// One warp per destination row; each lane assembles 4-byte words of the (128-byte aligned) destination row.
__global__ void __launch_bounds__(256) repitch_rows(const RepitchItem* __restrict__ items, int n, uint32_t total_rows) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < total_rows; r += nw) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (items[mid].row_base <= r) lo = mid;
      else hi = mid - 1;
    }
    const RepitchItem it = items[lo];
    const uint32_t y = r - it.row_base;
    const uint8_t* s = it.src + (size_t)y * it.row_bytes;
    uint32_t* d = reinterpret_cast<uint32_t*>(it.dst + (size_t)y * it.dst_pitch);
    const uint32_t words = (it.row_bytes + 3) / 4;  // the last word may cover pad bytes of the destination row
    for (uint32_t j = lane; j < words; j += 32) {
      const uint32_t b = 4 * j;
      uint32_t v = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (b + k < it.row_bytes) v |= (uint32_t)s[b + k] << (8 * k);
      d[j] = v;
    }
  }
}

namespace {

cudaEvent_t event_at(dtb_context ctx, size_t i) {
  while (ctx->evpool.size() <= i) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    ctx->evpool.push_back(e);
  }
  return ctx->evpool[i];
}

// One host <-> device copy of the pipeline: 1-D when rows == 1 (a run of adjacent packed planes), else 2-D.
// `dev` is an offset into the staging block.
struct Copy {
  size_t dev;
  uint8_t* host;
  size_t host_pitch, dev_pitch, width, rows;
};

dtb_status issue(dtb_context ctx, const Copy& c, uint8_t* stage, bool to_device, cudaStream_t st) {
  uint8_t* d = stage + c.dev;
  if (to_device) {
    if (c.rows == 1) DTB_CUDA(ctx, cudaMemcpyAsync(d, c.host, c.width, cudaMemcpyHostToDevice, st));
    else DTB_CUDA(ctx, cudaMemcpy2DAsync(d, c.dev_pitch, c.host, c.host_pitch, c.width, c.rows, cudaMemcpyHostToDevice, st));
  } else {
    if (c.rows == 1) DTB_CUDA(ctx, cudaMemcpyAsync(c.host, d, c.width, cudaMemcpyDeviceToHost, st));
    else DTB_CUDA(ctx, cudaMemcpy2DAsync(c.host, c.host_pitch, d, c.dev_pitch, c.width, c.rows, cudaMemcpyDeviceToHost, st));
  }
  return DTB_OK;
}

// Host side of one plane of one image.
struct HostPlane {
  const uint8_t* ptr;
  size_t pitch, row_bytes, rows;
  bool empty() const { return row_bytes == 0 || rows == 0; }
  bool packed() const { return pitch == row_bytes; }
  size_t bytes() const { return row_bytes * rows; }
};

// Device placement of one kind of plane (images, masks or distances) for the images [a, b) of a chunk.  Runs of
// consecutive packed planes that are adjacent in host memory move as ONE 1-D copy: their device staging mirrors
// the host byte range, at an offset congruent to the host address modulo 256, so each plane keeps the
// alignment it has on the host (few large copies overlap in both directions on the copy engines; per-image
// copies do not).  Planes with padded host rows get their own packed region and a 2-D copy.  `take(bytes)`
// returns 256-byte aligned offsets into the staging block; dev_off[i] receives the plane's offset.
template <class Take>
void place_plane(int a, int b, const std::vector<HostPlane>& hp, Take&& take, std::vector<size_t>& dev_off,
                 std::vector<Copy>& copies) {
  int i = a;
  while (i < b) {
    if (hp[i].empty()) { ++i; continue; }
    if (!hp[i].packed()) {
      dev_off[i] = take(hp[i].bytes());
      copies.push_back(Copy{dev_off[i], const_cast<uint8_t*>(hp[i].ptr), hp[i].pitch, hp[i].row_bytes, hp[i].row_bytes,
                            hp[i].rows});
      ++i;
      continue;
    }
    const uint8_t* start = hp[i].ptr;
    const uint8_t* end = start + hp[i].bytes();
    int j = i + 1;
    for (; j < b; ++j) {
      if (hp[j].empty()) continue;
      if (!hp[j].packed() || hp[j].ptr != end) break;
      end += hp[j].bytes();
    }
    const size_t shift = reinterpret_cast<uintptr_t>(start) & 255u;
    const size_t region = take((size_t)(end - start) + shift) + shift;
    for (int m = i; m < j; ++m)
      if (!hp[m].empty()) dev_off[m] = region + (size_t)(hp[m].ptr - start);
    copies.push_back(Copy{region, const_cast<uint8_t*>(start), 0, 0, (size_t)(end - start), 1});
    i = j;
  }
}

}  // namespace

dtb_status run_host_pipeline(dtb_context ctx, std::vector<Job> jobs, const dtb_image* const* imgs,
                             const dtb_image* const* masks, const dtb_image* const* dists, uint32_t flags,
                             cudaStream_t stream) {
  const TraceRange trace("dtb host pipeline");
  const int n = (int)jobs.size();
  if (!ctx->s_in) DTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_in, cudaStreamNonBlocking));
  if (!ctx->s_out) DTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_out, cudaStreamNonBlocking));
  if (!ctx->s_lane) DTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_lane, cudaStreamNonBlocking));
  if (!ctx->s_lane0) DTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_lane0, cudaStreamNonBlocking));
  if (!ctx->ev_pipe_done) DTB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_pipe_done, cudaEventDisableTiming));
  if (!ctx->ev_pipe_start) DTB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_pipe_start, cudaEventDisableTiming));
  for (int i = 0; i < 2; ++i)
    if (!ctx->ev_pset_free[i]) DTB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_pset_free[i], cudaEventDisableTiming));
  if (!ctx->dpipe) {
    DTB_CUDA(ctx, cudaMalloc(&ctx->dpipe, sizeof(QueueHdr)));
    DTB_CUDA(ctx, cudaMemset(ctx->dpipe, 0, sizeof(QueueHdr)));
  }
  const int set = ctx->pset_cur;
  ctx->pset_cur ^= 1;

  // ---- chunks of about host_chunk_px pixels, the first ones smaller (1/8, 1/4, 1/2) so that the first maps
  //      start their way back early ----
  std::vector<int> cut{0};
  uint64_t acc = 0, target = std::max<uint64_t>(ctx->host_chunk_px / 8, 1);
  for (int i = 0; i < n; ++i) {
    acc += (uint64_t)jobs[i].width * jobs[i].height;
    if (acc >= target && i + 1 < n) {
      cut.push_back(i + 1);
      acc = 0;
      target = std::min<uint64_t>(2 * target, ctx->host_chunk_px);
    }
  }
  cut.push_back(n);
  const int nchunks = (int)cut.size() - 1;

  // ---- device placement of the planes: mirrored runs, repitched copies where the TMA needs them ----
  std::vector<HostPlane> hi(n), hm(n), hd(n);
  for (int i = 0; i < n; ++i) {
    const Job& j = jobs[i];
    const size_t w = (size_t)j.width, h = (size_t)j.height;
    hi[i] = HostPlane{static_cast<const uint8_t*>(imgs[i]->buffer), (size_t)imgs[i]->pitch, w * j.channels, h};
    hm[i] = HostPlane{static_cast<const uint8_t*>(masks[i]->buffer), (size_t)masks[i]->pitch, w, h};
    hd[i] = HostPlane{static_cast<const uint8_t*>(dists[i]->buffer), (size_t)dists[i]->pitch, 4 * w, h};
  }
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + std::max<size_t>(bytes, 1), 256);
    return o;
  };
  std::vector<size_t> o_ip(n, 0), o_it(n, 0), o_mp(n, 0), o_mt(n, 0), o_d(n, 0);
  std::vector<std::vector<Copy>> cin(nchunks), cout(nchunks);
  for (int k = 0; k < nchunks; ++k) {
    place_plane(cut[k], cut[k + 1], hi, take, o_ip, cin[k]);
    place_plane(cut[k], cut[k + 1], hm, take, o_mp, cin[k]);
    place_plane(cut[k], cut[k + 1], hd, take, o_d, cout[k]);
  }
  for (int i = 0; i < n; ++i) {
    const Job& j = jobs[i];
    if (j.width == 0 || j.height == 0) continue;
    const size_t rb = (size_t)j.width * j.channels, h = (size_t)j.height;
    // The tile kernel reads images and masks through TMA maps: 16-byte aligned base and pitch.
    o_it[i] = (rb % 16 || o_ip[i] % 16) ? take(align_up(rb, 128) * h) : o_ip[i];
    o_mt[i] = ((size_t)j.width % 16 || o_mp[i] % 16) ? take(align_up((size_t)j.width, 128) * h) : o_mp[i];
  }
  dtb_status s = grow(ctx, &ctx->pstage[set], &ctx->pstage_size[set], off);
  if (s != DTB_OK) return s;
  uint8_t* stage = static_cast<uint8_t*>(ctx->pstage[set]);
  for (int i = 0; i < n; ++i) {
    const int64_t rb = (int64_t)jobs[i].width * jobs[i].channels;
    jobs[i].img = stage + o_it[i];
    jobs[i].img_pitch = (o_it[i] == o_ip[i]) ? rb : (int64_t)align_up((size_t)rb, 128);
    jobs[i].mask = stage + o_mt[i];
    jobs[i].mask_pitch = (o_mt[i] == o_mp[i]) ? (int64_t)jobs[i].width : (int64_t)align_up((size_t)jobs[i].width, 128);
    jobs[i].dist = reinterpret_cast<float*>(stage + o_d[i]);
    jobs[i].dist_pitch = 4 * (int64_t)jobs[i].width;
  }

  // ---- per-chunk scratch, tables and repitch lists, all uploaded in one copy ----
  LaunchTuning tuning = ctx->tuning;
  uint32_t total_all = 0;
  if ((s = count_tiles(ctx, jobs, &total_all)) != DTB_OK) return s;
  auto it = ctx->tuned.find(tuning_key(n, total_all));
  if (it != ctx->tuned.end()) tuning = it->second;
  // The two compute lanes below each take half of the co-resident CTAs, so they keep 4-warp CTAs with the same
  // warps per SM as the tuning: with 2 x 6 or 2 x 8 shapes a lane has one CTA per SM, and the 1024-image
  // host-buffer step ran in 50 ms instead of 36 ms on the B200 box.
  if (NS_VARIANT_TABLE[tuning.variant].wpc != PERSIST_WPC) {
    const NsVariant& v = NS_VARIANT_TABLE[tuning.variant];
    const int k = ns_variant_of(v.ctas * v.wpc / PERSIST_WPC, false, PERSIST_WPC);
    if (k >= 0) tuning.variant = k;
  }
  const uint32_t workers = resident_workers(ctx, MODE_NS, tuning);
  std::vector<ScratchLayout> L(nchunks);
  std::vector<size_t> o_chunk(nchunks), o_items(nchunks);
  std::vector<std::vector<RepitchItem>> items(nchunks);
  std::vector<uint32_t> rows(nchunks, 0);
  size_t soff = 0;
  for (int k = 0; k < nchunks; ++k) {
    std::vector<Job> cj(jobs.begin() + cut[k], jobs.begin() + cut[k + 1]);
    uint32_t total = 0;
    if ((s = count_tiles(ctx, cj, &total)) != DTB_OK) return s;
    L[k] = layout_for((int)cj.size(), total, workers, false, (uint32_t)tuning.buckets);
    o_chunk[k] = soff;
    soff = align_up(soff + L[k].bytes, 256);
    for (int i = cut[k]; i < cut[k + 1]; ++i) {
      const Job& j = jobs[i];
      if (j.width == 0 || j.height == 0) continue;
      const uint32_t rb = (uint32_t)(j.width * j.channels);
      if (o_it[i] != o_ip[i]) {
        items[k].push_back({stage + o_ip[i], stage + o_it[i], rb, (uint32_t)j.height, (uint32_t)j.img_pitch, rows[k]});
        rows[k] += (uint32_t)j.height;
      }
      if (o_mt[i] != o_mp[i]) {
        items[k].push_back({stage + o_mp[i], stage + o_mt[i], (uint32_t)j.width, (uint32_t)j.height, (uint32_t)j.mask_pitch,
                            rows[k]});
        rows[k] += (uint32_t)j.height;
      }
    }
    o_items[k] = soff;
    soff = align_up(soff + sizeof(RepitchItem) * std::max<size_t>(items[k].size(), 1), 256);
  }
  if ((s = grow(ctx, &ctx->pscratch[set], &ctx->pscratch_size[set], soff)) != DTB_OK) return s;
  uint8_t* scratch = static_cast<uint8_t*>(ctx->pscratch[set]);
  // Only the descriptor tables, tensor maps and repitch lists of each chunk go up (one pinned block, one copy
  // per part); queue headers, rings and tile states are reset on the device by each chunk's run.
  size_t hbytes = 0;
  std::vector<size_t> h_tab(nchunks), h_items(nchunks);
  for (int k = 0; k < nchunks; ++k) {
    h_tab[k] = hbytes;
    hbytes += L[k].o_act - L[k].o_desc;
    h_items[k] = hbytes;
    hbytes += sizeof(RepitchItem) * items[k].size();
  }
  uint8_t* host = nullptr;
  cudaEvent_t ev_host = nullptr;
  if ((s = pinned_stage(ctx, hbytes, &host, &ev_host)) != DTB_OK) return s;
  // Everything of this call follows s_in: it starts after the caller's earlier work on `stream` and, when this
  // set of staging and scratch served an earlier call, after that call's end.
  DTB_CUDA(ctx, cudaEventRecord(ctx->ev_pipe_start, stream));
  DTB_CUDA(ctx, cudaStreamWaitEvent(ctx->s_in, ctx->ev_pipe_start, 0));
  if (ctx->pset_used[set]) DTB_CUDA(ctx, cudaStreamWaitEvent(ctx->s_in, ctx->ev_pset_free[set], 0));
  for (int k = 0; k < nchunks; ++k) {
    std::vector<Job> cj(jobs.begin() + cut[k], jobs.begin() + cut[k + 1]);
    std::vector<uint8_t>& tab = ctx->hstage;
    if ((s = build_tables(ctx, cj, L[k], tab)) != DTB_OK) return s;
    std::copy(tab.begin(), tab.end(), host + h_tab[k]);
    std::copy(reinterpret_cast<const uint8_t*>(items[k].data()),
              reinterpret_cast<const uint8_t*>(items[k].data() + items[k].size()), host + h_items[k]);
    DTB_CUDA(ctx, cudaMemcpyAsync(scratch + o_chunk[k] + L[k].o_desc, host + h_tab[k], tab.size(), cudaMemcpyHostToDevice,
                                  ctx->s_in));
    ctx->pipe_h2d += tab.size();
    if (!items[k].empty()) {
      DTB_CUDA(ctx, cudaMemcpyAsync(scratch + o_items[k], host + h_items[k], sizeof(RepitchItem) * items[k].size(),
                                    cudaMemcpyHostToDevice, ctx->s_in));
      ctx->pipe_h2d += sizeof(RepitchItem) * items[k].size();
    }
  }
  DTB_CUDA(ctx, cudaEventRecord(ev_host, ctx->s_in));

  // ---- the pipeline: copies in, tile runs on the two lanes, copies out ----
  for (int k = 0; k < nchunks; ++k) {
    for (const Copy& c : cin[k]) {
      if ((s = issue(ctx, c, stage, true, ctx->s_in)) != DTB_OK) return s;
      ctx->pipe_h2d += c.width * c.rows;
    }
    cudaEvent_t e_in = event_at(ctx, 1 + 3 * k);
    if (!e_in) return fail(ctx, DTB_ERR_CUDA, "cudaEventCreate failed");
    DTB_CUDA(ctx, cudaEventRecord(e_in, ctx->s_in));
  }
  const int lanes = nchunks > 1 ? 2 : 1;
  LaunchTuning lane_tuning = tuning;
  lane_tuning.grid_percent = std::max(1, tuning.grid_percent / lanes);
  for (int k = 0; k < nchunks; ++k) {
    uint8_t* cbase = scratch + o_chunk[k];
    cudaStream_t lane = (k % lanes) ? ctx->s_lane : ctx->s_lane0;
    DTB_CUDA(ctx, cudaStreamWaitEvent(lane, event_at(ctx, 1 + 3 * k), 0));
    if (!items[k].empty()) {
      const uint32_t blocks = std::min<uint32_t>((rows[k] + 7) / 8, (uint32_t)ctx->num_sms * 8);
      repitch_rows<<<blocks, 256, 0, lane>>>(reinterpret_cast<const RepitchItem*>(scratch + o_items[k]),
                                            (int)items[k].size(), rows[k]);
      DTB_CUDA(ctx, cudaGetLastError());
    }
    if ((s = enqueue_persistent(ctx, cbase, L[k], MODE_NS, lane_tuning, lane, nullptr, nullptr, ctx->dpipe)) != DTB_OK)
      return s;
    cudaEvent_t e_run = event_at(ctx, 2 + 3 * k);
    if (!e_run) return fail(ctx, DTB_ERR_CUDA, "cudaEventCreate failed");
    DTB_CUDA(ctx, cudaEventRecord(e_run, lane));
    DTB_CUDA(ctx, cudaStreamWaitEvent(ctx->s_out, e_run, 0));
    for (const Copy& c : cout[k]) {
      if ((s = issue(ctx, c, stage, false, ctx->s_out)) != DTB_OK) return s;
      ctx->pipe_d2h += c.width * c.rows;
    }
  }
  // The call's end: its last copy out (each chunk's run, which folded its status into ctx->dpipe, came before
  // that chunk's copy out).  Only copies run on s_out, so the next calls are not held up by a kernel waiting
  // for SMs that the tile runs hold.
  DTB_CUDA(ctx, cudaEventRecord(ctx->ev_pset_free[set], ctx->s_out));
  ctx->pset_used[set] = true;
  DTB_CUDA(ctx, cudaEventRecord(ctx->ev_pipe_done, ctx->s_out));
  ctx->pipe_tiles += total_all;
  ctx->pipe_chunks += (uint64_t)nchunks;
  ctx->pipe_pending = true;
  ctx->async_pending = false;
  if (flags & DTB_FLAG_ASYNC) return DTB_OK;  // dtb_sync(ctx, stream) waits and reports
  DTB_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->ev_pipe_done, 0));
  DTB_CUDA(ctx, cudaStreamSynchronize(stream));
  return finish_pipeline(ctx);
}

dtb_status finish_pipeline(dtb_context ctx) {
  ctx->pipe_pending = false;
  dtb_stats st{};
  const dtb_status s = read_device_status(ctx, ctx->dpipe, &st);
  st.tiles = ctx->pipe_tiles;
  st.rounds = ctx->pipe_chunks;
  st.h2d_bytes = ctx->pipe_h2d;
  st.d2h_bytes = ctx->pipe_d2h;
  ctx->stats = st;
  ctx->pipe_tiles = ctx->pipe_chunks = ctx->pipe_h2d = ctx->pipe_d2h = 0;
  DTB_CUDA(ctx, cudaMemset(ctx->dpipe, 0, sizeof(QueueHdr)));
  return s;
}

}  // namespace dtb
