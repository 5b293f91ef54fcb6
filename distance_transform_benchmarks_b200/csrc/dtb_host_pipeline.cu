// dtb_host_pipeline.cu -- batches whose images, masks and distance maps are all in host memory.
//
// Host-to-device copies with a pitch change crawl (the copy engines move one narrow row at a time), so the
// pipeline copies every image and mask as one 1-D block into packed device memory, moves rows into 128-byte
// pitches on the device only where the TMA needs it (rows not a multiple of 16 bytes), and writes distances
// packed so that each map returns as one 1-D block.  The batch is cut into chunks of about host_chunk_px
// pixels; the copies in (stream s_in), the tile runs (the caller's stream) and the copies out (stream s_out)
// of successive chunks overlap.
#include <cuda_runtime.h>

#include <algorithm>
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

struct Plane {  // device placement of one image's planes
  uint8_t* img_packed;
  uint8_t* img_tma;   // == img_packed when the packed rows are TMA-aligned
  uint8_t* mask_packed;
  uint8_t* mask_tma;
  float* dist;        // packed rows of 4 * width bytes
  int64_t img_pitch, mask_pitch;
};

}  // namespace

dtb_status run_host_pipeline(dtb_context ctx, std::vector<Job> jobs, const dtb_image* const* imgs,
                             const dtb_image* const* masks, const dtb_image* const* dists, cudaStream_t stream) {
  const int n = (int)jobs.size();
  if (!ctx->s_in) DTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_in, cudaStreamNonBlocking));
  if (!ctx->s_out) DTB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_out, cudaStreamNonBlocking));

  // ---- device placement of the planes ----
  std::vector<Plane> pl(n);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + std::max<size_t>(bytes, 1), 256);
    return o;
  };
  std::vector<size_t> o_ip(n), o_it(n), o_mp(n), o_mt(n), o_d(n);
  for (int i = 0; i < n; ++i) {
    const Job& j = jobs[i];
    const size_t rb = (size_t)j.width * j.channels, h = (size_t)j.height;
    const size_t prb = align_up(rb, 128), pmb = align_up((size_t)j.width, 128);
    o_ip[i] = take(rb * h);
    o_it[i] = (rb % 16) ? take(prb * h) : o_ip[i];
    o_mp[i] = take((size_t)j.width * h);
    o_mt[i] = (j.width % 16) ? take(pmb * h) : o_mp[i];
    o_d[i] = take(4 * (size_t)j.width * h);
    pl[i].img_pitch = (rb % 16) ? (int64_t)prb : (int64_t)rb;
    pl[i].mask_pitch = (j.width % 16) ? (int64_t)pmb : (int64_t)j.width;
  }
  dtb_status s = grow(ctx, &ctx->dstage, &ctx->dstage_size, off);
  if (s != DTB_OK) return s;
  uint8_t* stage = static_cast<uint8_t*>(ctx->dstage);
  for (int i = 0; i < n; ++i) {
    pl[i].img_packed = stage + o_ip[i];
    pl[i].img_tma = stage + o_it[i];
    pl[i].mask_packed = stage + o_mp[i];
    pl[i].mask_tma = stage + o_mt[i];
    pl[i].dist = reinterpret_cast<float*>(stage + o_d[i]);
    jobs[i].img = pl[i].img_tma;
    jobs[i].img_pitch = pl[i].img_pitch;
    jobs[i].mask = pl[i].mask_tma;
    jobs[i].mask_pitch = pl[i].mask_pitch;
    jobs[i].dist = pl[i].dist;
    jobs[i].dist_pitch = 4 * (int64_t)jobs[i].width;
  }

  // ---- chunks of about host_chunk_px pixels ----
  std::vector<int> cut{0};
  uint64_t acc = 0;
  for (int i = 0; i < n; ++i) {
    acc += (uint64_t)jobs[i].width * jobs[i].height;
    if (acc >= ctx->host_chunk_px && i + 1 < n) {
      cut.push_back(i + 1);
      acc = 0;
    }
  }
  cut.push_back(n);
  const int nchunks = (int)cut.size() - 1;

  // ---- per-chunk scratch, tables and repitch lists, all uploaded in one copy ----
  LaunchTuning tuning = ctx->tuning;
  uint32_t total_all = 0;
  if ((s = count_tiles(ctx, jobs, &total_all)) != DTB_OK) return s;
  auto it = ctx->tuned.find(tuning_key(n, total_all));
  if (it != ctx->tuned.end()) tuning = it->second;
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
    L[k] = layout_for((int)cj.size(), total, workers, false);
    o_chunk[k] = soff;
    soff = align_up(soff + L[k].bytes, 256);
    for (int i = cut[k]; i < cut[k + 1]; ++i) {
      const Job& j = jobs[i];
      if (j.width == 0 || j.height == 0) continue;
      const uint32_t rb = (uint32_t)(j.width * j.channels);
      if (pl[i].img_tma != pl[i].img_packed) {
        items[k].push_back({pl[i].img_packed, pl[i].img_tma, rb, (uint32_t)j.height, (uint32_t)pl[i].img_pitch, rows[k]});
        rows[k] += (uint32_t)j.height;
      }
      if (pl[i].mask_tma != pl[i].mask_packed) {
        items[k].push_back({pl[i].mask_packed, pl[i].mask_tma, (uint32_t)j.width, (uint32_t)j.height,
                            (uint32_t)pl[i].mask_pitch, rows[k]});
        rows[k] += (uint32_t)j.height;
      }
    }
    o_items[k] = soff;
    soff = align_up(soff + sizeof(RepitchItem) * std::max<size_t>(items[k].size(), 1), 256);
  }
  if ((s = grow(ctx, &ctx->dscratch, &ctx->dscratch_size, soff)) != DTB_OK) return s;
  uint8_t* scratch = static_cast<uint8_t*>(ctx->dscratch);
  std::vector<uint8_t>& host = ctx->hstage;
  host.assign(soff, 0);
  for (int k = 0; k < nchunks; ++k) {
    std::vector<Job> cj(jobs.begin() + cut[k], jobs.begin() + cut[k + 1]);
    std::vector<uint8_t> tab;
    if ((s = build_tables(ctx, cj, L[k], tab)) != DTB_OK) return s;
    std::copy(tab.begin(), tab.end(), host.begin() + o_chunk[k] + L[k].o_desc);
    std::copy(reinterpret_cast<const uint8_t*>(items[k].data()),
              reinterpret_cast<const uint8_t*>(items[k].data() + items[k].size()), host.begin() + o_items[k]);
  }
  // Pageable source: the copy has consumed it when the call returns.
  DTB_CUDA(ctx, cudaMemcpyAsync(scratch, host.data(), soff, cudaMemcpyHostToDevice, stream));
  cudaEvent_t ev_tables = event_at(ctx, 0);
  if (!ev_tables) return fail(ctx, DTB_ERR_CUDA, "cudaEventCreate failed");
  DTB_CUDA(ctx, cudaEventRecord(ev_tables, stream));

  // ---- the pipeline ----
  DTB_CUDA(ctx, cudaStreamWaitEvent(ctx->s_in, ev_tables, 0));  // staging memory is free once earlier work is done
  for (int k = 0; k < nchunks; ++k) {
    for (int i = cut[k]; i < cut[k + 1]; ++i) {
      const dtb_image* ui = imgs[i];
      const dtb_image* um = masks[i];
      const Job& j = jobs[i];
      if (j.width == 0 || j.height == 0) continue;
      const size_t rb = (size_t)j.width * j.channels;
      if ((size_t)ui->pitch == rb)
        DTB_CUDA(ctx, cudaMemcpyAsync(pl[i].img_packed, ui->buffer, rb * j.height, cudaMemcpyHostToDevice, ctx->s_in));
      else
        DTB_CUDA(ctx, cudaMemcpy2DAsync(pl[i].img_packed, rb, ui->buffer, ui->pitch, rb, j.height, cudaMemcpyHostToDevice,
                                        ctx->s_in));
      if (um->pitch == j.width)
        DTB_CUDA(ctx, cudaMemcpyAsync(pl[i].mask_packed, um->buffer, (size_t)j.width * j.height, cudaMemcpyHostToDevice,
                                      ctx->s_in));
      else
        DTB_CUDA(ctx, cudaMemcpy2DAsync(pl[i].mask_packed, j.width, um->buffer, um->pitch, j.width, j.height,
                                        cudaMemcpyHostToDevice, ctx->s_in));
    }
    cudaEvent_t e_in = event_at(ctx, 1 + 3 * k);
    if (!e_in) return fail(ctx, DTB_ERR_CUDA, "cudaEventCreate failed");
    DTB_CUDA(ctx, cudaEventRecord(e_in, ctx->s_in));
  }
  for (int k = 0; k < nchunks; ++k) {
    uint8_t* cbase = scratch + o_chunk[k];
    DTB_CUDA(ctx, cudaStreamWaitEvent(stream, event_at(ctx, 1 + 3 * k), 0));
    if (!items[k].empty()) {
      const uint32_t blocks = std::min<uint32_t>((rows[k] + 7) / 8, (uint32_t)ctx->num_sms * 8);
      repitch_rows<<<blocks, 256, 0, stream>>>(reinterpret_cast<const RepitchItem*>(scratch + o_items[k]),
                                              (int)items[k].size(), rows[k]);
      DTB_CUDA(ctx, cudaGetLastError());
    }
    if ((s = enqueue_persistent(ctx, cbase, L[k], MODE_NS, tuning, stream, nullptr, nullptr)) != DTB_OK) return s;
    cudaEvent_t e_run = event_at(ctx, 2 + 3 * k);
    if (!e_run) return fail(ctx, DTB_ERR_CUDA, "cudaEventCreate failed");
    DTB_CUDA(ctx, cudaEventRecord(e_run, stream));
    DTB_CUDA(ctx, cudaStreamWaitEvent(ctx->s_out, e_run, 0));
    for (int i = cut[k]; i < cut[k + 1]; ++i) {
      const dtb_image* ud = dists[i];
      const Job& j = jobs[i];
      if (j.width == 0 || j.height == 0) continue;
      const size_t rb = 4 * (size_t)j.width;
      if ((size_t)ud->pitch == rb)
        DTB_CUDA(ctx, cudaMemcpyAsync(ud->buffer, pl[i].dist, rb * j.height, cudaMemcpyDeviceToHost, ctx->s_out));
      else
        DTB_CUDA(ctx, cudaMemcpy2DAsync(ud->buffer, ud->pitch, pl[i].dist, rb, rb, j.height, cudaMemcpyDeviceToHost,
                                        ctx->s_out));
    }
  }
  cudaEvent_t e_done = event_at(ctx, 3 + 3 * (nchunks - 1));
  if (!e_done) return fail(ctx, DTB_ERR_CUDA, "cudaEventCreate failed");
  DTB_CUDA(ctx, cudaEventRecord(e_done, ctx->s_out));
  DTB_CUDA(ctx, cudaStreamWaitEvent(stream, e_done, 0));
  DTB_CUDA(ctx, cudaStreamSynchronize(stream));

  // ---- status and counters of every chunk ----
  dtb_stats acc_st{};
  dtb_status first_err = DTB_OK;
  for (int k = 0; k < nchunks; ++k) {
    dtb_stats st{};
    const dtb_status cs = read_device_status(ctx, reinterpret_cast<QueueHdr*>(scratch + o_chunk[k] + L[k].o_hdr), &st);
    if (cs != DTB_OK && first_err == DTB_OK) first_err = cs;
    acc_st.tiles += L[k].total;
    acc_st.tile_visits += st.tile_visits;
    acc_st.phases += st.phases;
    acc_st.activations += st.activations;
    if (!acc_st.device_error) {
      acc_st.device_error = st.device_error;
      acc_st.device_error_info = st.device_error_info;
    }
  }
  acc_st.rounds = (uint64_t)nchunks;
  ctx->stats = acc_st;
  ctx->async_pending = false;
  return first_err;
}

}  // namespace dtb
