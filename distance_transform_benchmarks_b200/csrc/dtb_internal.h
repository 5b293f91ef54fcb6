// dtb_internal.h -- host-side types shared by the translation units of libdtb.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "dtb.h"
#include "dtb_device.cuh"

namespace dtb {

constexpr int PERSIST_WPC = 4;   // warps per CTA of the persistent tile kernel
constexpr int ROUND_WPC = 4;
constexpr size_t PERSIST_SMEM = PERSIST_WPC * sizeof(WarpSmem) + 128;
constexpr size_t PERSIST_SMEM_AHEAD = PERSIST_WPC * sizeof(WarpSmemP) + 128;
constexpr size_t ROUND_SMEM = ROUND_WPC * sizeof(WarpSmem) + 128;
constexpr uint64_t DEFAULT_TIMEOUT_NS = 2000000000ull;
constexpr int REF_CTAS = 3;  // resident CTAs per SM of the ref-mode tile kernels (168 registers)
// ns-mode tile kernel variants: CTAs per SM, whether a warp stages its next tile ahead (17 KB of shared memory a
// warp instead of 13 KB, so at most 3 CTAs of 4 warps per SM), and warps per CTA.  Registers per thread follow
// the warps per SM: 8 -> 255, 12 -> 168, 16 -> 128.  The 12- and 16-warp shapes come in several CTA sizes
// (2 x 6, 3 x 4, 6 x 2; 2 x 8, 4 x 4), which differ in how the SM's warps are grouped and scheduled only.
struct NsVariant {
  int ctas;
  bool ahead;
  int wpc;
};
constexpr int NS_VARIANTS = 8;
constexpr NsVariant NS_VARIANT_TABLE[NS_VARIANTS] = {{2, false, 4}, {3, false, 4}, {4, false, 4}, {2, true, 4},
                                                     {3, true, 4},  {6, false, 2}, {2, false, 6}, {2, false, 8}};
// Variant index of (ctas, ahead, warps per CTA), or -1.
inline int ns_variant_of(int ctas, bool ahead, int wpc = PERSIST_WPC) {
  for (int k = 0; k < NS_VARIANTS; ++k)
    if (NS_VARIANT_TABLE[k].ctas == ctas && NS_VARIANT_TABLE[k].ahead == ahead && NS_VARIANT_TABLE[k].wpc == wpc)
      return k;
  return -1;
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// One image of a call, resolved to device memory.
struct Job {
  const uint8_t* img = nullptr;
  int64_t img_pitch = 0;
  int channels = 1;
  const uint8_t* mask = nullptr;
  int64_t mask_pitch = 0;
  float* dist = nullptr;
  int64_t dist_pitch = 0;
  int width = 0, height = 0;
  float g2 = 0.0f, v = 0.0f, l_eucl = 0.0f, l_grad = 0.0f;
  int mode = 0, ref_fma = 1;

  int tiles_x() const { return (width + 31) / 32; }
  int tiles_y() const { return (height + 31) / 32; }

  static Job from(const dtb_image* img, const dtb_image* mask, const dtb_image* dist) {
    Job j;
    j.img = static_cast<const uint8_t*>(img->buffer);
    j.img_pitch = img->pitch;
    j.channels = img->elem_size;
    j.mask = static_cast<const uint8_t*>(mask->buffer);
    j.mask_pitch = mask->pitch;
    j.dist = static_cast<float*>(dist->buffer);
    j.dist_pitch = dist->pitch;
    j.width = img->width;
    j.height = img->height;
    return j;
  }
};

// g2 = fl32(gamma * gamma): the one place gamma is squared, so host and oracle agree on the bits.
inline float gamma_to_g2(float gamma) {
  const float g = gamma;
  return g * g;
}

// Device scratch of one run: [queue header | tile states | ring | descriptors | tensor maps | tile prefix |
// round flags | changed word], each part 256-byte aligned.
struct ScratchLayout {
  int n = 0;
  uint32_t total = 0;  // tiles
  uint32_t cap = 0;    // ring slots per bucket (power of two)
  uint32_t nb = 1;     // priority-bucket rings allocated (a power of two <= NBUCKET_MAX; 1 = one FIFO ring)
  size_t o_hdr = 0, o_states = 0, o_ring = 0, o_keys = 0, o_wacc = 0, o_desc = 0, o_tmap = 0, o_base = 0, o_act = 0,
         o_chg = 0, bytes = 0;
  size_t ring_bytes() const { return 4ull * cap * nb; }
};

// Queue policy defaults: 8 priority buckets half a tile-width of path cost wide.
constexpr int DEFAULT_BUCKETS = 8;
constexpr float DEFAULT_BUCKET_TILES = 0.5f;

// Launch parameters of the tile kernel chosen for a run, and the policy of its tile queue.
struct LaunchTuning {
  int variant = 0;        // ns-mode kernel variant (index into NS_VARIANT_TABLE)
  int grid_percent = 100; // share of the co-resident CTAs that is launched
  int buckets = DEFAULT_BUCKETS;              // 1 = FIFO, else 2 / 4 / 8 / 16 distance-ordered buckets
  float bucket_tiles = DEFAULT_BUCKET_TILES;  // bucket width in tile-widths of path cost
};

}  // namespace dtb

struct dtb_context_s {
  int device = 0;
  int num_sms = 0;
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  const void* ns_fn[dtb::NS_VARIANTS] = {};
  size_t ns_smem[dtb::NS_VARIANTS] = {};
  int ns_blocks_per_sm[dtb::NS_VARIANTS] = {};
  int ref_blocks_per_sm = 0;
  std::string gpu_name;                           // device name (key of the autotuner cache)
  dtb::LaunchTuning tuning;                       // default tuning of this context
  std::map<uint64_t, dtb::LaunchTuning> tuned;    // autotuner results by workload key
  std::string tune_cache_path;                    // autotuner cache file (JSON), empty = none
  void* dscratch = nullptr;
  size_t dscratch_size = 0;
  void* dstage = nullptr;
  size_t dstage_size = 0;
  std::vector<uint8_t> hstage;
  std::string msg;
  dtb_stats stats{};
  // Asynchronous bookkeeping: header of the last enqueued run and the stream it ran on.
  dtb::QueueHdr* last_hdr = nullptr;
  cudaStream_t last_stream = nullptr;
  bool async_pending = false;
  cudaEvent_t ev[2] = {nullptr, nullptr};  // DTB_FLAG_TIMING: around the tile kernel
  bool timed = false;
  // Pinned host staging of descriptor tables, double-buffered: buffer i may be refilled once event i (recorded
  // after the copies out of it) has completed.
  void* hpin[2] = {nullptr, nullptr};
  size_t hpin_size[2] = {0, 0};
  cudaEvent_t hpin_ev[2] = {nullptr, nullptr};
  bool hpin_used[2] = {false, false};
  int hpin_cur = 0;
  // Host-buffer pipeline: status accumulated over the calls since the last dtb_sync (device, QueueHdr layout),
  // completion of the last call, and its bookkeeping.
  dtb::QueueHdr* dpipe = nullptr;
  cudaEvent_t ev_pipe_done = nullptr;
  bool pipe_pending = false;
  uint64_t pipe_tiles = 0, pipe_chunks = 0, pipe_h2d = 0, pipe_d2h = 0;
  // Host-buffer pipeline: two sets of device staging + chunk scratch used by alternate calls, so that a call's
  // copies in overlap the previous call's copies out; set i is free once ev_pset_free[i] (its last call's end)
  // has completed.
  void* pstage[2] = {nullptr, nullptr};
  size_t pstage_size[2] = {0, 0};
  void* pscratch[2] = {nullptr, nullptr};
  size_t pscratch_size[2] = {0, 0};
  cudaEvent_t ev_pset_free[2] = {nullptr, nullptr};
  bool pset_used[2] = {false, false};
  int pset_cur = 0;
  cudaEvent_t ev_pipe_start = nullptr;
  // Host-buffer pipeline: copy streams, two compute lanes, events, chunk size in pixels.
  cudaStream_t s_in = nullptr, s_out = nullptr, s_lane = nullptr, s_lane0 = nullptr;
  std::vector<cudaEvent_t> evpool;
  uint64_t host_chunk_px = 16ull << 20;
  // dtb_gdt_ref_blocks: per-tile round counters of the running call (device scratch of `total` int32).
  int32_t* dround_counts = nullptr;
  size_t dround_counts_size = 0;
  bool count_rounds = false;
  // dtb_debug_inject_queue_stall: no-progress limit of the next persistent run (0 = no injection, one-shot).
  uint64_t inject_stall_ns = 0;
  std::mutex mu;
};

namespace dtb {

// A named range on a profiler's host timeline (NVTX domain "dtb": calls, plan runs, the autotuner, serve waves,
// live publishes and launches); header-only NVTX, which costs nothing when no profiler is attached.
struct TraceRange {
  explicit TraceRange(const char* name);
  ~TraceRange();
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

dtb_status fail(dtb_context ctx, dtb_status s, const char* fmt, ...);
dtb_status cuda_fail(dtb_context ctx, cudaError_t e, const char* what);
#define DTB_CUDA(ctx, call)                                    \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call); \
  } while (0)

dtb_status validate_view(dtb_context ctx, const dtb_image* im, const char* name, int elem_a, int elem_b);
// Checks that img / mask / dist form one image of the given kinds (rgb allowed or not).
dtb_status check_triplet(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist, bool allow_rgb);

// Scratch layout for n images with `total` tiles, `workers` resident warps; `rounds` adds the round flags;
// `buckets`: priority-bucket rings to allocate (a power of two <= NBUCKET_MAX; 1 = one FIFO ring).  A run may
// use fewer buckets than its layout holds.
ScratchLayout layout_for(int n, uint32_t total, uint32_t workers, bool rounds, uint32_t buckets);
// Enqueues the reset of the queue part of a scratch block (header, rings, activation keys, bucket widths).
dtb_status reset_queue(dtb_context ctx, uint8_t* dbase, const ScratchLayout& L, cudaStream_t stream);
// Host image of [descriptors | tensor maps | tile prefix] (bytes o_desc .. o_act of the layout).
dtb_status build_tables(dtb_context ctx, const std::vector<Job>& jobs, const ScratchLayout& L, std::vector<uint8_t>& out);
// Descriptor and tensor maps (image box, mask tile) of one image whose tile ids start at tile_base; `index`
// names the image in error messages.
dtb_status fill_desc(dtb_context ctx, const Job& j, uint32_t tile_base, int index, ImgDesc* d, CUtensorMap* tm);
// Total tiles of the jobs (error if beyond the 31-bit tile id space).
dtb_status count_tiles(dtb_context ctx, const std::vector<Job>& jobs, uint32_t* total);
// Resident warps of the tile kernel of `mode` under `t`.
uint32_t resident_workers(dtb_context ctx, int mode, const LaunchTuning& t);
// Enqueues queue reset, seed scan, the persistent tile kernel and finalize on `stream` (capturable).
// ev0 / ev1 (optional) are recorded around the tile kernel; `fold` (optional) receives the run's status and
// counters, added by finalize.
dtb_status enqueue_persistent(dtb_context ctx, uint8_t* dbase, const ScratchLayout& L, int mode, const LaunchTuning& t,
                              cudaStream_t stream, cudaEvent_t ev0, cudaEvent_t ev1, QueueHdr* fold = nullptr);
// Enqueues the cooperative persistent tile kernel of `mode` under `t` (grid: resident_workers / PERSIST_WPC).
dtb_status launch_tile_kernel(dtb_context ctx, int mode, const LaunchTuning& t, const ImgDesc* descs,
                              const CUtensorMap* tmaps, uint32_t* states, const Queue& q, cudaStream_t stream);
dtb_status run_jobs(dtb_context ctx, const std::vector<Job>& jobs, const dtb_image* const* imgs,
                    const dtb_image* const* masks, const dtb_image* const* dists, uint32_t flags, cudaStream_t stream);
// All images, masks and distances in host memory (ns-mode): chunked pipeline of 1-D host-to-device copies,
// repitch, tile runs and 1-D device-to-host copies on overlapping streams.
// The call starts after the work enqueued on `stream` before it.  DTB_FLAG_ASYNC: returns after enqueueing,
// without making `stream` wait for the call; dtb_sync waits for all such calls and reports their status.
dtb_status run_host_pipeline(dtb_context ctx, std::vector<Job> jobs, const dtb_image* const* imgs,
                             const dtb_image* const* masks, const dtb_image* const* dists, uint32_t flags,
                             cudaStream_t stream);
dtb_status grow(dtb_context ctx, void** p, size_t* size, size_t need);
// Next pinned table-staging buffer of at least `need` bytes (waits until its previous copies are done);
// *ev is to be recorded after the copies out of it.
dtb_status pinned_stage(dtb_context ctx, size_t need, uint8_t** out, cudaEvent_t* ev);

// Kernels shared across translation units (defined in dtb_api.cu / dtb_host_pipeline.cu).
__global__ void __launch_bounds__(128) ggdt_finalize(const ImgDesc* __restrict__ descs, const uint32_t* __restrict__ tile_base,
                                                     int n, uint32_t total, const uint32_t* __restrict__ states,
                                                     const QueueHdr* hdr, QueueHdr* fold);
struct RepitchItem {
  const uint8_t* src;
  uint8_t* dst;
  uint32_t row_bytes;
  uint32_t rows;
  uint32_t dst_pitch;
  uint32_t row_base;  // prefix of rows over the items of the launch
};
// Failure self-test: counts one queued tile that is never pushed (the run ends on its no-progress limit).
__global__ void ggdt_phantom_pending(QueueHdr* hdr);
__global__ void __launch_bounds__(256) repitch_rows(const RepitchItem* __restrict__ items, int n, uint32_t total_rows);
// The device queue of a scratch block; `t` (optional) selects the bucket count (at most the layout's) and width.
Queue make_queue(uint8_t* dbase, const ScratchLayout& L, uint64_t timeout_ns = DEFAULT_TIMEOUT_NS,
                 const LaunchTuning* t = nullptr);
// Valid queue policy: buckets a power of two in [1, NBUCKET_MAX], width in (0, 64].
bool valid_policy(int buckets, float bucket_tiles);
// Workload key of the autotuner cache: image count and tile count, each rounded to a power of two.
uint64_t tuning_key(int n, uint32_t total);
dtb_status read_device_status(dtb_context ctx, const QueueHdr* hdr, dtb_stats* stats);
// Autotuner cache file of the context (ctx->tune_cache_path): load this GPU's entries into ctx->tuned; write
// one entry.  The caller holds ctx->mu.
dtb_status load_tuning_cache(dtb_context ctx);
dtb_status save_tuning_cache(dtb_context ctx, uint64_t key, const LaunchTuning& t, double ms);
// The C ABI view of a launch tuning (host_chunk_kpx from the context).
void tuning_to_abi(dtb_context ctx, const LaunchTuning& lt, dtb_tuning* t);
// Reads and clears the status accumulated by host-pipeline calls since the last read (the caller synchronised).
dtb_status finish_pipeline(dtb_context ctx);

}  // namespace dtb
