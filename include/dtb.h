/*
 * dtb.h -- C ABI of the B200 generalised geodesic distance transform (GGDT).
 *
 * This is the drop-in boundary for the reference library's GGDT entry points
 * (namespace dt, dt/include/dt/generalised_distance_transform.hpp:7-27) and its transfer helpers
 * (dt/include/dt/transfert.hpp:9-17).  Plain C: pointers, sizes and status codes; no C++ types, no
 * exceptions, no torch types.  Every function is thread-safe per context; a context owns its device
 * scratch and may be used from one thread at a time.
 *
 * Distances are FP32.  The map is the greatest fixpoint of single-edge relaxations from
 * D = (mask != 0) ? 0 : v, i.e. the value the reference's raster rounds converge to
 * (dt/src/generalised_distance_transform.cu:126-134), bit for bit.
 */
#ifndef DTB_H
#define DTB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTB_API __attribute__((visibility("default")))
#define DTB_ABI_VERSION 3  /* 3: dtb_tuning.warps_per_cta, dtb_serve_config.live*, dtb_serve_stats.live_ended_* */

typedef enum dtb_status {
  DTB_OK = 0,
  DTB_ERR_INVALID_ARG = 1,   /* bad size / kind / parameter (reference: assert in generalised_distance_transform.cu:104-107) */
  DTB_ERR_CUDA = 2,          /* a CUDA runtime call failed (reference: std::runtime_error, generalised_distance_transform.cu:136-137) */
  DTB_ERR_OUT_OF_MEMORY = 3, /* device allocation failed (reference: image2d_data_gpu.hpp:29-30) */
  DTB_ERR_TIMEOUT = 4,       /* a bounded device wait gave up (no progress); the result is invalid */
  DTB_ERR_DEVICE = 5,        /* the kernel reported an internal error (phase limit, ring full) */
  DTB_ERR_NO_DEVICE = 6,     /* no usable sm_100 device */
  DTB_ERR_CAPACITY = 7,      /* a fixed-size limit was exceeded */
  DTB_ERR_IO = 8             /* an image file could not be read or written (reference: std::runtime_error, imread.cpp:15-16) */
} dtb_status;

/* Memory kinds, reference dt::e_memory_kind (dt/include/dt/image2d_view.hpp:9-13). */
typedef enum dtb_memory_kind { DTB_CPU = 0, DTB_GPU = 1 } dtb_memory_kind;

/* A non-owning pitched 2-D view: the fields of dt::image2d_view<void> (image2d_view.hpp:117-123).
 * Pixel (x, y) is at buffer + y * pitch + x * elem_size.
 * elem_size: 1 = gray uint8 (or seed mask), 3 = rgb8 (interleaved r, g, b; reference dt::rgb8,
 * dt/include/dt/rgb.hpp:7-12), 4 = float distances. */
typedef struct dtb_image {
  void* buffer;
  int32_t width;
  int32_t height;
  int32_t pitch;       /* bytes between rows */
  int32_t elem_size;   /* bytes per pixel */
  int32_t memory_kind; /* dtb_memory_kind */
} dtb_image;

typedef struct dtb_context_s* dtb_context;

/* Flags (bitwise or). */
#define DTB_FLAG_ASYNC 0x1u       /* return after enqueueing; dtb_sync() waits and reports the status.  For images in
                                     device memory (the work is ordered on `stream`), and for ns-mode batches whose
                                     images, masks and maps are all in host memory: such a call starts after the
                                     work enqueued on `stream` before it, but `stream` does not wait for its end
                                     (successive calls overlap their copies); its buffers must stay valid and
                                     untouched until dtb_sync returns, and the status covers every such call since
                                     the last dtb_sync.  Other host-memory calls ignore the flag. */
#define DTB_FLAG_ROUNDS 0x2u      /* plain per-image path: host-driven rounds over active tiles */
#define DTB_FLAG_REF_NO_FMA 0x4u  /* ref-mode: round l_eucl*d and l_grad*|dI| separately instead of contracting */
#define DTB_FLAG_TIMING 0x8u      /* record CUDA events around the tile kernel; dtb_stats.kernel_ms */

/* Counters of the last synchronous call (or of the call waited for by dtb_sync). */
typedef struct dtb_stats {
  uint64_t tiles;         /* tiles in the call */
  uint64_t tile_visits;   /* warp visits of tiles (>= tiles reached) */
  uint64_t phases;        /* sweep phases over all visits */
  uint64_t activations;   /* neighbour re-activations issued */
  uint64_t rounds;        /* host rounds (DTB_FLAG_ROUNDS), else 1 */
  uint32_t device_error;  /* 0, or the device error code */
  uint32_t device_error_info;
  double kernel_ms;       /* DTB_FLAG_TIMING: device time of the tile kernel(s) of the call, else 0 */
  uint64_t h2d_bytes;     /* host-buffer batches: bytes copied host -> device (images, masks, tables), else 0 */
  uint64_t d2h_bytes;     /* host-buffer batches: bytes copied device -> host (maps), else 0 */
} dtb_stats;

DTB_API int32_t dtb_abi_version(void);
DTB_API const char* dtb_status_string(dtb_status s);

/* Context: owns device scratch (tile states, queue ring, descriptor tables, staging copies).
 * device < 0 selects the current device. */
DTB_API dtb_status dtb_context_create(int32_t device, dtb_context* out);
DTB_API void dtb_context_destroy(dtb_context ctx);
/* Detailed text of the last error of this context ("" if none). */
DTB_API const char* dtb_context_message(dtb_context ctx);
DTB_API dtb_status dtb_last_stats(dtb_context ctx, dtb_stats* out);
/* Waits for work enqueued with DTB_FLAG_ASYNC on `stream` and for every asynchronous host-buffer batch of the
 * context, and returns their device status. */
DTB_API dtb_status dtb_sync(dtb_context ctx, void* stream);

/* Launch tuning and queue policy of the ns-mode tile kernel (chosen by dtb_plan_autotune, or set by hand).
 * The reference fixes its choices at build time: 64 priority levels from seed distances
 * (dt/src/task_queue.cuh:23, dt/src/block_priority.cu:71-155) and 4 blocks of one warp per SM
 * (dt/src/generalised_distance_transform_task.cu:184).  0 keeps a field's current value.
 * ctas_per_sm and warps_per_cta: the launch shape, one warp per 32 x 32 tile visit; (2, 4), (3, 4), (4, 4),
 * (6, 2), (2, 6) or (2, 8) -- 8, 12 or 16 warps per SM, registers per thread 255 / 168 / 128 (with only
 * ctas_per_sm given, warps_per_cta stays if it fits, else becomes 4);
 * grid_percent: share of the co-resident CTAs launched, 1..100 (fewer workers re-visit fewer tiles on
 * narrow fronts); host_chunk_kpx: pixels (in units of 1024) per chunk of the pipeline that serves batches in
 * host memory (host-to-device copies, tile runs on two alternating compute lanes and device-to-host copies of
 * successive chunks overlap; default 16384); queue_buckets: 1 = one FIFO ring, or 2 / 4 / 8 / 16 rings ordered
 * by the distance an activation can bring (default 8); bucket_width_pct: width of one bucket in percent of
 * one tile-width of path cost of the image (32 x its mean edge weight), 1..6400 (default 50);
 * staging: 1 = a visit stages its own tile, 2 = a warp stages the image box of its next tile while it visits
 * the current one (double-buffered shared memory; ctas_per_sm 2 or 3 only). */
typedef struct dtb_tuning {
  int32_t ctas_per_sm;
  int32_t grid_percent;
  int32_t host_chunk_kpx;
  int32_t queue_buckets;
  int32_t bucket_width_pct;
  int32_t staging;
  int32_t warps_per_cta;
} dtb_tuning;
DTB_API dtb_status dtb_context_set_tuning(dtb_context ctx, const dtb_tuning* t);
DTB_API dtb_status dtb_context_get_tuning(dtb_context ctx, dtb_tuning* t);

/* Reference-weight GGDT (C8 neighbourhood, D(q) + (1-lambda)*{1, sqrt2} + lambda*|I(p)-I(q)|), gray input.
 * Replaces dt::generalised_distance_transform (generalised_distance_transform.hpp:7-8),
 * dt::generalised_distance_transform_blocks (:13-15) and dt::generalised_distance_transform_task (:21-23):
 * all three converge to the same map.  img, mask: elem_size 1; dist: elem_size 4; same width/height.
 * 0 <= lambda <= 1, v >= 0 (the reference default is v = 1e10).  Images may be CPU or GPU memory. */
DTB_API dtb_status dtb_gdt_ref(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist,
                               float lambda, float v, uint32_t flags, void* stream);

/* dt::generalised_distance_transform_blocks with its round counters
 * (generalised_distance_transform.hpp:13-15, _blocks.cu:114-165): ref-mode GGDT by host-driven rounds over
 * active 32x32 tiles (DTB_FLAG_ROUNDS is implied).  rounds_per_tile, if not NULL, points to
 * ceil(width/32) * ceil(height/32) int32 counters, tile (bx, by) at index by * ceil(width/32) + bx, in host or
 * device memory; each is incremented once per round in which its tile was visited.  As in the reference, the
 * first round visits every tile and a tile runs again in a later round when a neighbour's border changed.
 * Same map as dtb_gdt_ref. */
DTB_API dtb_status dtb_gdt_ref_blocks(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist,
                                      float lambda, float v, int32_t* rounds_per_tile, uint32_t flags, void* stream);

/* Geodesic GGDT with C4 connectivity and w(p,q) = sqrt(1 + gamma^2 * |I(p)-I(q)|^2); gray (elem_size 1)
 * or rgb8 (elem_size 3, |.| the Euclidean RGB difference).  Extends the reference entry point of
 * generalised_distance_transform.hpp:7-8 to the C4 neighbourhood (dt/include/dt/c4.hpp:9-27) and rgb8. */
DTB_API dtb_status dtb_gdt(dtb_context ctx, const dtb_image* img, const dtb_image* mask, const dtb_image* dist,
                           float gamma, float v, uint32_t flags, void* stream);

/* Ragged batch of n independent images (any mix of gray and rgb8, any sizes) in one persistent launch
 * over a shared tile queue.  gammas[i] per image.  No reference counterpart (the reference runs one image
 * per call). */
DTB_API dtb_status dtb_gdt_batch(dtb_context ctx, int32_t n, const dtb_image* imgs, const dtb_image* masks,
                                 const dtb_image* dists, const float* gammas, float v, uint32_t flags, void* stream);

/* Batch plans: a ragged ns-mode batch prepared once and run many times.  dtb_plan_create validates the views
 * (device memory only: images and masks 16-byte aligned in buffer and pitch, distances 4-byte aligned), builds
 * the image descriptors and TMA tensor maps, allocates the plan's own device scratch and captures one run
 * (queue reset, seed scan, the cooperative persistent tile kernel, finalize) in a CUDA graph.  The buffers
 * must stay allocated while the plan lives; their contents may change between runs.  dtb_plan_run launches
 * the graph on `stream` and returns; dtb_plan_wait waits for it and returns the device status and counters
 * (flags: reserved, pass 0).  dtb_plan_autotune searches, on this batch (median of reps runs each), the
 * tile-kernel variant (CTAs per SM, staging), the grid share and the tile-queue policy (FIFO, or 8 / 16
 * distance-ordered buckets of 1/4, 1/2 or 1 tile-width of path cost): variants x grid shares first, then the
 * queue policies under the best launch, then the variants again under the best policy.  It keeps the fastest
 * in the plan and, for batches of the same size class (image count and tile count, each rounded up to a power
 * of two), in the context and in its autotuner cache file if one is set; and reports it.  dtb_plan_get_tuning
 * reports the plan's current tuning.  No reference counterpart: the reference fixes these choices
 * (dt/src/task_queue.cuh:23, dt/src/generalised_distance_transform_task.cu:184). */
typedef struct dtb_plan_s* dtb_plan;
DTB_API dtb_status dtb_plan_create(dtb_context ctx, int32_t n, const dtb_image* imgs, const dtb_image* masks,
                                   const dtb_image* dists, const float* gammas, float v, uint32_t flags, dtb_plan* out);
DTB_API dtb_status dtb_plan_run(dtb_plan plan, void* stream);
DTB_API dtb_status dtb_plan_wait(dtb_plan plan, void* stream, dtb_stats* stats);
DTB_API dtb_status dtb_plan_autotune(dtb_plan plan, void* stream, int32_t reps, dtb_tuning* chosen);
DTB_API dtb_status dtb_plan_get_tuning(dtb_plan plan, dtb_tuning* out);
DTB_API void dtb_plan_destroy(dtb_plan plan);

/* Autotuner cache file (JSON, {"format": "dtb-autotune-1", "entries": [...]}, one entry per GPU name and size
 * class): loads this GPU's entries into the context (plans and calls of those size classes start from them)
 * and makes dtb_plan_autotune write its results there (entries of other GPUs and size classes are kept; the
 * file is replaced atomically).  A missing file is not an error; NULL or "" turns the cache off.  The
 * environment variable DTB_AUTOTUNE_CACHE names a cache that dtb_context_create loads. */
DTB_API dtb_status dtb_context_set_tuning_cache(dtb_context ctx, const char* path);

/* Serving engine: continuous batching of requests on one device.  A worker thread runs waves: each wave
 * admits, in arrival order, the pending requests that fit the device-memory budget (evicting least recently
 * used idle images) and runs all of them in one persistent launch over a shared tile queue; requests that
 * arrive meanwhile join the next wave.  Images stay resident with their distance maps, so a seed edit
 * warm-starts from the previous map (exact: added seeds only lower distances).  No reference counterpart.
 * Request data (img, mask, out buffers) is host memory owned by the caller and must stay valid until the
 * request's completion has been returned by dtb_serve_poll; the disk list is copied by dtb_serve_submit.
 * dtb_serve_create allocates everything the engine uses: the resident arena (hbm_budget_bytes) and, for each of
 * the two waves that can be in flight, its scratch, staging and pinned table buffers, sized by the per-wave
 * limits of the config; a wave that would exceed a limit is closed and the rest waits for the next wave, so no
 * allocation and no device-wide synchronisation happens while waves run.  An edit may add at most 65536 disks.
 * With live = 1 there are no waves: one persistent tile kernel keeps running while requests flow, and each
 * request is published into a device ring once its image is copied in; idle warps of the running kernel claim
 * it and queue its work beside the tiles of the requests already running (a new image's set-up -- tile states
 * and the seed scan -- runs as kernel jobs; an edit draws its disks and queues the tiles they touch), so a
 * request never waits for another to end.  Each request's completion is signalled by the kernel itself, and
 * its map is copied out while the kernel goes on.  The kernel occupies every SM while it runs and ends after
 * live_idle_us without work; the engine launches it again for the next request.  The live tile queue is one
 * FIFO ring.  A request whose run fails (a device error, or dtb_debug_inject_queue_stall) drops its image. */
#define DTB_REQ_IMAGE 0  /* new image: img (gray / rgb8), mask, gamma; resident under image_id afterwards */
#define DTB_REQ_EDIT 1   /* seed edit of the resident image image_id: n_disks disks (cx, cy, r) added */
typedef struct dtb_serve_config {
  uint64_t hbm_budget_bytes;  /* device memory reserved for resident images, masks and maps */
  int32_t max_wave_requests;  /* at most this many requests per wave (0 = 4096) */
  float v;                    /* value of unreached pixels (>= 0) */
  uint32_t max_wave_tiles;    /* at most this many 32 x 32 tiles per wave (0 = 2^20); an image alone above it is
                                 rejected with DTB_ERR_CAPACITY */
  uint64_t wave_stage_bytes;  /* device staging per wave for new images whose rows need a new pitch (0 = 256 MiB) */
  int32_t live;               /* 0: waves; 1: live admission -- requests join the tile queue of one persistent kernel
                                 that keeps running, and max_wave_requests / max_wave_tiles bound the requests and
                                 tiles in flight at once */
  uint32_t live_idle_us;      /* live: the kernel ends after this long with nothing queued and nothing claimed
                                 (0 = 20000); the next request launches it again */
} dtb_serve_config;
typedef struct dtb_serve_request {
  int32_t kind;
  int64_t image_id;
  dtb_image img;
  dtb_image mask;
  float gamma;
  int32_t n_disks;
  const int32_t* disks;
  dtb_image out;  /* host float map (elem_size 4) of the image's size: the result */
} dtb_serve_request;
typedef struct dtb_serve_completion {
  int64_t request_id;
  int32_t status;     /* dtb_status of the request */
  double latency_ms;  /* from dtb_serve_submit to the result being in `out` */
} dtb_serve_completion;
typedef struct dtb_serve_stats {
  int64_t submitted, completed, failed, waves, evictions, pending, resident_images;
  uint64_t resident_bytes, tiles, tile_visits;
  /* Where the time of the ended waves went (sums over waves, milliseconds): host preparation of a wave (admission
   * to the last enqueue), its copies in (first to last, stream time), its tile run (scan or warm start, persistent
   * kernel, finalize) and its copies out; and the requests' queueing (submit to the start of their wave's
   * preparation; sum and maximum over requests). */
  double host_prep_ms, copy_in_ms, kernel_ms, copy_out_ms, queue_wait_ms, queue_wait_max_ms;
  int64_t waves_split;        /* waves closed by a per-wave limit (tiles, staging, disks) with requests left over */
  /* Live engine: launches of the live kernel that ended idle (live_idle_us without work), at the end of their
   * lifetime (4 s, then drained), on a device error, or on dtb_serve_destroy. */
  int64_t live_ended_idle, live_ended_lifetime, live_ended_error, live_ended_stop;
} dtb_serve_stats;
typedef struct dtb_server_s* dtb_server;
DTB_API dtb_status dtb_serve_create(dtb_context ctx, const dtb_serve_config* cfg, dtb_server* out);
DTB_API dtb_status dtb_serve_submit(dtb_server s, const dtb_serve_request* r, int64_t* request_id);
/* Returns up to max completions, waiting up to wait_ms for the first one. */
DTB_API int32_t dtb_serve_poll(dtb_server s, dtb_serve_completion* out, int32_t max, int32_t wait_ms);
DTB_API dtb_status dtb_serve_release(dtb_server s, int64_t image_id);
DTB_API dtb_status dtb_serve_get_stats(dtb_server s, dtb_serve_stats* out);
DTB_API void dtb_serve_destroy(dtb_server s);

/* Allocation-free dtb_gdt for one image; no counterpart in the reference.
 * For callers that must not allocate device memory behind their own allocator: a host that owns all device
 * memory through its own pool or budget, or a loop that cannot afford the device-wide synchronisation of
 * cudaMalloc / cudaFree.  No context: the scratch is a fixed array in the library's device memory (about
 * 324 KB on every GPU that loads the library, held until exit), so the image may have at most 16384 tiles of
 * 32 x 32 pixels (e.g. 4096 x 4096); larger images return DTB_ERR_CAPACITY.  img, mask and dist must be device
 * memory, img and mask with 16-byte aligned buffer and pitch, dist with 4-byte alignment (no staging copies);
 * otherwise DTB_ERR_INVALID_ARG.  Synchronous: returns after the map is written.  The first call on a device
 * does a one-time set-up with that device current (symbol address, driver entry point, kernel attributes);
 * make that first call before any stream capture.  Every call reuses the same array and clears what must start
 * at zero; calls that overlap on the GPU (other threads or streams) race on it and must be serialised. */
DTB_API dtb_status dtb_gdt_noalloc(const dtb_image* img, const dtb_image* mask, const dtb_image* dist, float gamma,
                                   float v, void* stream);

/* Failure-detection self-test (host-side injection, no device fault): the next persistent tile run of this
 * context (a call, or the next wave of a server created on it) counts one queued tile that is never pushed and
 * uses timeout_ms (1..60000) as the no-progress limit of its tile queue.  Its workers find no work, the bounded
 * wait in every worker ends, the kernel returns and the call (or every request of the wave) reports
 * DTB_ERR_TIMEOUT; the context and the server stay usable.  One-shot. */
DTB_API dtb_status dtb_debug_inject_queue_stall(dtb_context ctx, uint32_t timeout_ms);

/* Pitched image storage, reference dt::image2d<T> allocation (dt/include/dt/image2d.hpp:36-50,
 * details/image2d_data_gpu.hpp:23-39).  DTB_GPU: device memory of the current device, pitch rounded up to
 * 128 bytes (the alignment the tile kernel's bulk tensor copies read fastest); DTB_CPU: host memory, pitch =
 * width * elem_size as in the reference.  Fills *out (buffer, width, height, pitch, elem_size, memory_kind).
 * dtb_image_free releases it (NULL buffer: no-op) and clears out->buffer. */
DTB_API dtb_status dtb_image_alloc(int32_t width, int32_t height, int32_t elem_size, int32_t memory_kind, dtb_image* out);
DTB_API dtb_status dtb_image_free(dtb_image* img);

/* Image files, reference dt::imread / dt::imsave (dt/include/dt/imread.hpp:7-8, imsave.hpp:13-43; the reference
 * reads any stb_image format and writes PNG).  Formats: PNG (read: gray, gray + alpha, rgb, rgba, palette at 8 bits
 * per sample, gray and palette also at 1 / 2 / 4, not interlaced; write: 8-bit gray or rgb), binary PGM / PPM, and
 * JPEG on read (baseline, extended and progressive Huffman frames of 8-bit samples, 1 or 3 components, restart
 * intervals; gray samples identical to stb_image's, the decoder the reference's benchmark inputs go through),
 * chosen by the file name (.png, .pgm, .ppm) on write and by the contents on read.  dtb_image_read: `channels` 1 (gray) or 3 (rgb8) must match the file's
 * components, as the reference requires one component for imread<uint8_t>; the pixels go into new host memory
 * (free with dtb_image_free).  dtb_image_write: a host image of elem_size 1 or 3. */
DTB_API dtb_status dtb_image_read(const char* path, int32_t channels, dtb_image* out);
DTB_API dtb_status dtb_image_write(const char* path, const dtb_image* img);

/* Host <-> device copies of a pitched image, reference dt::host_to_device / dt::device_to_host
 * (dt/include/dt/transfert.hpp:13-15, dt/src/transfert.cpp:10-28).  Synchronous when stream is NULL. */
DTB_API dtb_status dtb_host_to_device(const dtb_image* src, const dtb_image* dst, void* stream);
DTB_API dtb_status dtb_device_to_host(const dtb_image* src, const dtb_image* dst, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DTB_H */
