// dtb_plan.cu -- batch plans: a ragged ns-mode batch prepared once, captured in a CUDA graph, run many times;
// the autotuner that picks the tile-kernel variant (CTAs per SM x warps per CTA, staging), grid share and tile-queue policy
// (FIFO or distance-ordered buckets, their count and width) for a batch; and its JSON cache, keyed by GPU
// name and workload size class, which later processes reuse.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "dtb.h"
#include "dtb_internal.h"

using namespace dtb;

struct dtb_plan_s {
  dtb_context ctx = nullptr;
  std::vector<Job> jobs;
  ScratchLayout L;
  uint8_t* dbase = nullptr;
  LaunchTuning tuning;
  uint64_t key = 0;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  dtb_stats stats{};
};

namespace {

void drop_graph(dtb_plan p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->exec = nullptr;
  p->graph = nullptr;
}

// Captures queue reset + seed scan + tile kernel + finalize with the plan's current tuning.
dtb_status capture(dtb_plan p) {
  drop_graph(p);
  dtb_context ctx = p->ctx;
  DTB_CUDA(ctx, cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
  dtb_status s = enqueue_persistent(ctx, p->dbase, p->L, MODE_NS, p->tuning, p->cap, nullptr, nullptr);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(p->cap, &g);
  if (s != DTB_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
  p->graph = g;
  DTB_CUDA(ctx, cudaGraphInstantiate(&p->exec, p->graph, 0));
  return DTB_OK;
}

bool aligned16(const dtb_image* im) {
  return (reinterpret_cast<uintptr_t>(im->buffer) & 15u) == 0 && (im->pitch & 15) == 0;
}

// ---- autotuner cache: {"format": "dtb-autotune-1", "entries": [{"gpu": ..., "images_pow2": ..., ...}, ...]} ----
struct CacheEntry {
  std::string gpu;
  uint64_t images = 0, tiles = 0;
  int ctas = 0, staging = 0, grid = 0, buckets = 0, width_pct = 0, wpc = 4;  // wpc: 4 in caches written without it
  double ms = 0.0;
};

// Parses the flat entry objects of a cache file (string and number values only, as written below).
std::vector<CacheEntry> parse_cache(const std::string& text) {
  std::vector<CacheEntry> out;
  size_t i = text.find("\"entries\"");
  if (i == std::string::npos) return out;
  i = text.find('[', i);
  while (i != std::string::npos) {
    const size_t o = text.find('{', i), e = text.find('}', o == std::string::npos ? i : o);
    if (o == std::string::npos || e == std::string::npos) break;
    CacheEntry c;
    size_t k = o + 1;
    while (k < e) {
      const size_t q0 = text.find('"', k);
      if (q0 == std::string::npos || q0 >= e) break;
      const size_t q1 = text.find('"', q0 + 1);
      const size_t colon = text.find(':', q1);
      if (q1 == std::string::npos || colon == std::string::npos || colon >= e) break;
      const std::string key = text.substr(q0 + 1, q1 - q0 - 1);
      size_t v = colon + 1;
      while (v < e && std::isspace((unsigned char)text[v])) ++v;
      std::string val;
      if (v < e && text[v] == '"') {
        const size_t v1 = text.find('"', v + 1);
        if (v1 == std::string::npos || v1 > e) break;
        val = text.substr(v + 1, v1 - v - 1);
        k = v1 + 1;
      } else {
        size_t v1 = v;
        while (v1 < e && text[v1] != ',' && !std::isspace((unsigned char)text[v1])) ++v1;
        val = text.substr(v, v1 - v);
        k = v1;
      }
      if (key == "gpu") c.gpu = val;
      else if (key == "images_pow2") c.images = std::strtoull(val.c_str(), nullptr, 10);
      else if (key == "tiles_pow2") c.tiles = std::strtoull(val.c_str(), nullptr, 10);
      else if (key == "ctas_per_sm") c.ctas = std::atoi(val.c_str());
      else if (key == "staging") c.staging = std::atoi(val.c_str());
      else if (key == "warps_per_cta") c.wpc = std::atoi(val.c_str());
      else if (key == "grid_percent") c.grid = std::atoi(val.c_str());
      else if (key == "queue_buckets") c.buckets = std::atoi(val.c_str());
      else if (key == "bucket_width_pct") c.width_pct = std::atoi(val.c_str());
      else if (key == "ms") c.ms = std::atof(val.c_str());
    }
    out.push_back(c);
    i = e + 1;
    if (text.find('{', i) == std::string::npos) break;
  }
  return out;
}

bool read_file(const std::string& path, std::string* out) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) out->append(buf, n);
  std::fclose(f);
  return true;
}

uint64_t key_of(const CacheEntry& c) { return (c.images << 32) | c.tiles; }

}  // namespace

namespace dtb {

// Entries of this context's GPU whose fields are valid go into ctx->tuned (the caller holds ctx->mu).
dtb_status load_tuning_cache(dtb_context ctx) {
  std::string text;
  if (!read_file(ctx->tune_cache_path, &text)) return DTB_OK;  // no cache yet
  for (const CacheEntry& c : parse_cache(text)) {
    if (c.gpu != ctx->gpu_name) continue;
    const int v = ns_variant_of(c.ctas, c.staging == 2, c.wpc);
    if (v < 0 || c.grid < 1 || c.grid > 100 || !valid_policy(c.buckets, (float)c.width_pct / 100.0f)) continue;
    LaunchTuning t;
    t.variant = v;
    t.grid_percent = c.grid;
    t.buckets = c.buckets;
    t.bucket_tiles = (float)c.width_pct / 100.0f;
    ctx->tuned[key_of(c)] = t;
  }
  return DTB_OK;
}

// Rewrites the cache file with the entry of (this GPU, key) replaced by t (other entries kept); written to a
// temporary file first and renamed, so readers never see a partial file (the caller holds ctx->mu).
dtb_status save_tuning_cache(dtb_context ctx, uint64_t key, const LaunchTuning& t, double ms) {
  std::string text;
  std::vector<CacheEntry> entries;
  if (read_file(ctx->tune_cache_path, &text)) entries = parse_cache(text);
  CacheEntry n;
  n.gpu = ctx->gpu_name;
  n.images = key >> 32;
  n.tiles = key & 0xFFFFFFFFull;
  n.ctas = NS_VARIANT_TABLE[t.variant].ctas;
  n.staging = NS_VARIANT_TABLE[t.variant].ahead ? 2 : 1;
  n.wpc = NS_VARIANT_TABLE[t.variant].wpc;
  n.grid = t.grid_percent;
  n.buckets = t.buckets;
  n.width_pct = (int)lrintf(t.bucket_tiles * 100.0f);
  n.ms = ms;
  bool replaced = false;
  for (CacheEntry& c : entries)
    if (c.gpu == n.gpu && key_of(c) == key) {
      c = n;
      replaced = true;
    }
  if (!replaced) entries.push_back(n);
  const std::string tmp = ctx->tune_cache_path + ".tmp";
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return fail(ctx, DTB_ERR_IO, "cannot write %s", tmp.c_str());
  std::fprintf(f, "{\"format\": \"dtb-autotune-1\", \"entries\": [");
  for (size_t i = 0; i < entries.size(); ++i) {
    const CacheEntry& c = entries[i];
    std::fprintf(f,
                 "%s\n  {\"gpu\": \"%s\", \"images_pow2\": %llu, \"tiles_pow2\": %llu, \"ctas_per_sm\": %d, \"staging\": %d, "
                 "\"warps_per_cta\": %d, \"grid_percent\": %d, \"queue_buckets\": %d, \"bucket_width_pct\": %d, \"ms\": %.4f}",
                 i ? "," : "", c.gpu.c_str(), (unsigned long long)c.images, (unsigned long long)c.tiles, c.ctas, c.staging,
                 c.wpc, c.grid, c.buckets, c.width_pct, c.ms);
  }
  std::fprintf(f, "\n]}\n");
  const bool ok = std::fclose(f) == 0 && std::rename(tmp.c_str(), ctx->tune_cache_path.c_str()) == 0;
  return ok ? DTB_OK : fail(ctx, DTB_ERR_IO, "cannot write %s", ctx->tune_cache_path.c_str());
}

}  // namespace dtb

extern "C" {

DTB_API dtb_status dtb_plan_create(dtb_context ctx, int32_t n, const dtb_image* imgs, const dtb_image* masks,
                                   const dtb_image* dists, const float* gammas, float v, uint32_t flags, dtb_plan* out) {
  if (!ctx || !out) return DTB_ERR_INVALID_ARG;
  *out = nullptr;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->msg.clear();
  if (n < 0 || (n > 0 && (!imgs || !masks || !dists || !gammas))) return fail(ctx, DTB_ERR_INVALID_ARG, "bad batch arrays");
  if (!(v >= 0.0f)) return fail(ctx, DTB_ERR_INVALID_ARG, "v must be >= 0");
  dtb_plan p = new (std::nothrow) dtb_plan_s();
  if (!p) return DTB_ERR_OUT_OF_MEMORY;
  p->ctx = ctx;
  (void)flags;
  auto bail = [&](dtb_status s) {
    dtb_plan_destroy(p);
    return s;
  };
  for (int i = 0; i < n; ++i) {
    dtb_status s = check_triplet(ctx, &imgs[i], &masks[i], &dists[i], true);
    if (s != DTB_OK) return bail(fail(ctx, s, "image %d: %s", i, ctx->msg.c_str()));
    if (imgs[i].width > 0 && imgs[i].height > 0) {
      if (imgs[i].memory_kind != DTB_GPU || masks[i].memory_kind != DTB_GPU || dists[i].memory_kind != DTB_GPU)
        return bail(fail(ctx, DTB_ERR_INVALID_ARG, "image %d: plans take device memory only", i));
      if (!aligned16(&imgs[i]) || !aligned16(&masks[i]) || (reinterpret_cast<uintptr_t>(dists[i].buffer) & 3u) ||
          (dists[i].pitch & 3))
        return bail(fail(ctx, DTB_ERR_INVALID_ARG, "image %d: buffers are not aligned for TMA", i));
    }
    if (!(gammas[i] >= 0.0f) || std::isinf(gammas[i])) return bail(fail(ctx, DTB_ERR_INVALID_ARG, "image %d: bad gamma", i));
    Job j = Job::from(&imgs[i], &masks[i], &dists[i]);
    j.mode = MODE_NS;
    j.v = v;
    j.g2 = gamma_to_g2(gammas[i]);
    p->jobs.push_back(j);
  }
  uint32_t total = 0;
  dtb_status s = count_tiles(ctx, p->jobs, &total);
  if (s != DTB_OK) return bail(s);
  // The ring must hold every resident warp of any variant the autotuner may pick.
  uint32_t workers = 0;
  for (int k = 0; k < NS_VARIANTS; ++k) workers = std::max(workers, resident_workers(ctx, MODE_NS, LaunchTuning{k, 100}));
  p->L = layout_for(n, total, workers, false, NBUCKET_MAX);  // room for every queue policy of the autotuner
  p->key = tuning_key(n, total);
  auto it = ctx->tuned.find(p->key);
  p->tuning = it != ctx->tuned.end() ? it->second : ctx->tuning;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return bail(DTB_ERR_CUDA);
  cudaError_t e = cudaMalloc((void**)&p->dbase, p->L.bytes);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "cudaMalloc(plan scratch)"));
  std::vector<uint8_t> tables;
  if ((s = build_tables(ctx, p->jobs, p->L, tables)) != DTB_OK) return bail(s);
  e = cudaMemcpy(p->dbase + p->L.o_desc, tables.data(), tables.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "cudaMemcpy(plan tables)"));
  if ((e = cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(cuda_fail(ctx, e, "plan capture stream"));
  if ((s = capture(p)) != DTB_OK) return bail(s);
  p->stats.tiles = total;
  *out = p;
  return DTB_OK;
}

DTB_API dtb_status dtb_plan_run(dtb_plan p, void* stream) {
  if (!p || !p->exec) return DTB_ERR_INVALID_ARG;
  const TraceRange trace("dtb plan run");
  DTB_CUDA(p->ctx, cudaGraphLaunch(p->exec, reinterpret_cast<cudaStream_t>(stream)));
  return DTB_OK;
}

DTB_API dtb_status dtb_plan_wait(dtb_plan p, void* stream, dtb_stats* stats) {
  if (!p) return DTB_ERR_INVALID_ARG;
  dtb_context ctx = p->ctx;
  DTB_CUDA(ctx, cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
  dtb_stats st{};
  st.tiles = p->L.total;
  st.rounds = 1;
  const dtb_status s = read_device_status(ctx, reinterpret_cast<QueueHdr*>(p->dbase + p->L.o_hdr), &st);
  p->stats = st;
  if (stats) *stats = st;
  return s;
}

DTB_API dtb_status dtb_plan_autotune(dtb_plan p, void* stream, int32_t reps, dtb_tuning* chosen) {
  if (!p || reps < 1) return DTB_ERR_INVALID_ARG;
  const TraceRange trace("dtb autotune");
  dtb_context ctx = p->ctx;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaEvent_t a, b;
  DTB_CUDA(ctx, cudaEventCreate(&a));
  DTB_CUDA(ctx, cudaEventCreate(&b));
  float best_ms = INFINITY;
  LaunchTuning best = p->tuning;
  dtb_status s = DTB_OK;
  // Median time of `reps` graph runs under tuning t (after one untimed run); keeps the fastest.
  auto trial = [&](const LaunchTuning& t) {
    if (s != DTB_OK) return;
    p->tuning = t;
    if ((s = capture(p)) != DTB_OK) return;
    if ((s = dtb_plan_run(p, stream)) != DTB_OK || (s = dtb_plan_wait(p, stream, nullptr)) != DTB_OK) return;
    std::vector<float> ts;
    for (int r = 0; r < reps && s == DTB_OK; ++r) {
      cudaEventRecord(a, st);
      s = dtb_plan_run(p, stream);
      cudaEventRecord(b, st);
      if (s == DTB_OK) s = dtb_plan_wait(p, stream, nullptr);
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, a, b);
      ts.push_back(ms);
    }
    if (s != DTB_OK) return;
    std::sort(ts.begin(), ts.end());
    const float med = ts[ts.size() / 2];
    if (med < best_ms) {
      best_ms = med;
      best = t;
    }
  };
  // Coordinate search: (1) kernel variant (CTAs per SM x warps per CTA x staging) x grid share under the current
  // queue policy; (2) queue policy (FIFO; 8 or 16 buckets of 1/10, 1/4, 1/2 or 1 tile-width) under the best launch;
  // (3) the variants again under the best policy.
  static const int kPercent[3] = {100, 75, 50};
  const LaunchTuning start = p->tuning;
  for (int v = 0; v < NS_VARIANTS; ++v)
    for (int pc = 0; pc < 3; ++pc) {
      LaunchTuning t = start;
      t.variant = v;
      t.grid_percent = kPercent[pc];
      trial(t);
    }
  {
    const LaunchTuning launch = best;
    LaunchTuning t = launch;
    t.buckets = 1;
    trial(t);
    static const int kBuckets[2] = {8, 16};
    static const float kWidth[4] = {0.1f, 0.25f, 0.5f, 1.0f};
    for (int nb : kBuckets)
      for (float w : kWidth) {
        t = launch;
        t.buckets = nb;
        t.bucket_tiles = w;
        trial(t);
      }
  }
  {
    const LaunchTuning policy = best;
    for (int v = 0; v < NS_VARIANTS; ++v) {
      LaunchTuning t = policy;
      t.variant = v;
      trial(t);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  p->tuning = best;
  if (s != DTB_OK) return s;
  if ((s = capture(p)) != DTB_OK) return s;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tuned[p->key] = best;
    if (!ctx->tune_cache_path.empty()) save_tuning_cache(ctx, p->key, best, best_ms);
  }
  if (chosen) tuning_to_abi(ctx, best, chosen);
  return DTB_OK;
}

DTB_API dtb_status dtb_plan_get_tuning(dtb_plan p, dtb_tuning* out) {
  if (!p || !out) return DTB_ERR_INVALID_ARG;
  tuning_to_abi(p->ctx, p->tuning, out);
  return DTB_OK;
}

DTB_API dtb_status dtb_context_set_tuning_cache(dtb_context ctx, const char* path) {
  if (!ctx) return DTB_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->tune_cache_path = path ? path : "";
  if (ctx->tune_cache_path.empty()) return DTB_OK;
  return load_tuning_cache(ctx);
}

DTB_API void dtb_plan_destroy(dtb_plan p) {
  if (!p) return;
  if (p->cap) cudaStreamSynchronize(p->cap);
  drop_graph(p);
  if (p->dbase) cudaFree(p->dbase);
  if (p->cap) cudaStreamDestroy(p->cap);
  delete p;
}

}  // extern "C"
