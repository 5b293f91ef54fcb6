// dtb_plan.cu -- batch plans: a ragged ns-mode batch prepared once, captured in a CUDA graph, run many times;
// and the autotuner that picks the tile-kernel launch variant for a batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
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

}  // namespace

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
  p->L = layout_for(n, total, workers, false);
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
  dtb_context ctx = p->ctx;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaEvent_t a, b;
  DTB_CUDA(ctx, cudaEventCreate(&a));
  DTB_CUDA(ctx, cudaEventCreate(&b));
  static const int kPercent[3] = {100, 75, 50};
  float best_ms = INFINITY;
  LaunchTuning best = p->tuning;
  dtb_status s = DTB_OK;
  for (int v = 0; v < NS_VARIANTS && s == DTB_OK; ++v) {
    for (int pc = 0; pc < 3 && s == DTB_OK; ++pc) {
      p->tuning = LaunchTuning{v, kPercent[pc]};
      if ((s = capture(p)) != DTB_OK) break;
      if ((s = dtb_plan_run(p, stream)) != DTB_OK || (s = dtb_plan_wait(p, stream, nullptr)) != DTB_OK) break;
      std::vector<float> t;
      for (int r = 0; r < reps && s == DTB_OK; ++r) {
        cudaEventRecord(a, st);
        s = dtb_plan_run(p, stream);
        cudaEventRecord(b, st);
        if (s == DTB_OK) s = dtb_plan_wait(p, stream, nullptr);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        t.push_back(ms);
      }
      if (s != DTB_OK) break;
      std::sort(t.begin(), t.end());
      const float med = t[t.size() / 2];
      if (med < best_ms) {
        best_ms = med;
        best = p->tuning;
      }
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
  }
  if (chosen) {
    chosen->ctas_per_sm = NS_VARIANT_CTAS[best.variant];
    chosen->grid_percent = best.grid_percent;
    chosen->host_chunk_kpx = (int32_t)(ctx->host_chunk_px / 1024ull);
  }
  return DTB_OK;
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
