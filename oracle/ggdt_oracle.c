/*
 * ggdt_oracle.c -- CPU restatement of the reference's generalised geodesic distance transform.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: it may be loaded by tests/,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline / reference legs, never by the product
 * library in distance_transform_benchmarks_b200/.
 *
 * Parity pinning
 *   ref-mode (C8, lambda blend, gray) is pinned by the two golden tensors of the reference test suite
 *   (tests/distance_transform.cpp:14-281 and :283-476), extracted by tests/golden/make_golden.py and
 *   checked bit-exactly in tests/test_oracle.py.
 *   ns-mode (C4, w = sqrt(1 + g2*dI^2), gray or rgb8) has no counterpart in the reference, so it is
 *   "parity unpinned" with respect to the reference: it shares the fixpoint solver with ref-mode and is
 *   cross-checked against the FP64 Dijkstra below.
 *
 * Algorithm
 *   Both modes compute the greatest fixpoint of single-edge relaxations
 *        D(p) <- min(D(p), relax(D(q), edge q->p))
 *   starting from D = v where mask == 0 and D = 0 where mask != 0
 *   (reference dt/src/utils.cu:12, `D(x, y) = v * (mask(x, y) == 0)`).
 *   relax() is monotone in D(q), so every schedule that runs to quiescence ends in the same fixpoint:
 *   the raster schedule of the reference (dt/src/generalised_distance_transform.cu:126-134: forward rows,
 *   backward rows, forward columns, backward columns, repeated until nothing changes) is used here.
 *
 *   ref-mode relax, reference dt/src/generalised_distance_transform.cu:44-45 and
 *   dt/src/dt_block_passes.cuh:45-46:
 *        D(q) + l_eucl * local_dist2d[k] + l_grad * |I(p) - I(q)|
 *   with local_dist2d = {sqrt(2), 1, sqrt(2)} (generalised_distance_transform.cu:111), l_grad = lambda,
 *   l_eucl = 1 - lambda (:108-109), |I(p) - I(q)| on uint8 (dt/src/utils.cuh:38-41).  The reference is
 *   built without --fmad=false, so the oracle offers both the contracted form
 *        fmaf(l_grad, |dI|, fmaf(l_eucl, d, D(q)))
 *   and the plain left-to-right form; for lambda in {0, 0.5, 1} every product is exact and they agree.
 *   Out-of-image neighbours are skipped (generalised_distance_transform.cu:41-42).
 *
 *   ns-mode relax: D(q) + w(p,q), w = sqrtf(1 + g2 * dI2), dI2 = sum over channels of (I_c(p)-I_c(q))^2
 *   (an exact integer in fp32), every operation rounded to fp32 (this file is compiled with
 *   -ffp-contract=off; sqrtf is correctly rounded).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------------------------------ */
/* shared helpers                                                                                    */
/* ------------------------------------------------------------------------------------------------ */

static inline float minf_(float a, float b) { return b < a ? b : a; }

/* Initial map, reference dt/src/utils.cu:12.  Seeds get 0 (not v*0, which is NaN for v = inf). */
static void init_map(const uint8_t* mask, int mask_pitch, float* D, int W, int H, float v)
{
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
      D[(size_t)y * W + x] = mask[(size_t)y * mask_pitch + x] ? 0.0f : v;
}

/* ------------------------------------------------------------------------------------------------ */
/* ref-mode: C8, lambda blend, gray                                                                  */
/* ------------------------------------------------------------------------------------------------ */

static inline float ref_relax(float dq, float eucl_term_d, float l_eucl, float l_grad, int absdi, int use_fma)
{
  /* reference dt/src/dt_block_passes.cuh:46: D[..] + l_eucl * local_dist2d[dy + 1] + l_grad * l_dist */
  if (use_fma)
    return fmaf(l_grad, (float)absdi, fmaf(l_eucl, eucl_term_d, dq));
  float t = dq + l_eucl * eucl_term_d;
  return t + l_grad * (float)absdi;
}

static inline int absdiff_u8(uint8_t a, uint8_t b) { return a < b ? b - a : a - b; }

/* One directional raster pass over rows (Forward: x increasing) with the three predecessors at column
 * x - inc, rows y-1..y+1; reference generalised_distance_transform.cu:17-57. */
static int ref_pass_rows(const uint8_t* img, int ip, float* D, int W, int H, int forward, float l_eucl, float l_grad,
                         const float ld[3], int use_fma)
{
  int changed = 0;
  const int inc = forward ? 1 : -1, dx = -inc;
  const int x0 = forward ? 1 : W - 2, x1 = forward ? W : -1;
  for (int y = 0; y < H; ++y)
    for (int x = x0; x != x1; x += inc)
    {
      float best = D[(size_t)y * W + x];
      for (int dy = -1; dy <= 1; ++dy)
      {
        const int ny = y + dy;
        if (ny < 0 || ny >= H) continue;
        const int a = absdiff_u8(img[(size_t)y * ip + x], img[(size_t)ny * ip + x + dx]);
        best = minf_(best, ref_relax(D[(size_t)ny * W + x + dx], ld[dy + 1], l_eucl, l_grad, a, use_fma));
      }
      if (best < D[(size_t)y * W + x]) { D[(size_t)y * W + x] = best; changed = 1; }
    }
  return changed;
}

/* Column pass, reference generalised_distance_transform.cu:60-99. */
static int ref_pass_cols(const uint8_t* img, int ip, float* D, int W, int H, int forward, float l_eucl, float l_grad,
                         const float ld[3], int use_fma)
{
  int changed = 0;
  const int inc = forward ? 1 : -1, dy = -inc;
  const int y0 = forward ? 1 : H - 2, y1 = forward ? H : -1;
  for (int y = y0; y != y1; y += inc)
    for (int x = 0; x < W; ++x)
    {
      float best = D[(size_t)y * W + x];
      for (int dx = -1; dx <= 1; ++dx)
      {
        const int nx = x + dx;
        if (nx < 0 || nx >= W) continue;
        const int a = absdiff_u8(img[(size_t)y * ip + x], img[(size_t)(y + dy) * ip + nx]);
        best = minf_(best, ref_relax(D[(size_t)(y + dy) * W + nx], ld[dx + 1], l_eucl, l_grad, a, use_fma));
      }
      if (best < D[(size_t)y * W + x]) { D[(size_t)y * W + x] = best; changed = 1; }
    }
  return changed;
}

/* Returns the number of raster rounds run (>= 1), or -1 if max_rounds was reached first.
 * D is dense (pitch W floats). */
ORACLE_EXPORT int oracle_ggdt_ref(const uint8_t* img, int img_pitch, const uint8_t* mask, int mask_pitch, float* D,
                                  int W, int H, float lambda, float v, int use_fma, int max_rounds)
{
  if (W <= 0 || H <= 0) return 0;
  const float l_grad = lambda, l_eucl = 1.0f - lambda;
  const float ld[3] = {sqrtf(2.0f), 1.0f, sqrtf(2.0f)};
  init_map(mask, mask_pitch, D, W, H, v);
  for (int round = 1; round <= max_rounds; ++round)
  {
    int ch = 0;
    ch |= ref_pass_rows(img, img_pitch, D, W, H, 1, l_eucl, l_grad, ld, use_fma);
    ch |= ref_pass_rows(img, img_pitch, D, W, H, 0, l_eucl, l_grad, ld, use_fma);
    ch |= ref_pass_cols(img, img_pitch, D, W, H, 1, l_eucl, l_grad, ld, use_fma);
    ch |= ref_pass_cols(img, img_pitch, D, W, H, 0, l_eucl, l_grad, ld, use_fma);
    if (!ch) return round;
  }
  return -1;
}

/* ------------------------------------------------------------------------------------------------ */
/* ns-mode: C4, w = sqrt(1 + g2 * dI2), gray (channels = 1) or interleaved rgb8 (channels = 3)         */
/* ------------------------------------------------------------------------------------------------ */

static inline int dI2_at(const uint8_t* a, const uint8_t* b, int channels)
{
  int s = 0;
  for (int c = 0; c < channels; ++c)
  {
    const int d = (int)a[c] - (int)b[c];
    s += d * d;
  }
  return s;
}

static inline float ns_weight(float g2, int dI2)
{
  /* (float)dI2 is exact (dI2 <= 3 * 255^2 < 2^24); each operation is rounded to fp32. */
  const float t = g2 * (float)dI2;
  const float u = 1.0f + t;
  return sqrtf(u);
}

/* Forward + backward pass along one row (x), weights computed on the fly into wbuf (W-1 entries). */
static int ns_row(const uint8_t* row, int channels, float* d, int W, float g2, float* wbuf)
{
  for (int x = 1; x < W; ++x)
    wbuf[x - 1] = ns_weight(g2, dI2_at(row + (size_t)(x - 1) * channels, row + (size_t)x * channels, channels));
  int ch = 0;
  for (int x = 1; x < W; ++x)
  {
    const float t = d[x - 1] + wbuf[x - 1];
    if (t < d[x]) { d[x] = t; ch = 1; }
  }
  for (int x = W - 2; x >= 0; --x)
  {
    const float t = d[x + 1] + wbuf[x];
    if (t < d[x]) { d[x] = t; ch = 1; }
  }
  return ch;
}

/* Forward then backward pass along columns for the column strip [xa, xb). */
static int ns_cols(const uint8_t* img, int ip, int channels, float* D, int W, int H, int xa, int xb, float g2)
{
  int ch = 0;
  for (int y = 1; y < H; ++y)
  {
    const uint8_t* r0 = img + (size_t)(y - 1) * ip;
    const uint8_t* r1 = img + (size_t)y * ip;
    float* d0 = D + (size_t)(y - 1) * W;
    float* d1 = D + (size_t)y * W;
    for (int x = xa; x < xb; ++x)
    {
      const float w = ns_weight(g2, dI2_at(r0 + (size_t)x * channels, r1 + (size_t)x * channels, channels));
      const float t = d0[x] + w;
      if (t < d1[x]) { d1[x] = t; ch = 1; }
    }
  }
  for (int y = H - 2; y >= 0; --y)
  {
    const uint8_t* r0 = img + (size_t)y * ip;
    const uint8_t* r1 = img + (size_t)(y + 1) * ip;
    float* d0 = D + (size_t)y * W;
    float* d1 = D + (size_t)(y + 1) * W;
    for (int x = xa; x < xb; ++x)
    {
      const float w = ns_weight(g2, dI2_at(r0 + (size_t)x * channels, r1 + (size_t)x * channels, channels));
      const float t = d1[x] + w;
      if (t < d0[x]) { d0[x] = t; ch = 1; }
    }
  }
  return ch;
}

/* Raster fixpoint starting from the map already in D (dense, pitch W).  nthreads <= 0 uses all threads.
 * Rows are independent in the row passes and columns in the column passes (C4), so the parallel form
 * has no data race and the result is the same fixpoint for any thread count. */
static int ns_fixpoint(const uint8_t* img, int ip, int channels, float* D, int W, int H, float g2, int nthreads,
                       int max_rounds)
{
#ifdef _OPENMP
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  const int nt = 1;
  (void)nthreads;
#endif
  float* wbuf_all = (float*)malloc(sizeof(float) * (size_t)(W > 1 ? W : 2) * nt);
  int rounds = -1;
  for (int round = 1; round <= max_rounds; ++round)
  {
    int ch = 0;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(static) reduction(| : ch)
#endif
    for (int y = 0; y < H; ++y)
    {
#ifdef _OPENMP
      float* wbuf = wbuf_all + (size_t)omp_get_thread_num() * (W > 1 ? W : 2);
#else
      float* wbuf = wbuf_all;
#endif
      ch |= ns_row(img + (size_t)y * ip, channels, D + (size_t)y * W, W, g2, wbuf);
    }
    const int strip = 64;
    const int nstrips = (W + strip - 1) / strip;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1) reduction(| : ch)
#endif
    for (int s = 0; s < nstrips; ++s)
    {
      const int xa = s * strip, xb = xa + strip < W ? xa + strip : W;
      ch |= ns_cols(img, ip, channels, D, W, H, xa, xb, g2);
    }
    if (!ch) { rounds = round; break; }
  }
  free(wbuf_all);
  return rounds;
}

ORACLE_EXPORT int oracle_ggdt_ns(const uint8_t* img, int img_pitch, int channels, const uint8_t* mask, int mask_pitch,
                                 float* D, int W, int H, float g2, float v, int nthreads, int max_rounds)
{
  if (W <= 0 || H <= 0) return 0;
  init_map(mask, mask_pitch, D, W, H, v);
  return ns_fixpoint(img, img_pitch, channels, D, W, H, g2, nthreads, max_rounds);
}

/* Warm start: D holds a previous fixpoint; pixels where new_seeds != 0 are set to 0 and the map relaxes
 * again.  Because relaxation only lowers values, the result equals a cold run with the union of seeds. */
ORACLE_EXPORT int oracle_ggdt_ns_warm(const uint8_t* img, int img_pitch, int channels, const uint8_t* new_seeds,
                                      int seeds_pitch, float* D, int W, int H, float g2, int nthreads, int max_rounds)
{
  if (W <= 0 || H <= 0) return 0;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
      if (new_seeds[(size_t)y * seeds_pitch + x]) D[(size_t)y * W + x] = 0.0f;
  return ns_fixpoint(img, img_pitch, channels, D, W, H, g2, nthreads, max_rounds);
}

/* Plain sequential Gauss-Seidel form (one thread, rows then columns, no strips): a second schedule of the
 * same fixpoint, used by the tests to show schedule independence of the oracle itself. */
ORACLE_EXPORT int oracle_ggdt_ns_serial(const uint8_t* img, int img_pitch, int channels, const uint8_t* mask,
                                        int mask_pitch, float* D, int W, int H, float g2, float v, int max_rounds)
{
  if (W <= 0 || H <= 0) return 0;
  init_map(mask, mask_pitch, D, W, H, v);
  float* wbuf = (float*)malloc(sizeof(float) * (size_t)(W > 1 ? W : 2));
  int rounds = -1;
  for (int round = 1; round <= max_rounds; ++round)
  {
    int ch = 0;
    /* columns first this time, then rows */
    ch |= ns_cols(img, img_pitch, channels, D, W, H, 0, W, g2);
    for (int y = 0; y < H; ++y) ch |= ns_row(img + (size_t)y * img_pitch, channels, D + (size_t)y * W, W, g2, wbuf);
    if (!ch) { rounds = round; break; }
  }
  free(wbuf);
  return rounds;
}

/* ------------------------------------------------------------------------------------------------ */
/* FP64 Dijkstra on the ns-mode graph (binary heap, lazy deletion)                                    */
/* ------------------------------------------------------------------------------------------------ */

typedef struct { double d; int64_t i; } heap_item;

static void heap_push(heap_item* h, int64_t* n, heap_item it)
{
  int64_t k = (*n)++;
  while (k > 0)
  {
    int64_t p = (k - 1) >> 1;
    if (h[p].d <= it.d) break;
    h[k] = h[p];
    k = p;
  }
  h[k] = it;
}

static heap_item heap_pop(heap_item* h, int64_t* n)
{
  heap_item top = h[0];
  heap_item last = h[--(*n)];
  int64_t k = 0;
  for (;;)
  {
    int64_t c = 2 * k + 1;
    if (c >= *n) break;
    if (c + 1 < *n && h[c + 1].d < h[c].d) ++c;
    if (h[c].d >= last.d) break;
    h[k] = h[c];
    k = c;
  }
  if (*n > 0) h[k] = last;
  return top;
}

/* Exact-sum (FP64) geodesic distance with weights sqrt(1 + g2 * dI2) evaluated in double.
 * Unreached pixels get v.  Returns 0, or -1 on allocation failure. */
ORACLE_EXPORT int oracle_dijkstra_ns_f64(const uint8_t* img, int img_pitch, int channels, const uint8_t* mask,
                                         int mask_pitch, double* D, int W, int H, double g2, double v)
{
  const int64_t N = (int64_t)W * H;
  if (N <= 0) return 0;
  /* every pixel enters the heap at most 4 times + seeds */
  int64_t cap = 5 * N + 16;
  heap_item* h = (heap_item*)malloc(sizeof(heap_item) * (size_t)cap);
  uint8_t* done = (uint8_t*)calloc((size_t)N, 1);
  if (!h || !done) { free(h); free(done); return -1; }
  int64_t n = 0;
  for (int64_t i = 0; i < N; ++i) D[i] = INFINITY;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x)
      if (mask[(size_t)y * mask_pitch + x])
      {
        D[(int64_t)y * W + x] = 0.0;
        heap_item it = {0.0, (int64_t)y * W + x};
        heap_push(h, &n, it);
      }
  static const int ox[4] = {-1, 0, 1, 0}, oy[4] = {0, -1, 0, 1};
  while (n > 0)
  {
    heap_item it = heap_pop(h, &n);
    if (done[it.i]) continue;
    done[it.i] = 1;
    const int x = (int)(it.i % W), y = (int)(it.i / W);
    const uint8_t* pp = img + (size_t)y * img_pitch + (size_t)x * channels;
    for (int k = 0; k < 4; ++k)
    {
      const int nx = x + ox[k], ny = y + oy[k];
      if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
      const int64_t j = (int64_t)ny * W + nx;
      if (done[j]) continue;
      const uint8_t* qp = img + (size_t)ny * img_pitch + (size_t)nx * channels;
      const double nd = it.d + sqrt(1.0 + g2 * (double)dI2_at(pp, qp, channels));
      if (nd < D[j])
      {
        D[j] = nd;
        if (n >= cap) { free(h); free(done); return -1; }
        heap_item ni = {nd, j};
        heap_push(h, &n, ni);
      }
    }
  }
  for (int64_t i = 0; i < N; ++i)
    if (D[i] > v) D[i] = v;
  free(h);
  free(done);
  return 0;
}

ORACLE_EXPORT int oracle_max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
