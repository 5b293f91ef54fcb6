// datagen.cpp -- seeded synthetic inputs for the GGDT workloads (host only, OpenMP).
//
// The reference benchmarks real photographs from /data/dt_images (benchmarks/distance_transform.cpp:17,
// :55-74), which are not available; these generators stand in with the shapes and value distributions
// of the configured workloads.  Every pixel depends only on (seed, generator parameters, x, y): the
// output is identical for any thread count.
//
// Random numbers: splitmix64 (Steele, Lea, Flood 2014) to derive streams, xoshiro256** (Blackman, Vigna
// 2018) for sequential draws, and the Box-Muller transform for normal deviates.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#define DTBG_API extern "C" __attribute__((visibility("default")))

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct Xoshiro {
  uint64_t s[4];
  explicit Xoshiro(uint64_t seed) {
    uint64_t z = seed;
    for (auto& w : s) { z = splitmix64(z); w = z; }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }      // [0, 1)
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  uint32_t below(uint32_t n) { return (uint32_t)(uniform() * n); }    // [0, n)
};

// Counter-based standard normal for pixel (index, stream): Box-Muller on two hashed uniforms.
inline double pixel_normal(uint64_t seed, uint64_t index) {
  const uint64_t a = splitmix64(seed ^ splitmix64(index * 2 + 1));
  const uint64_t b = splitmix64(a ^ 0xD1B54A32D192ED03ull);
  const double u1 = ((double)(a >> 11) + 1.0) * 0x1.0p-53;  // (0, 1]
  const double u2 = (double)(b >> 11) * 0x1.0p-53;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

inline uint64_t pixel_bits(uint64_t seed, uint64_t index) { return splitmix64(seed ^ splitmix64(index * 2 + 1)); }

inline uint8_t clip_round(double v) {
  v = std::nearbyint(v);
  return (uint8_t)(v < 0.0 ? 0.0 : v > 255.0 ? 255.0 : v);
}

}  // namespace

// Sum of `nblobs` isotropic Gaussian blobs (centre uniform in the image, sigma U[smin, smax], amplitude
// U[amin, amax]), clipped to [0, 255], plus N(0, noise_sigma^2) per pixel, clipped and rounded.
DTBG_API void dtbg_blobs_gray(uint64_t seed, int W, int H, int nblobs, double smin, double smax, double amin, double amax,
                              double noise_sigma, uint8_t* out, int64_t pitch) {
  Xoshiro rng(seed);
  std::vector<double> cx(nblobs), cy(nblobs), sg(nblobs), amp(nblobs);
  for (int k = 0; k < nblobs; ++k) {
    cx[k] = rng.uniform(0.0, W);
    cy[k] = rng.uniform(0.0, H);
    sg[k] = rng.uniform(smin, smax);
    amp[k] = rng.uniform(amin, amax);
  }
  // Separable: exp(-(dx^2 + dy^2) / 2s^2) = gx[x] * gy[y].
  std::vector<double> gx((size_t)nblobs * W), gy((size_t)nblobs * H);
  for (int k = 0; k < nblobs; ++k) {
    const double inv = 1.0 / (2.0 * sg[k] * sg[k]);
    for (int x = 0; x < W; ++x) gx[(size_t)k * W + x] = std::exp(-((x - cx[k]) * (x - cx[k])) * inv);
    for (int y = 0; y < H; ++y) gy[(size_t)k * H + y] = amp[k] * std::exp(-((y - cy[k]) * (y - cy[k])) * inv);
  }
  const uint64_t nseed = splitmix64(seed ^ 0x6E6F697365ull);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y) {
    uint8_t* row = out + (int64_t)y * pitch;
    for (int x = 0; x < W; ++x) {
      double f = 0.0;
      for (int k = 0; k < nblobs; ++k) f += gy[(size_t)k * H + y] * gx[(size_t)k * W + x];
      f = f > 255.0 ? 255.0 : f;
      f += noise_sigma * pixel_normal(nseed, (uint64_t)y * (uint64_t)W + (uint64_t)x);
      row[x] = clip_round(f);
    }
  }
}

// Voronoi mosaic: `nsites` sites uniform in [0, W) x [0, H), each with a uniform random RGB colour;
// every pixel takes the colour of its nearest site (squared Euclidean distance, ties to the lower index)
// plus N(0, noise_sigma^2) per channel, rounded and clipped.  Interleaved rgb8 output.
DTBG_API void dtbg_voronoi_rgb(uint64_t seed, int W, int H, int nsites, double noise_sigma, uint8_t* out, int64_t pitch) {
  Xoshiro rng(seed);
  std::vector<double> sx(nsites), sy(nsites);
  std::vector<uint8_t> col(3 * (size_t)nsites);
  for (int k = 0; k < nsites; ++k) {
    sx[k] = rng.uniform(0.0, W);
    sy[k] = rng.uniform(0.0, H);
    for (int c = 0; c < 3; ++c) col[3 * (size_t)k + c] = (uint8_t)rng.below(256);
  }
  // Uniform bucket grid over the sites.
  const double cs = std::max(4.0, std::sqrt((double)W * H / std::max(1, nsites)));
  const int gw = std::max(1, (int)std::ceil(W / cs)), gh = std::max(1, (int)std::ceil(H / cs));
  std::vector<std::vector<int>> cell((size_t)gw * gh);
  for (int k = 0; k < nsites; ++k) {
    const int gx = std::min(gw - 1, (int)(sx[k] / cs)), gy = std::min(gh - 1, (int)(sy[k] / cs));
    cell[(size_t)gy * gw + gx].push_back(k);
  }
  const uint64_t nseed = splitmix64(seed ^ 0x766F726F6E6F69ull);
#pragma omp parallel for schedule(dynamic, 16)
  for (int y = 0; y < H; ++y) {
    uint8_t* row = out + (int64_t)y * pitch;
    const int cy = std::min(gh - 1, (int)(y / cs));
    for (int x = 0; x < W; ++x) {
      const int cx = std::min(gw - 1, (int)(x / cs));
      double best = 1e300;
      int bk = 0;
      for (int r = 0;; ++r) {
        // cells at Chebyshev ring r around (cx, cy)
        for (int gy = cy - r; gy <= cy + r; ++gy) {
          if (gy < 0 || gy >= gh) continue;
          for (int gx = cx - r; gx <= cx + r; ++gx) {
            if (gx < 0 || gx >= gw) continue;
            if (std::max(std::abs(gx - cx), std::abs(gy - cy)) != r) continue;
            for (int k : cell[(size_t)gy * gw + gx]) {
              const double dx = x - sx[k], dy = y - sy[k], d = dx * dx + dy * dy;
              if (d < best || (d == best && k < bk)) { best = d; bk = k; }
            }
          }
        }
        // every site in ring r + 1 or beyond is at least r * cs away from the pixel
        const double lim = (double)r * cs;
        if ((best < 1e299 && best <= lim * lim) || (r > gw && r > gh)) break;
      }
      const uint64_t idx = ((uint64_t)y * (uint64_t)W + (uint64_t)x) * 3;
      for (int c = 0; c < 3; ++c) row[3 * x + c] = clip_round(col[3 * (size_t)bk + c] + noise_sigma * pixel_normal(nseed, idx + c));
    }
  }
}

// Perfect maze from a randomized depth-first search on a (W / cell) x (H / cell) grid, started at cell
// (0, 0).  Walls `wall` pixels thick between cells (wall / 2 on each side, and at the image border),
// corridor pixels 0 and wall pixels 255, plus uniform integer noise in [0, noise_max] clipped at 255.
// Writes the centre of the first dead-end cell in raster order (a corridor end) to *seed_x, *seed_y.
DTBG_API int dtbg_maze_gray(uint64_t seed, int W, int H, int cell, int wall, int noise_max, uint8_t* out, int64_t pitch,
                            int* seed_x, int* seed_y) {
  const int cw = W / cell, ch = H / cell;
  if (cw < 1 || ch < 1 || wall < 2 || wall >= cell) return -1;
  // open[c] bits: 1 right, 2 down, 4 left, 8 up
  std::vector<uint8_t> open((size_t)cw * ch, 0), seen((size_t)cw * ch, 0);
  Xoshiro rng(seed);
  std::vector<int> stack;
  stack.reserve((size_t)cw * ch);
  stack.push_back(0);
  seen[0] = 1;
  static const int dx[4] = {1, 0, -1, 0}, dy[4] = {0, 1, 0, -1};
  while (!stack.empty()) {
    const int c = stack.back();
    const int x = c % cw, y = c / cw;
    int cand[4], nc = 0;
    for (int k = 0; k < 4; ++k) {
      const int nx = x + dx[k], ny = y + dy[k];
      if (nx >= 0 && ny >= 0 && nx < cw && ny < ch && !seen[(size_t)ny * cw + nx]) cand[nc++] = k;
    }
    if (!nc) { stack.pop_back(); continue; }
    const int k = cand[rng.below((uint32_t)nc)];
    const int nx = x + dx[k], ny = y + dy[k], n = ny * cw + nx;
    open[c] |= (uint8_t)(1u << k);
    open[n] |= (uint8_t)(1u << ((k + 2) & 3));
    seen[n] = 1;
    stack.push_back(n);
  }
  const int hw = wall / 2;
  const uint64_t nseed = splitmix64(seed ^ 0x6D617A65ull);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y) {
    uint8_t* row = out + (int64_t)y * pitch;
    const int cy = std::min(ch - 1, y / cell), ly = y - cy * cell;
    for (int x = 0; x < W; ++x) {
      const int cx = std::min(cw - 1, x / cell), lx = x - cx * cell;
      const uint8_t o = open[(size_t)cy * cw + cx];
      const bool bl = lx < hw, br = lx >= cell - hw, bt = ly < hw, bb = ly >= cell - hw;
      bool is_wall;
      if (x >= cw * cell || y >= ch * cell) is_wall = true;   // leftover margin
      else if ((bl || br) && (bt || bb)) is_wall = true;      // pillars
      else if (bl) is_wall = !(o & 4);
      else if (br) is_wall = !(o & 1);
      else if (bt) is_wall = !(o & 8);
      else if (bb) is_wall = !(o & 2);
      else is_wall = false;
      const int noise = noise_max > 0 ? (int)(pixel_bits(nseed, (uint64_t)y * (uint64_t)W + (uint64_t)x) % (uint64_t)(noise_max + 1)) : 0;
      const int val = (is_wall ? 255 : 0) + noise;
      row[x] = (uint8_t)(val > 255 ? 255 : val);
    }
  }
  *seed_x = cell / 2;
  *seed_y = cell / 2;
  for (int c = 0; c < cw * ch; ++c) {
    const uint8_t o = open[c];
    if (o == 1 || o == 2 || o == 4 || o == 8) {
      *seed_x = (c % cw) * cell + cell / 2;
      *seed_y = (c / cw) * cell + cell / 2;
      break;
    }
  }
  return 0;
}

// Seed disks: mask = 1 where (x - cx)^2 + (y - cy)^2 <= r^2 for any disk (clipped to the image).
DTBG_API void dtbg_draw_disks(uint8_t* mask, int64_t pitch, int W, int H, int n, const int32_t* cx, const int32_t* cy,
                              const int32_t* r) {
  for (int k = 0; k < n; ++k) {
    const int rr = r[k];
    for (int y = std::max(0, cy[k] - rr); y <= std::min(H - 1, cy[k] + rr); ++y)
      for (int x = std::max(0, cx[k] - rr); x <= std::min(W - 1, cx[k] + rr); ++x) {
        const int ddx = x - cx[k], ddy = y - cy[k];
        if (ddx * ddx + ddy * ddy <= rr * rr) mask[(int64_t)y * pitch + x] = 1;
      }
  }
}
