// dt_api_check.cpp -- exercises the C++ namespace dt layer (include/dt/*.hpp) over libdtb on a GPU.
//
//   dt_api_check <dir>
//
// <dir>/cases.txt holds one case per line: `name kind width height channels param v`, kind `ref` (reference
// weight, param = lambda, channels 1) or `c4` (geodesic weight, param = gamma, channels 1 or 3).  Inputs are
// <dir>/name.img (height * width * channels bytes) and <dir>/name.mask (height * width bytes); the map is
// written to <dir>/name.out (height * width float32).  The program checks, bit for bit, that every overload of
// a case returns the same map (allocating / in place, device / host views, the raster, blocks and task
// variants, single calls / one batch), that round counters and error paths behave, and exits non-zero on the
// first mismatch.  The caller compares name.out with the oracle.
#include <dt/c4.hpp>
#include <dt/c8.hpp>
#include <dt/fill.hpp>
#include <dt/generalised_distance_transform.hpp>
#include <dt/image2d.hpp>
#include <dt/imprint.hpp>
#include <dt/rgb.hpp>
#include <dt/transfert.hpp>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace
{
  int g_failures = 0;

#define CHECK(cond, ...)                                   \
  do                                                       \
  {                                                        \
    if (!(cond))                                           \
    {                                                      \
      std::fprintf(stderr, "FAIL %s:%d: ", __FILE__, __LINE__); \
      std::fprintf(stderr, __VA_ARGS__);                   \
      std::fprintf(stderr, "\n");                          \
      ++g_failures;                                        \
    }                                                      \
  } while (0)

  std::vector<std::uint8_t> read_file(const std::string& path, size_t bytes)
  {
    std::vector<std::uint8_t> v(bytes);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(bytes));
    if (!f)
      throw std::runtime_error("cannot read " + path);
    return v;
  }

  template <typename T>
  dt::image2d<T> cpu_image(const std::vector<std::uint8_t>& raw, int w, int h)
  {
    dt::image2d<T> img(w, h, dt::e_memory_kind::CPU);
    for (int y = 0; y < h; ++y)
      std::memcpy(&img(0, y), raw.data() + static_cast<size_t>(y) * w * sizeof(T), static_cast<size_t>(w) * sizeof(T));
    return img;
  }

  // Bitwise equality of two float maps (any memory kind).
  bool same(const dt::image2d_view<float>& a, const dt::image2d_view<float>& b)
  {
    const auto ha = a.memory_kind() == dt::e_memory_kind::GPU ? dt::device_to_host(a) : dt::image2d<float>();
    const auto hb = b.memory_kind() == dt::e_memory_kind::GPU ? dt::device_to_host(b) : dt::image2d<float>();
    const dt::image2d_view<float>& A = a.memory_kind() == dt::e_memory_kind::GPU ? ha : a;
    const dt::image2d_view<float>& B = b.memory_kind() == dt::e_memory_kind::GPU ? hb : b;
    if (A.width() != B.width() || A.height() != B.height())
      return false;
    for (int y = 0; y < A.height(); ++y)
      if (std::memcmp(&A(0, y), &B(0, y), static_cast<size_t>(A.width()) * sizeof(float)) != 0)
        return false;
    return true;
  }

  void write_map(const std::string& path, const dt::image2d_view<float>& m)
  {
    const auto h = m.memory_kind() == dt::e_memory_kind::GPU ? dt::device_to_host(m) : dt::image2d<float>();
    const dt::image2d_view<float>& H = m.memory_kind() == dt::e_memory_kind::GPU ? h : m;
    std::ofstream f(path, std::ios::binary);
    for (int y = 0; y < H.height(); ++y)
      f.write(reinterpret_cast<const char*>(&H(0, y)), static_cast<std::streamsize>(H.width() * sizeof(float)));
  }

  struct Case
  {
    std::string name, kind;
    int         w = 0, h = 0, ch = 1;
    float       param = 0, v = 1e10f;
  };

  void run_ref(const std::string& dir, const Case& c)
  {
    const auto img  = cpu_image<std::uint8_t>(read_file(dir + "/" + c.name + ".img", size_t(c.w) * c.h), c.w, c.h);
    const auto mask = cpu_image<std::uint8_t>(read_file(dir + "/" + c.name + ".mask", size_t(c.w) * c.h), c.w, c.h);
    auto d_img  = dt::host_to_device(img);
    auto d_mask = dt::host_to_device(mask);

    const auto d1 = dt::generalised_distance_transform(d_img, d_mask, c.param, c.v);
    const int  tiles = ((c.w + 31) / 32) * ((c.h + 31) / 32);
    std::vector<int> rounds(tiles, 0);
    const auto d2 = dt::generalised_distance_transform_blocks(d_img, d_mask, c.param, c.v, rounds.data());
    const auto d3 = dt::generalised_distance_transform_task(d_img, d_mask, c.param, c.v);
    dt::image2d<float> d4(c.w, c.h, dt::e_memory_kind::GPU);
    dt::generalised_distance_transform(d_img, d_mask, d4, c.param, c.v);
    const auto h5 = dt::generalised_distance_transform(img, mask, c.param, c.v);  // host views
    CHECK(h5.memory_kind() == dt::e_memory_kind::CPU, "%s: host call returned a device image", c.name.c_str());
    CHECK(same(d1, d2), "%s: raster != blocks", c.name.c_str());
    CHECK(same(d1, d3), "%s: raster != task", c.name.c_str());
    CHECK(same(d1, d4), "%s: allocating != in place", c.name.c_str());
    CHECK(same(d1, h5), "%s: device views != host views", c.name.c_str());

    // Round counters: host and device memory give the same counts; every tile of an image with a seed is visited.
    dtb_image dcounts{};
    dt::details::check(dtb_image_alloc(tiles, 1, 4, DTB_GPU, &dcounts), "dtb_image_alloc");
    std::vector<int> zeros(tiles, 0), rounds_dev(tiles, 0);
    dtb_image hz{zeros.data(), tiles, 1, tiles * 4, 4, DTB_CPU};
    dt::details::check(dtb_host_to_device(&hz, &dcounts, nullptr), "host_to_device");
    dt::image2d<float> d6(c.w, c.h, dt::e_memory_kind::GPU);
    dt::generalised_distance_transform_blocks(d_img, d_mask, d6, c.param, c.v, static_cast<int*>(dcounts.buffer));
    dtb_image hr{rounds_dev.data(), tiles, 1, tiles * 4, 4, DTB_CPU};
    dt::details::check(dtb_device_to_host(&dcounts, &hr, nullptr), "device_to_host");
    dtb_image_free(&dcounts);
    CHECK(same(d1, d6), "%s: blocks with device counters differs", c.name.c_str());
    CHECK(rounds == rounds_dev, "%s: host and device round counters differ", c.name.c_str());
    bool any_seed = false;
    for (int y = 0; y < c.h && !any_seed; ++y)
      for (int x = 0; x < c.w; ++x)
        if (mask(x, y))
        {
          any_seed = true;
          break;
        }
    // As in the reference's blocks variant, the first round visits every tile; without seeds nothing changes, so
    // every tile runs in exactly that one round.
    for (int t = 0; t < tiles; ++t) {
      CHECK(rounds[t] >= 1, "%s: tile %d never visited", c.name.c_str(), t);
      if (!any_seed) CHECK(rounds[t] == 1, "%s: tile %d counted %d rounds without seeds", c.name.c_str(), t, rounds[t]);
    }
    write_map(dir + "/" + c.name + ".out", d1);
  }

  template <typename P>
  dt::image2d<float> run_c4_typed(const std::string& dir, const Case& c, dt::image2d<P>& d_img_out,
                                  dt::image2d<std::uint8_t>& d_mask_out)
  {
    const auto img  = cpu_image<P>(read_file(dir + "/" + c.name + ".img", size_t(c.w) * c.h * sizeof(P)), c.w, c.h);
    const auto mask = cpu_image<std::uint8_t>(read_file(dir + "/" + c.name + ".mask", size_t(c.w) * c.h), c.w, c.h);
    d_img_out  = dt::host_to_device(img);
    d_mask_out = dt::host_to_device(mask);
    auto d1 = dt::generalised_distance_transform(d_img_out, d_mask_out, dt::c4, c.param, c.v);
    const auto h2 = dt::generalised_distance_transform(img, mask, dt::c4, c.param, c.v);
    dt::image2d<float> d3(c.w, c.h, dt::e_memory_kind::GPU);
    dt::generalised_distance_transform(d_img_out, d_mask_out, d3, dt::c4, c.param, c.v);
    CHECK(same(d1, h2), "%s: device views != host views", c.name.c_str());
    CHECK(same(d1, d3), "%s: allocating != in place", c.name.c_str());
    write_map(dir + "/" + c.name + ".out", d1);
    return d1;
  }

  void check_view_semantics()
  {
    dt::image2d<std::uint8_t> a(7, 5);
    dt::fill(a, std::uint8_t(9));
    dt::image2d<std::uint8_t> b = a;  // shared ownership: same pixels
    b(3, 2) = 1;
    CHECK(a(3, 2) == 1 && a.buffer() == b.buffer(), "image2d copies must alias");
    dt::image2d_view<std::uint8_t> v(a);
    dt::image2d_view<std::uint8_t> w(std::move(v));
    CHECK(!v.valid() && w.valid() && w(3, 2) == 1, "moved-from view must lose its buffer");
    CHECK(a.pitch() == 7 && a.elem_size() == 1, "CPU rows are packed");
    dt::image2d<dt::rgb8> g(33, 3, dt::e_memory_kind::GPU);
    CHECK(g.elem_size() == 3 && g.pitch() % 128 == 0 && g.pitch() >= 99, "GPU rows are pitched to 128 bytes");
    CHECK(dt::c4(dt::point2d{5, 5}).size() == 4 && dt::c8(dt::point2d{0, 0}).size() == 8, "neighbourhood sizes");
    CHECK(*dt::c8(dt::point2d{0, 0}).begin() == dt::point2d(-1, 0), "c8 starts on the left neighbour");
  }

  void check_errors()
  {
    dt::image2d<std::uint8_t> img(40, 30, dt::e_memory_kind::GPU), mask(41, 30, dt::e_memory_kind::GPU);
    bool thrown = false;
    try
    {
      (void)dt::generalised_distance_transform(img, mask, 0.5f);
    }
    catch (const dt::error& e)
    {
      thrown = e.status() == DTB_ERR_INVALID_ARG;
    }
    CHECK(thrown, "shape mismatch must throw dt::error(DTB_ERR_INVALID_ARG)");
    dt::image2d<std::uint8_t> mask2(40, 30, dt::e_memory_kind::GPU);
    thrown = false;
    try
    {
      (void)dt::generalised_distance_transform(img, mask2, 1.5f);
    }
    catch (const std::runtime_error&)
    {
      thrown = true;
    }
    CHECK(thrown, "lambda outside [0, 1] must throw a std::runtime_error");
  }
} // namespace

int main(int argc, char** argv)
{
  if (argc != 2)
  {
    std::fprintf(stderr, "usage: %s <dir>\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  std::ifstream     f(dir + "/cases.txt");
  std::vector<Case> cases;
  for (std::string line; std::getline(f, line);)
  {
    if (line.empty())
      continue;
    std::istringstream is(line);
    Case c;
    is >> c.name >> c.kind >> c.w >> c.h >> c.ch >> c.param >> c.v;
    cases.push_back(c);
  }

  try
  {
    check_view_semantics();
    check_errors();
    // Single calls, and every C4 case again in one ragged batch.
    std::vector<dt::image2d<std::uint8_t>> gray_imgs, masks;
    std::vector<dt::image2d<dt::rgb8>>     rgb_imgs;
    std::vector<dt::image2d<float>>        singles;
    std::vector<dt::image2d_view<void>>    b_img, b_mask, b_dist;
    std::vector<float>                     b_gamma;
    std::vector<dt::image2d<float>>        batch_out;
    for (const Case& c : cases)
    {
      if (c.kind == "ref")
      {
        run_ref(dir, c);
        continue;
      }
      dt::image2d<std::uint8_t> dm;
      dt::image2d<float>        out;
      if (c.ch == 3)
      {
        dt::image2d<dt::rgb8> di;
        out = run_c4_typed<dt::rgb8>(dir, c, di, dm);
        rgb_imgs.push_back(di);
        b_img.push_back(di);
      }
      else
      {
        dt::image2d<std::uint8_t> di;
        out = run_c4_typed<std::uint8_t>(dir, c, di, dm);
        gray_imgs.push_back(di);
        b_img.push_back(di);
      }
      masks.push_back(dm);
      b_mask.push_back(dm);
      singles.push_back(out);
      batch_out.emplace_back(c.w, c.h, dt::e_memory_kind::GPU);
      b_dist.push_back(batch_out.back());
      b_gamma.push_back(c.param);
    }
    if (!b_img.empty())
    {
      // The batch takes one v; use the first C4 case's.
      float v = 1e10f;
      for (const Case& c : cases)
        if (c.kind == "c4")
        {
          v = c.v;
          break;
        }
      dt::generalised_distance_transform_batch(b_img, b_mask, b_dist, b_gamma, dt::c4, v);
      size_t k = 0;
      for (const Case& c : cases)
      {
        if (c.kind != "c4")
          continue;
        if (c.v == v)
          CHECK(same(singles[k], batch_out[k]), "%s: batch != single call", c.name.c_str());
        ++k;
      }
    }
  }
  catch (const std::exception& e)
  {
    std::fprintf(stderr, "FAIL: exception: %s\n", e.what());
    return 1;
  }
  if (g_failures)
  {
    std::fprintf(stderr, "%d check(s) failed\n", g_failures);
    return 1;
  }
  std::printf("ok %zu cases\n", cases.size());
  return 0;
}
