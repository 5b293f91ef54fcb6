"""The C++ namespace dt layer (include/dt/*.hpp, the reference's API over the C ABI).

CPU: the check program tests/cpp/dt_api_check.cpp compiles and links against libdtb with the headers, and the
host-only pieces (CPU image2d, fill, imprint) behave.  GPU: the program runs every overload on seeded cases and
its maps equal the reference's golden tensors (ref-mode) and the oracle (C4 geodesic), bit for bit.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from distance_transform_benchmarks_b200 import _native, workloads as wl
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.dirname(_native.LIBDTB_PATH)
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "ref_goldens.npz"))


def _cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    pytest.skip("no g++")


def _compile(src, out):
    if not os.path.exists(_native.LIBDTB_PATH):
        pytest.skip("libdtb.so not built")
    cmd = [_cxx(), "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"), src,
           "-L" + PKG, "-ldtb", "-Wl,-rpath," + PKG, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def test_cpp_layer_compiles_and_links(tmp_path):
    _compile(os.path.join(ROOT, "tests", "cpp", "dt_api_check.cpp"), str(tmp_path / "dt_api_check"))


def test_cpp_host_pieces(tmp_path):
    """CPU-only parts of the layer: image2d CPU allocation, fill, imprint, neighbourhoods, errors (no GPU call)."""
    src = tmp_path / "host_pieces.cpp"
    src.write_text(r'''
#include <dt/c4.hpp>
#include <dt/c8.hpp>
#include <dt/fill.hpp>
#include <dt/image2d.hpp>
#include <dt/imprint.hpp>
#include <dt/random_image2d.hpp>
#include <sstream>
#include <cstdio>
int main() {
  dt::image2d<std::uint8_t> a(3, 2);
  dt::fill(a, std::uint8_t(7));
  a(2, 1) = 200;
  std::ostringstream os;
  dt::imprint(a, os);
  if (os.str() != "[  7   7   7]\n[  7   7 200]\n") { std::printf("imprint u8: %s", os.str().c_str()); return 1; }
  dt::image2d<float> f(2, 1);
  f(0, 0) = 1.5f; f(1, 0) = 0.25f;
  std::ostringstream fs;
  dt::imprint(f, fs);
  if (fs.str() != "[1.50000 0.25000]\n") { std::printf("imprint f32: %s", fs.str().c_str()); return 1; }
  auto r = dt::random_image2d<std::uint8_t>(16, 16);
  if (r.width() != 16 || r.pitch() != 16) return 1;
  int n = 0;
  for (auto p : dt::c4(dt::point2d{1, 1})) n += p.x() + p.y();
  if (n != 8) return 1;
  try { dt::image2d<float> bad(-1, 3); return 1; } catch (const dt::error& e) { if (e.status() != DTB_ERR_INVALID_ARG) return 1; }
  std::printf("ok\n");
  return 0;
}
''')
    exe = _compile(str(src), str(tmp_path / "host_pieces"))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def _write_case(d, lines, name, kind, img, mask, param, v=1e10):
    h, w = mask.shape
    ch = 3 if img.ndim == 3 else 1
    img.astype(np.uint8).tofile(os.path.join(d, name + ".img"))
    mask.astype(np.uint8).tofile(os.path.join(d, name + ".mask"))
    lines.append("%s %s %d %d %d %r %r" % (name, kind, w, h, ch, float(param), float(v)))


@pytest.mark.gpu
def test_cpp_layer_on_gpu(tmp_path):
    exe = _compile(os.path.join(ROOT, "tests", "cpp", "dt_api_check.cpp"), str(tmp_path / "dt_api_check"))
    d = str(tmp_path)
    lines, expect = [], {}
    for name in ("euclid", "geodesic"):
        _write_case(d, lines, name, "ref", GOLD[name + "_img"], GOLD[name + "_mask"], float(GOLD[name + "_lambda"]))
        expect[name] = GOLD[name + "_ref"]
    rng = np.random.default_rng(11)
    img = rng.integers(0, 256, size=(230, 250), dtype=np.uint8)
    mask = np.zeros_like(img)
    mask[115, 125] = 1
    _write_case(d, lines, "random_ref", "ref", img, mask, 0.3)
    expect["random_ref"] = orc.ggdt_ref(img, mask, 0.3, fma=True)
    # no seeds: every tile runs in exactly the first blocks round (the reference's first round visits them all)
    _write_case(d, lines, "noseed_ref", "ref", img[:100, :140], np.zeros((100, 140), np.uint8), 0.5)
    expect["noseed_ref"] = orc.ggdt_ref(img[:100, :140], np.zeros((100, 140), np.uint8), 0.5, fma=True)
    g, m, gamma = wl.config0()
    _write_case(d, lines, "blobs_c4", "c4", g, m, gamma)
    expect["blobs_c4"] = orc.ggdt_ns(g, m, gamma)
    rgb = wl.voronoi_rgb(4, 161, 97)
    m2 = wl.random_disks(np.random.default_rng(2), 161, 97, 4, 2, 5)
    _write_case(d, lines, "voronoi_c4", "c4", rgb, m2, 0.02)
    expect["voronoi_c4"] = orc.ggdt_ns(rgb, m2, 0.02)
    with open(os.path.join(d, "cases.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    r = subprocess.run([exe, d], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    for name, ref in expect.items():
        out = np.fromfile(os.path.join(d, name + ".out"), dtype=np.float32).reshape(ref.shape)
        assert np.array_equal(out.view(np.uint32), ref.astype(np.float32).view(np.uint32)), name
