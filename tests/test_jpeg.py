"""JPEG input (dtb_image_read / dtb.imread): the reference's dt::imread (dt/src/imread.cpp:10-31) decodes its
benchmark inputs with stb_image and keeps only 1-component files.

Gray files must match the reference decoder byte for byte: against the committed fixtures (tests/golden/jpeg/,
made by tests/golden/make_jpeg_golden.py with stb_image built from the reference's source) and, where that build
is present (oracle/_ref/libstb_ref.so), against it live on a seeded sweep of encoder modes.  Colour files (which
the reference rejects) must stay within 3 levels of stb_image's RGB output.
"""
import os
import subprocess

import numpy as np
import pytest

import distance_transform_benchmarks_b200 as dtb
from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN_DIR = os.path.join(HERE, "golden", "jpeg")
GOLDENS = np.load(os.path.join(HERE, "golden", "jpeg_goldens.npz"))
GRAY = sorted(k for k in GOLDENS.files if k.startswith("gray"))
RGB = sorted(k for k in GOLDENS.files if k.startswith("rgb"))
RGB_TOLERANCE = 3  # levels: chroma upsampling and YCbCr -> RGB rounding differ from stb_image's


@pytest.mark.parametrize("name", GRAY)
def test_gray_matches_reference_decoder(name):
    got = dtb.imread(os.path.join(GOLDEN_DIR, name + ".jpg"), 1)
    assert got.dtype == np.uint8 and got.shape == GOLDENS[name].shape
    assert np.array_equal(got, GOLDENS[name])


@pytest.mark.parametrize("name", RGB)
def test_rgb_within_tolerance_of_reference_decoder(name):
    got = dtb.imread(os.path.join(GOLDEN_DIR, name + ".jpg"), 3)
    want = GOLDENS[name]
    assert got.shape == want.shape
    assert int(np.abs(got.astype(np.int16) - want.astype(np.int16)).max()) <= RGB_TOLERANCE


def test_component_count_must_match():
    # dt::imread throws for files that are not 1-component (dt/src/imread.cpp:16-20); reading a gray file as rgb is
    # no conversion either
    with pytest.raises(dtb.DtbError):
        dtb.imread(os.path.join(GOLDEN_DIR, RGB[0] + ".jpg"), 1)
    with pytest.raises(dtb.DtbError):
        dtb.imread(os.path.join(GOLDEN_DIR, GRAY[0] + ".jpg"), 3)


def _patched(tmp_path, name, fn):
    data = bytearray(open(os.path.join(GOLDEN_DIR, name + ".jpg"), "rb").read())
    fn(data)
    p = tmp_path / "patched.jpg"
    p.write_bytes(bytes(data))
    return p


def test_unsupported_frames_rejected(tmp_path):
    name = "gray_base_q90"
    # arithmetic-coded frame (SOF9 in place of SOF0)
    def arith(d):
        d[d.index(b"\xff\xc0") + 1] = 0xC9
    # 12-bit samples (the frame header's precision byte)
    def twelve(d):
        d[d.index(b"\xff\xc0") + 4] = 12
    for fn in (arith, twelve):
        with pytest.raises(dtb.DtbError):
            dtb.imread(_patched(tmp_path, name, fn), 1)
    with pytest.raises(dtb.DtbError):  # the start-of-image marker alone
        dtb.imread(_patched(tmp_path, name, lambda d: d.__delitem__(slice(2, None))), 1)


def test_corrupt_and_truncated_files_do_not_crash(tmp_path):
    rng = np.random.default_rng(5)
    for it in range(150):
        name = (GRAY + RGB)[it % (len(GRAY) + len(RGB))]
        channels = 1 if name.startswith("gray") else 3

        def damage(d):
            if it % 2:
                del d[int(rng.integers(2, len(d))):]
            else:
                for _ in range(int(rng.integers(1, 6))):
                    d[int(rng.integers(2, len(d)))] = int(rng.integers(0, 256))
        try:
            got = dtb.imread(_patched(tmp_path, name, damage), channels)
        except dtb.DtbError:
            continue
        assert got.dtype == np.uint8 and got.ndim == (2 if channels == 1 else 3)


def _encoder_sweep():
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(11)
    for h, w in ((8, 8), (9, 17), (45, 67), (100, 33), (256, 130)):
        y, x = np.mgrid[0:h, 0:w]
        img = np.clip(128 + 100 * np.sin(x / 6.0) * np.cos(y / 9.0) + rng.normal(0, 18, (h, w)), 0, 255)
        img = img.astype(np.uint8)
        for q in (30, 85, 100):
            for prog in (0, 1):
                for rst in (0, 1, 4):
                    params = [cv2.IMWRITE_JPEG_QUALITY, q, cv2.IMWRITE_JPEG_PROGRESSIVE, prog,
                              cv2.IMWRITE_JPEG_RST_INTERVAL, rst, cv2.IMWRITE_JPEG_OPTIMIZE, (q + rst) % 2]
                    ok, buf = cv2.imencode(".jpg", img, params)
                    assert ok
                    yield (h, w, q, prog, rst), buf.tobytes()


@pytest.mark.skipif(not orc.stb_ref_available(), reason="stb_image of the reference not built (oracle/_ref)")
def test_gray_sweep_matches_reference_decoder_live(tmp_path):
    n = 0
    for case, data in _encoder_sweep():
        p = tmp_path / "sweep.jpg"
        p.write_bytes(data)
        want, comps = orc.stb_ref_load(p, 0)
        assert comps == 1
        assert np.array_equal(dtb.imread(p, 1), want[..., 0]), case
        n += 1
    assert n == 90


def test_cpp_imread_reads_jpeg(tmp_path):
    """dt::imread<std::uint8_t> (include/dt/imread.hpp) on the JPEG fixtures: the gray file's samples, and the
    reference's std::invalid_argument for a colour file (dt/src/imread.cpp:16-20)."""
    from tests.test_cpp_api import _compile
    src = tmp_path / "jpeg_read.cpp"
    src.write_text(r'''
#include <dt/imread.hpp>
#include <cstdio>
#include <stdexcept>
int main(int argc, char** argv) {
  if (argc != 4) return 2;
  auto img = dt::imread<std::uint8_t>(argv[1]);
  FILE* f = std::fopen(argv[2], "wb");
  for (int y = 0; y < img.height(); ++y) std::fwrite(&img(0, y), 1, img.width(), f);
  std::fclose(f);
  try { dt::imread<std::uint8_t>(argv[3]); return 3; } catch (const std::invalid_argument&) {}
  std::printf("%d %d\n", img.width(), img.height());
  return 0;
}
''')
    exe = _compile(str(src), str(tmp_path / "jpeg_read"))
    name = "gray_prog_q75"
    raw = tmp_path / "out.raw"
    r = subprocess.run([exe, os.path.join(GOLDEN_DIR, name + ".jpg"), str(raw), os.path.join(GOLDEN_DIR, RGB[0] + ".jpg")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    want = GOLDENS[name]
    assert r.stdout.split() == [str(want.shape[1]), str(want.shape[0])]
    assert np.array_equal(np.fromfile(raw, dtype=np.uint8).reshape(want.shape), want)
