"""Image files (dtb_image_read / dtb_image_write, dt::imread / dt::imsave): the PNG decoder against files that
an independent encoder (PIL) writes with every colour type and adaptive row filters, the encoder read back by
PIL, PGM / PPM round trips, and the error cases.  CPU only; the command line tool runs on the GPU."""
import os
import subprocess
import sys

import numpy as np
import pytest
from PIL import Image

import distance_transform_benchmarks_b200 as dtb
from distance_transform_benchmarks_b200._native import DtbError
from distance_transform_benchmarks_b200 import workloads as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _gray(h=37, w=53, seed=1):
    return wl.blobs_gray(seed, w, h)


def _rgb(h=29, w=41, seed=2):
    return wl.voronoi_rgb(seed, w, h, nsites=12)


@pytest.mark.parametrize("optimize", [False, True])
def test_png_decoder_against_pil_gray_and_rgb(tmp_path, optimize):
    g, c = _gray(), _rgb()
    Image.fromarray(g, "L").save(tmp_path / "g.png", optimize=optimize)
    Image.fromarray(c, "RGB").save(tmp_path / "c.png", optimize=optimize)
    assert np.array_equal(dtb.imread(tmp_path / "g.png", 1), g)
    assert np.array_equal(dtb.imread(tmp_path / "c.png", 3), c)


def test_png_decoder_palette_expands_to_rgb(tmp_path):
    c = _rgb()
    pal = Image.fromarray(c, "RGB").quantize(colors=16)
    pal.save(tmp_path / "p.png")
    expect = np.asarray(pal.convert("RGB"))
    assert np.array_equal(dtb.imread(tmp_path / "p.png", 3), expect)


def test_png_decoder_one_bit_gray(tmp_path):
    g = (_gray() > 128).astype(np.uint8) * 255
    Image.fromarray(g, "L").convert("1").save(tmp_path / "b.png")
    assert Image.open(tmp_path / "b.png").mode == "1"
    assert np.array_equal(dtb.imread(tmp_path / "b.png", 1), g)


def test_component_count_must_match(tmp_path):
    g, c = _gray(), _rgb()
    Image.fromarray(g, "L").save(tmp_path / "g.png")
    Image.fromarray(np.dstack([c, c[..., :1]]), "RGBA").save(tmp_path / "a.png")
    with pytest.raises(DtbError):
        dtb.imread(tmp_path / "g.png", 3)
    with pytest.raises(DtbError):
        dtb.imread(tmp_path / "a.png", 3)
    with pytest.raises(DtbError) as e:
        dtb.imread(tmp_path / "missing.png", 1)
    assert e.value.status == 8  # DTB_ERR_IO


def test_png_encoder_read_by_pil(tmp_path):
    g, c = _gray(), _rgb()
    dtb.imsave(tmp_path / "g.png", g)
    dtb.imsave(tmp_path / "c.png", c)
    assert np.array_equal(np.asarray(Image.open(tmp_path / "g.png")), g)
    assert np.array_equal(np.asarray(Image.open(tmp_path / "c.png").convert("RGB")), c)


def test_pnm_round_trip_and_pil(tmp_path):
    g, c = _gray(), _rgb()
    dtb.imsave(tmp_path / "g.pgm", g)
    dtb.imsave(tmp_path / "c.ppm", c)
    assert np.array_equal(dtb.imread(tmp_path / "g.pgm", 1), g)
    assert np.array_equal(dtb.imread(tmp_path / "c.ppm", 3), c)
    assert np.array_equal(np.asarray(Image.open(tmp_path / "g.pgm")), g)
    Image.fromarray(c, "RGB").save(tmp_path / "pil.ppm")
    assert np.array_equal(dtb.imread(tmp_path / "pil.ppm", 3), c)


def test_write_rejects_unknown_extension_and_mismatched_kind(tmp_path):
    with pytest.raises(DtbError):
        dtb.imsave(tmp_path / "g.jpg", _gray())
    with pytest.raises(DtbError):
        dtb.imsave(tmp_path / "c.pgm", _rgb())


def test_cli_normalize_matches_reference_formula():
    from distance_transform_benchmarks_b200.cli import normalize_u8
    d = np.array([[0.0, 1.0], [2.5, 10.0]], np.float32)
    assert np.array_equal(normalize_u8(d), np.array([[0, 25], [63, 255]], np.uint8))


@pytest.mark.gpu
def test_cli_end_to_end(tmp_path):
    from oracle import oracle as orc
    g = _gray(90, 120, seed=4)
    mask = np.zeros_like(g)
    mask[10, 20] = 255
    dtb.imsave(tmp_path / "in.png", g)
    dtb.imsave(tmp_path / "mask.png", mask)
    r = subprocess.run([sys.executable, "-m", "distance_transform_benchmarks_b200.cli", str(tmp_path / "in.png"), "0.5",
                        str(tmp_path / "out.png"), str(tmp_path / "mask.png"), "--raw", str(tmp_path / "d.npy")],
                       capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    d = np.load(tmp_path / "d.npy")
    assert np.array_equal(d.view(np.uint32), orc.ggdt_ref(g, mask, 0.5).view(np.uint32))
    from distance_transform_benchmarks_b200.cli import normalize_u8
    assert np.array_equal(dtb.imread(tmp_path / "out.png", 1), normalize_u8(d))
