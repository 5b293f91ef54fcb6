"""CPU tests of the oracle: pinned against the reference's golden tensors, and self-consistent.

Reference golden tests: tests/distance_transform.cpp:14-281 (EuclidianFastGeodis, lambda = 0) and :283-476
(GeodesicFastGeodis, lambda = 1); fixtures extracted by tests/golden/make_golden.py.
"""
import os

import numpy as np
import pytest

from oracle import oracle as orc
from tests.helpers import assert_images_eq

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_goldens.npz"))


@pytest.mark.parametrize("name", ["euclid", "geodesic"])
@pytest.mark.parametrize("fma", [True, False])
def test_oracle_matches_reference_goldens(name, fma):
    img, mask, ref = GOLD[name + "_img"], GOLD[name + "_mask"], GOLD[name + "_ref"]
    d = orc.ggdt_ref(img, mask, float(GOLD[name + "_lambda"]), float(GOLD["v"]), fma=fma)
    assert_images_eq(d, ref, "oracle vs reference golden %s" % name)


def test_golden_fixture_shapes():
    assert GOLD["euclid_ref"].shape == (40, 50)
    assert GOLD["geodesic_ref"].shape == (34, 36)
    assert int(GOLD["euclid_mask"].sum()) == 23 * 10
    assert GOLD["geodesic_mask"][17, 18] == 1 and int(GOLD["geodesic_mask"].sum()) == 1


def _blobs(seed, h, w):
    from distance_transform_benchmarks_b200 import workloads as wl
    return wl.blobs_gray(seed, w, h)


@pytest.mark.parametrize("lam", [0.0, 0.5, 1.0])
def test_ref_fma_irrelevant_for_exact_products(lam):
    # lambda in {0, 0.5, 1}: every product is exact, so contraction cannot change a bit.
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, (37, 45), dtype=np.uint8)
    mask = np.zeros_like(img); mask[18, 22] = 1; mask[3, 40] = 1
    assert_images_eq(orc.ggdt_ref(img, mask, lam, fma=True), orc.ggdt_ref(img, mask, lam, fma=False))


@pytest.mark.parametrize("rgb", [False, True])
def test_ns_schedule_independence(rgb):
    rng = np.random.default_rng(2)
    shape = (61, 83, 3) if rgb else (61, 83)
    img = rng.integers(0, 256, shape, dtype=np.uint8)
    mask = np.zeros((61, 83), np.uint8); mask[5, 7] = 1; mask[50, 70] = 1
    a = orc.ggdt_ns(img, mask, 0.1)
    b = orc.ggdt_ns(img, mask, 0.1, serial=True)
    c = orc.ggdt_ns(img, mask, 0.1, nthreads=1)
    assert_images_eq(a, b, "parallel vs serial")
    assert_images_eq(a, c, "parallel vs 1 thread")


def test_ns_close_to_fp64_dijkstra():
    img = _blobs(5, 128, 160)
    mask = np.zeros(img.shape, np.uint8); mask[10, 10] = 1; mask[100, 150] = 1
    d = orc.ggdt_ns(img, mask, 0.0392156876)
    dj = orc.dijkstra_ns_f64(img, mask, 0.0392156876)
    rel = np.abs(d - dj) / np.maximum(dj, 1e-30)
    assert rel.max() < 1e-5


def test_ns_warm_start_equals_cold_union():
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, (70, 90), dtype=np.uint8)
    m1 = np.zeros(img.shape, np.uint8); m1[10, 10] = 1
    m2 = np.zeros(img.shape, np.uint8); m2[60, 80] = 1; m2[30, 5] = 1
    prev = orc.ggdt_ns(img, m1, 0.5)
    warm = orc.ggdt_ns_warm(img, m2, prev, 0.5)
    cold = orc.ggdt_ns(img, m1 | m2, 0.5)
    assert_images_eq(warm, cold, "warm vs cold")


def test_no_seed_gives_v_everywhere():
    img = np.zeros((9, 11), np.uint8)
    mask = np.zeros_like(img)
    assert np.all(orc.ggdt_ns(img, mask, 1.0, v=123.0) == np.float32(123.0))
    assert np.all(orc.ggdt_ref(img, mask, 0.5, v=7.0) == np.float32(7.0))


@pytest.mark.parametrize("kind", ["gray", "rgb8", "const"])
def test_ns_unit_weights_are_city_block_distance(kind):
    """gamma = 0 (or an image without intensity steps) makes every C4 edge weigh exactly 1: the map is then the
    integer city-block distance to the nearest seed, computed independently by scipy's chamfer transform."""
    from scipy import ndimage
    from distance_transform_benchmarks_b200 import workloads as wl
    rng = np.random.default_rng(17)
    h, w = 97, 131
    if kind == "const":
        img, gamma = np.full((h, w), 77, np.uint8), 1.0
    elif kind == "gray":
        img, gamma = rng.integers(0, 256, (h, w), dtype=np.uint8), 0.0
    else:
        img, gamma = rng.integers(0, 256, (h, w, 3), dtype=np.uint8), 0.0
    mask = wl.random_disks(rng, w, h, 5, 1, 6)
    expect = ndimage.distance_transform_cdt(mask == 0, metric="taxicab").astype(np.float32)
    assert_images_eq(orc.ggdt_ns(img, mask, gamma), expect, "unit weights, %s" % kind)


@pytest.mark.parametrize("rgb", [False, True])
def test_ns_union_of_seed_sets_is_elementwise_min(rgb):
    """A value is the minimum over paths of the path's fp32 sum from its seed: T(A | B) == min(T(A), T(B))."""
    from distance_transform_benchmarks_b200 import workloads as wl
    rng = np.random.default_rng(5)
    img = wl.voronoi_rgb(3, 150, 120) if rgb else wl.blobs_gray(3, 150, 120)
    a = wl.random_disks(rng, 150, 120, 3, 1, 4)
    b = wl.random_disks(rng, 150, 120, 4, 1, 4)
    for g in (0.02, 1.0):
        expect = np.minimum(orc.ggdt_ns(img, a, g), orc.ggdt_ns(img, b, g))
        assert_images_eq(orc.ggdt_ns(img, a | b, g), expect, "union, gamma %g" % g)


@pytest.mark.parametrize("lam", [0.0, 0.5, 1.0])
def test_ref_union_of_seed_sets_is_elementwise_min(lam):
    from distance_transform_benchmarks_b200 import workloads as wl
    rng = np.random.default_rng(6)
    img = wl.blobs_gray(4, 140, 110)
    a = wl.random_disks(rng, 140, 110, 3, 1, 4)
    b = wl.random_disks(rng, 140, 110, 4, 1, 4)
    for fma in (True, False):
        expect = np.minimum(orc.ggdt_ref(img, a, lam, fma=fma), orc.ggdt_ref(img, b, lam, fma=fma))
        assert_images_eq(orc.ggdt_ref(img, a | b, lam, fma=fma), expect, "ref union, fma %s" % fma)
