"""Seeded synthetic workloads of the GGDT benchmark configurations.

The reference measures on photographs that are not available here (benchmarks/distance_transform.cpp:17);
these generators produce inputs with the configured shapes and value distributions instead:

* ``config0``: 512x512 gray, 16 Gaussian blobs (sigma U[20, 80], amplitude U[0, 255]) + N(0, 4^2) noise,
  5 seed disks of radius 3, gamma = fl32(fl32(1/255) * 10).
* ``config1``: 4096x4096 gray perfect maze (128x128 cells of 32 px, walls 4 px = 255, corridors 0, + U{0..8}),
  one 1-px seed at the first dead end, gamma = 0.5.
* ``config2``: 8192x8192 rgb8 Voronoi mosaic (256 sites, uniform colours + N(0, 6^2) per channel),
  64 seed disks of radius 5, gamma = 0.02.
* ``config3``: ragged batch of 1024 images, sides log-uniform in [64, 2048] (independent H and W), even index
  gray blobs / odd index rgb8 Voronoi, 1-8 seed disks of radius 2-6, gamma from {0.01, 0.1, 1.0}.

Per-image parameters come from numpy's PCG64; pixels from the C++ generators of csrc/datagen.cpp, loaded from
libdtb_host.so unless ``use_generator`` names another build of the same source (bench.py's CPU reference arm
uses the oracle's copy, so that process loads no library of this package).
"""
import ctypes
import math

import numpy as np

from ._native import declare_generator, host

_gen_lib = None


def use_generator(path):
    """Takes the pixel generators from the shared library at `path`, a build of csrc/datagen.cpp (same source,
    same pixels), instead of libdtb_host.so."""
    global _gen_lib
    _gen_lib = declare_generator(ctypes.CDLL(path))


def _gen():
    return _gen_lib if _gen_lib is not None else host()


GAMMA_C0 = np.float32(np.float32(1.0) / np.float32(255.0) * np.float32(10.0))


def _seed_of(*parts):
    s = np.random.SeedSequence(list(parts))
    return int(s.generate_state(1, np.uint64)[0])


def blobs_gray(seed, w, h, nblobs=16, smin=20.0, smax=80.0, amin=0.0, amax=255.0, noise=4.0):
    out = np.empty((h, w), np.uint8)
    _gen().dtbg_blobs_gray(seed, w, h, nblobs, smin, smax, amin, amax, noise, out.ctypes.data, w)
    return out


def voronoi_rgb(seed, w, h, nsites=256, noise=6.0):
    out = np.empty((h, w, 3), np.uint8)
    _gen().dtbg_voronoi_rgb(seed, w, h, nsites, noise, out.ctypes.data, 3 * w)
    return out


def maze_gray(seed, w, h, cell=32, wall=4, noise_max=8):
    out = np.empty((h, w), np.uint8)
    sx, sy = ctypes.c_int(), ctypes.c_int()
    r = _gen().dtbg_maze_gray(seed, w, h, cell, wall, noise_max, out.ctypes.data, w, ctypes.byref(sx), ctypes.byref(sy))
    if r != 0:
        raise ValueError("bad maze parameters")
    return out, (sx.value, sy.value)


def disks_mask(w, h, centres, radii):
    mask = np.zeros((h, w), np.uint8)
    n = len(radii)
    if n:
        cx = np.ascontiguousarray([c[0] for c in centres], np.int32)
        cy = np.ascontiguousarray([c[1] for c in centres], np.int32)
        r = np.ascontiguousarray(radii, np.int32)
        _gen().dtbg_draw_disks(mask.ctypes.data, w, w, h, n, cx.ctypes.data, cy.ctypes.data, r.ctypes.data)
    return mask


def random_disks(rng, w, h, n, rmin, rmax):
    centres = [(int(rng.integers(0, w)), int(rng.integers(0, h))) for _ in range(n)]
    radii = [int(rng.integers(rmin, rmax + 1)) for _ in range(n)]
    return disks_mask(w, h, centres, radii)


def config0(seed=0, w=512, h=512):
    rng = np.random.default_rng(_seed_of(0, seed))
    img = blobs_gray(_seed_of(0, seed, 1), w, h)
    mask = random_disks(rng, w, h, 5, 3, 3)
    return img, mask, float(GAMMA_C0)


def config1(seed=1, w=4096, h=4096):
    img, (sx, sy) = maze_gray(_seed_of(1, seed, 1), w, h)
    mask = np.zeros((h, w), np.uint8)
    mask[sy, sx] = 1
    return img, mask, 0.5


def config2(seed=2, w=8192, h=8192):
    rng = np.random.default_rng(_seed_of(2, seed))
    img = voronoi_rgb(_seed_of(2, seed, 1), w, h)
    mask = random_disks(rng, w, h, 64, 5, 5)
    return img, mask, 0.02


def config3_specs(seed=3, n=1024, smin=64, smax=2048):
    """Per-image (kind, w, h, gamma, seed) of the ragged batch, without generating pixels."""
    rng = np.random.default_rng(_seed_of(3, seed))
    lo, hi = math.log(smin), math.log(smax)
    specs = []
    for i in range(n):
        w = int(min(smax, max(smin, round(math.exp(rng.uniform(lo, hi))))))
        h = int(min(smax, max(smin, round(math.exp(rng.uniform(lo, hi))))))
        gamma = float(np.float32(rng.choice([0.01, 0.1, 1.0])))
        specs.append(("gray" if i % 2 == 0 else "rgb8", w, h, gamma, _seed_of(3, seed, i)))
    return specs


def make_image(spec):
    """(img, mask, gamma) of one config3-style spec."""
    kind, w, h, gamma, s = spec
    rng = np.random.default_rng(_seed_of(s, 7))
    img = blobs_gray(s, w, h) if kind == "gray" else voronoi_rgb(s, w, h)
    k = int(rng.integers(1, 9))
    mask = random_disks(rng, w, h, k, 2, 6)
    return img, mask, gamma


def config3(seed=3, n=1024, smin=64, smax=2048):
    return [make_image(s) for s in config3_specs(seed, n, smin, smax)]


def stratified_indices(specs, target_mpx):
    """Every k-th image of a batch (k odd, so gray and rgb8 images alternate in the sample), k chosen so that the
    sample holds about `target_mpx` million pixels: a deterministic sample with the batch's size and kind mix."""
    total = sum(s[1] * s[2] for s in specs)
    k = max(1, int(round(total / max(1.0, target_mpx * 1e6))))
    if k % 2 == 0:
        k += 1
    return list(range(0, len(specs), k))


def pixels(batch):
    return sum(int(img.shape[0]) * int(img.shape[1]) for img, _, _ in batch)


def bytes_per_pixel(img):
    """Algorithmic bytes per pixel: image read (1 or 3) + seed mask read (1) + distance write (4)."""
    return (3 if img.ndim == 3 else 1) + 1 + 4
