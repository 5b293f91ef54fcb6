"""ref-mode parity against the reference's own compiled arithmetic.

oracle/_ref/libref_passes.so (built by oracle/Makefile `ref` from the reference source tree) runs the reference's
tile-pass device functions (dt/src/dt_block_passes.cuh:12-127) to quiescence on images of at most 32x32 pixels,
which is the reference's blocks-variant result for such an image.  These tests compare dtb_gdt_ref (C ABI) and
the CPU oracle with it bit for bit at lambdas whose products are inexact, which settles how nvcc contracts the
reference's weight expression (the golden tensors only cover lambda 0 and 1, where every product is exact).
"""
import numpy as np
import pytest
import torch

import distance_transform_benchmarks_b200 as dtb
from oracle import oracle as orc

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not orc.ref_passes_available(),
                       reason="oracle/_ref/libref_passes.so not built (the reference source tree was absent at build time)"),
]

LAMBDAS = [0.0, 0.1, 0.123, 0.3, 0.5, 0.7, 0.9, 0.999, 1.0]
SHAPES = [(32, 32), (17, 29), (1, 32), (32, 1), (5, 5), (31, 2)]


def _stack(rng, n, h, w, kind):
    if kind == "noise":
        imgs = rng.integers(0, 256, size=(n, h, w), dtype=np.uint8)
    else:  # smooth ramps plus a little noise: many near-ties between paths
        yy, xx = np.mgrid[0:h, 0:w]
        base = (xx * rng.uniform(0, 8, size=(n, 1, 1)) + yy * rng.uniform(0, 8, size=(n, 1, 1)))
        imgs = np.clip(base + rng.normal(0, 2, size=(n, h, w)), 0, 255).astype(np.uint8)
    masks = np.zeros((n, h, w), dtype=np.uint8)
    for k in range(n):
        for _ in range(int(rng.integers(1, 4))):
            masks[k, rng.integers(0, h), rng.integers(0, w)] = rng.choice([1, 255])
    masks[0] = 0  # one image without seeds: every pixel stays v
    return imgs, masks


def _ours(ctx, img, mask, lam, v, fma=True):
    d = dtb.generalised_distance_transform(torch.from_numpy(img).cuda(), torch.from_numpy(mask).cuda(), lam, v=v,
                                           ctx=ctx, fma=fma)
    return d.cpu().numpy()


@pytest.mark.parametrize("kind", ["noise", "smooth"])
@pytest.mark.parametrize("h,w", SHAPES)
def test_ref_mode_bit_exact_vs_reference_passes(ctx, h, w, kind):
    rng = np.random.default_rng(h * 131 + w + (7 if kind == "smooth" else 0))
    imgs, masks = _stack(rng, 6, h, w, kind)
    for lam in LAMBDAS:
        for v in (1e10, 300.0):
            ref = orc.ref_passes(imgs, masks, lam, v)
            for k in range(len(imgs)):
                ours = _ours(ctx, imgs[k], masks[k], lam, v)
                cpu = orc.ggdt_ref(imgs[k], masks[k], lam, v=v, fma=True)
                assert np.array_equal(ours.view(np.uint32), ref[k].view(np.uint32)), \
                    "GPU vs reference passes: lambda=%r v=%r image %d (%dx%d %s)" % (lam, v, k, h, w, kind)
                assert np.array_equal(cpu.view(np.uint32), ref[k].view(np.uint32)), \
                    "oracle vs reference passes: lambda=%r v=%r image %d" % (lam, v, k)


def test_reference_passes_reproduce_goldens_crop():
    """The reference's passes reproduce the reference's own golden tensors on a 32x32 crop (lambda 1, exact
    products), i.e. the driver wires the passes the way the reference does."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_goldens.npz"))
    for name in ("euclid", "geodesic"):
        img = g[name + "_img"][:32, :32]
        mask = g[name + "_mask"][:32, :32]
        if not mask.any():
            continue
        lam = float(g[name + "_lambda"])
        ref = orc.ref_passes(img[None], mask[None], lam)[0]
        assert np.array_equal(ref.view(np.uint32), orc.ggdt_ref(img, mask, lam, fma=True).view(np.uint32)), name


def test_no_fma_differs_somewhere(ctx):
    """The left-to-right rounding (DTB_FLAG_REF_NO_FMA) is a different function from the reference's compiled
    arithmetic at inexact lambdas: at least one pixel differs over a stack of noisy tiles.  (At lambda 0, 0.5
    and 1 both agree, which test_gpu_parity checks.)"""
    rng = np.random.default_rng(5)
    imgs, masks = _stack(rng, 16, 32, 32, "noise")
    lam = 0.3
    ref = orc.ref_passes(imgs, masks, lam)
    diff = 0
    for k in range(len(imgs)):
        nf = _ours(ctx, imgs[k], masks[k], lam, 1e10, fma=False)
        diff += int(np.count_nonzero(nf.view(np.uint32) != ref[k].view(np.uint32)))
    assert diff > 0
