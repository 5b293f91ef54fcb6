"""GPU test of dtb_gdt_noalloc, the entry point for callers that must not allocate device memory (a host that
owns all device memory through its own pool or budget, or a loop that cannot pay for the synchronisation of
cudaMalloc / cudaFree).  It keeps its scratch in a fixed device array of the library instead of a context.

Its output must equal the regular entry point's (dtb_gdt through a context) and the oracle's bit for bit -- the
tolerance of every parity test here -- on two calls in a row, which also shows that a call does not depend on
what the previous call left in the shared array.  A call after the first must leave the device's free memory
unchanged, the largest image the fixed array allows must work, and inputs it cannot take without a staging copy
(host memory, unaligned rows) must be rejected.  This file is collected last so that a run that stops at the
first failure has already run every other test; it passes alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

import distance_transform_benchmarks_b200 as dtb
from distance_transform_benchmarks_b200 import _native
from distance_transform_benchmarks_b200 import workloads as wl
from distance_transform_benchmarks_b200.verify import ns_fixpoint_violations
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

DTB_ERR_INVALID_ARG = 1
DTB_ERR_CAPACITY = 7


def _noalloc(img, mask, dist, gamma, v=1e10):
    es = 3 if img.dim() == 3 else 1
    vi, vm, vd = dtb.image_view(img, es), dtb.image_view(mask, 1), dtb.image_view(dist, 4)
    return _native.lib().dtb_gdt_noalloc(ctypes.byref(vi), ctypes.byref(vm), ctypes.byref(vd), float(gamma), float(v),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def _case(kind):
    if kind == "gray":
        img, mask, gamma = wl.config0()
    else:
        img = wl.voronoi_rgb(77, 400, 272)
        mask = wl.random_disks(np.random.default_rng(77), 400, 272, 6, 2, 5)
        gamma = 0.02
    return torch.from_numpy(img).cuda(), torch.from_numpy(mask).cuda(), gamma


def test_noalloc_matches_context_entry_point_on_consecutive_calls():
    ctx = dtb.Context(0)
    for kind in ("gray", "rgb8"):  # two calls in a row on different images
        img, mask, gamma = _case(kind)
        out = torch.full(img.shape[:2], -1.0, dtype=torch.float32, device="cuda")
        assert _noalloc(img, mask, out, gamma) == 0
        ref = dtb.geodesic_distance_transform(img, mask, gamma, ctx=ctx)
        torch.cuda.synchronize()
        assert torch.equal(out.view(torch.int32), ref.view(torch.int32)), kind
        host = out.cpu().numpy()
        expect = orc.ggdt_ns(img.cpu().numpy(), mask.cpu().numpy(), gamma)
        assert np.array_equal(host.view(np.uint32), expect.view(np.uint32)), kind
    ctx.close()


def test_noalloc_call_allocates_nothing():
    img, mask, gamma = _case("rgb8")
    out = torch.empty(img.shape[:2], dtype=torch.float32, device="cuda")
    out.fill_(-1.0)
    assert _noalloc(img, mask, out, gamma) == 0  # set-up call (module load, symbol address, attributes)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        out.fill_(-1.0)
        assert _noalloc(img, mask, out, gamma) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    expect = orc.ggdt_ns(img.cpu().numpy(), mask.cpu().numpy(), gamma)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), expect.view(np.uint32))


def test_noalloc_largest_image():
    # 4096 x 4096 pixels: exactly the 16384 tiles the fixed array holds.
    img, mask, gamma = wl.config1()
    ti, tm = torch.from_numpy(img).cuda(), torch.from_numpy(mask).cuda()
    out = torch.empty(img.shape, dtype=torch.float32, device="cuda")
    assert _noalloc(ti, tm, out, gamma) == 0
    ctx = dtb.Context(0)
    ref = dtb.geodesic_distance_transform(ti, tm, gamma, ctx=ctx)
    torch.cuda.synchronize()
    assert torch.equal(out.view(torch.int32), ref.view(torch.int32))
    va, vb, _ = ns_fixpoint_violations(ti, tm, gamma, 1e10, out)
    assert va == 0 and vb == 0
    ctx.close()


def test_noalloc_rejects_inputs_it_would_have_to_stage():
    img, mask, gamma = _case("gray")
    out = torch.empty(img.shape[:2], dtype=torch.float32, device="cuda")
    # host memory
    assert _noalloc(img.cpu(), mask, out, gamma) == DTB_ERR_INVALID_ARG
    assert _noalloc(img, mask, out.cpu(), gamma) == DTB_ERR_INVALID_ARG
    # rows not on 16-byte boundaries (TMA needs them): a 512-wide view of 520-byte rows
    h, w = img.shape
    wide = torch.zeros((h, w + 8), dtype=torch.uint8, device="cuda")
    wide[:, :w] = img
    assert _noalloc(wide[:, :w], mask, out, gamma) == DTB_ERR_INVALID_ARG


def test_noalloc_rejects_images_beyond_its_fixed_scratch():
    w, h = 4128, 4096  # 129 x 128 = 16512 tiles > 16384
    img = torch.zeros((h, w), dtype=torch.uint8, device="cuda")
    mask = torch.zeros((h, w), dtype=torch.uint8, device="cuda")
    dist = torch.zeros((h, w), dtype=torch.float32, device="cuda")
    assert _noalloc(img, mask, dist, 0.1) == DTB_ERR_CAPACITY
