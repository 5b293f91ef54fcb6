"""Failure detection on the GPU without a device fault.

Every wait of the tile kernel is bounded (no-progress watchdog on the tile queue, TMA timeout, phase and visit
caps).  dtb_debug_inject_queue_stall makes the queue wait run out on purpose: the next run counts one tile that
is never queued, so no worker can finish; after the (short) limit each worker records DERR_QUEUE_TIMEOUT and
returns, and the call reports DTB_ERR_TIMEOUT.  The context must stay usable afterwards.
"""
import time

import numpy as np
import pytest
import torch

import distance_transform_benchmarks_b200 as dtb
from distance_transform_benchmarks_b200 import workloads as wl
from distance_transform_benchmarks_b200._native import DtbError
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

DTB_ERR_TIMEOUT = 4


def test_queue_watchdog_ends_a_stalled_run_and_the_context_stays_usable(ctx):
    img, mask, gamma = wl.config0()
    ti, tm = torch.from_numpy(img).cuda(), torch.from_numpy(mask).cuda()
    ref = orc.ggdt_ns(img, mask, gamma)
    ctx.inject_queue_stall(200)
    t0 = time.perf_counter()
    with pytest.raises(DtbError) as e:
        dtb.geodesic_distance_transform(ti, tm, gamma, ctx=ctx)
    elapsed = time.perf_counter() - t0
    assert e.value.status == DTB_ERR_TIMEOUT, str(e.value)
    assert "no progress" in str(e.value)
    assert 0.15 < elapsed < 30.0, elapsed
    # The injection is one-shot and the context (and device) are still good.
    for _ in range(2):
        d = dtb.geodesic_distance_transform(ti, tm, gamma, ctx=ctx)
        assert np.array_equal(d.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_stalled_batch_reports_timeout_then_recovers(ctx):
    specs = wl.config3_specs(seed=5, n=12)
    batch = [wl.make_image(s) for s in specs]
    imgs = [torch.from_numpy(i).cuda() for i, _, _ in batch]
    masks = [torch.from_numpy(m).cuda() for _, m, _ in batch]
    gammas = [g for _, _, g in batch]
    ctx.inject_queue_stall(100)
    with pytest.raises(DtbError) as e:
        dtb.geodesic_distance_transform_batch(imgs, masks, gammas, ctx=ctx)
    assert e.value.status == DTB_ERR_TIMEOUT
    out = dtb.geodesic_distance_transform_batch(imgs, masks, gammas, ctx=ctx)
    for (i, m, g), d in zip(batch, out):
        assert np.array_equal(d.cpu().numpy().view(np.uint32), orc.ggdt_ns(i, m, g).view(np.uint32))
