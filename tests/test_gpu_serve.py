"""GPU tests of the serving engine: every result is exact against the oracle, alone and in the mix.

A new-image request must equal a cold run of its image and mask; a seed edit must equal a cold run with the
union of the image's original seeds and every disk added to it so far (warm starts are exact because added
seeds only lower distances).  The tests that apply to both engines run with waves (live=False) and with live
admission into a running tile kernel (live=True).
"""
import time

import numpy as np
import pytest
import torch

import distance_transform_benchmarks_b200 as dtb
from distance_transform_benchmarks_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import assert_images_eq

pytestmark = pytest.mark.gpu


def _drain(srv, n, timeout=60.0):
    got, t0 = {}, time.time()
    while len(got) < n:
        for c in srv.poll(wait_ms=50):
            got[c["request_id"]] = c
        assert time.time() - t0 < timeout, "serve requests did not complete"
    return got


def _images(seed, count, smin=40, smax=300):
    return wl.config3(seed=seed, n=count, smin=smin, smax=smax)


def _disks(rng, img, k):
    h, w = img.shape[:2]
    return [(int(rng.integers(0, w)), int(rng.integers(0, h)), 3) for _ in range(k)]


def _mask_with(mask, disks):
    h, w = mask.shape
    return mask | wl.disks_mask(w, h, [(x, y) for x, y, _ in disks], [r for _, _, r in disks])


BOTH = pytest.mark.parametrize("live", [False, True], ids=["waves", "live"])


@BOTH
def test_requests_in_the_mix_match_the_oracle_and_running_alone(live):
    rng = np.random.default_rng(0)
    batch = _images(31, 8)
    srv = dtb.Server(256 << 20, live=live)
    expected, outs = {}, {}
    masks_now = {}
    # all new images at once, then edits submitted while the first waves still run
    for i, (img, mask, g) in enumerate(batch):
        out = torch.empty(img.shape[:2], dtype=torch.float32).pin_memory()
        rid = srv.submit_image(100 + i, torch.from_numpy(img).pin_memory(), torch.from_numpy(mask).pin_memory(), g, out)
        outs[rid] = out
        expected[rid] = orc.ggdt_ns(img, mask, g)
        masks_now[100 + i] = mask.copy()
    for round_ in range(2):
        for i in (1, 4, 6):
            img, _, g = batch[i]
            disks = _disks(rng, img, int(rng.integers(1, 4)))
            masks_now[100 + i] = _mask_with(masks_now[100 + i], disks)
            out = torch.empty(img.shape[:2], dtype=torch.float32).pin_memory()
            rid = srv.submit_edit(100 + i, disks, out)
            outs[rid] = out
            expected[rid] = orc.ggdt_ns(img, masks_now[100 + i], g)
    got = _drain(srv, len(outs))
    for rid, c in got.items():
        assert c["status"] == 0, c
        assert c["latency_ms"] > 0
        assert_images_eq(outs[rid], expected[rid], "request %d" % rid)
    st = srv.stats()
    assert st["completed"] == len(outs) and st["failed"] == 0 and st["waves"] >= 1
    srv.close()
    # the same new image alone in its own server gives the same bits
    img, mask, g = batch[4]
    alone = dtb.Server(64 << 20, live=live)
    out = torch.empty(img.shape[:2], dtype=torch.float32)
    rid = alone.submit_image(1, torch.from_numpy(img), torch.from_numpy(mask), g, out)
    assert _drain(alone, 1)[rid]["status"] == 0
    first = [r for r in expected if np.array_equal(expected[r], orc.ggdt_ns(img, mask, g))][0]
    assert_images_eq(out, outs[first].numpy(), "alone vs mixed")
    alone.close()


@BOTH
def test_budget_eviction_and_capacity(live):
    batch = _images(32, 6, smin=200, smax=260)
    def a128(x):
        return -(-x // 128) * 128

    def planes(img):  # device bytes of one resident image, as the engine lays them out
        h, w = img.shape[:2]
        c = 3 if img.ndim == 3 else 1
        rb = w * c
        return h * ((rb if rb % 16 == 0 else a128(rb)) + (w if w % 16 == 0 else a128(w)) + a128(4 * w)) + 3 * 256

    per_image = max(planes(i) for i, _, _ in batch)
    srv = dtb.Server(3 * per_image, live=live)
    outs = {}
    for i, (img, mask, g) in enumerate(batch):
        out = torch.empty(img.shape[:2], dtype=torch.float32)
        outs[srv.submit_image(i, torch.from_numpy(img), torch.from_numpy(mask), g, out)] = (out, img, mask, g)
        _drain(srv, 1)  # one at a time: older images become evictable
    for rid, (out, img, mask, g) in outs.items():
        assert_images_eq(out, orc.ggdt_ns(img, mask, g), "evicting server %d" % rid)
    st = srv.stats()
    assert st["evictions"] >= 1
    # an edit of an evicted image fails; an image larger than the whole budget fails
    out = torch.empty(batch[0][0].shape[:2], dtype=torch.float32)
    rid = srv.submit_edit(0, [(5, 5, 3)], out)
    assert _drain(srv, 1)[rid]["status"] == 1
    big = np.zeros((2048, 2048), np.uint8)
    out = torch.empty((2048, 2048), dtype=torch.float32)
    rid = srv.submit_image(99, torch.from_numpy(big), torch.from_numpy(big), 0.1, out)
    assert _drain(srv, 1)[rid]["status"] == 7
    srv.close()


@BOTH
def test_overlapping_small_waves_keep_per_image_order(live):
    """Two waves in flight at a time: with at most two requests per wave, new images and edits of images whose
    own wave may still be running (they wait for it) are all exact, edits applied in submission order.  Live:
    at most two requests in flight at once, the same order rule."""
    rng = np.random.default_rng(7)
    batch = _images(33, 24, smin=40, smax=260)
    srv = dtb.Server(512 << 20, max_wave_requests=2, live=live)
    masks_now, outs, expected = {}, {}, {}

    def edit(j):
        img, _, g = batch[j]
        disks = _disks(rng, img, int(rng.integers(1, 4)))
        masks_now[j] = _mask_with(masks_now[j], disks)
        out = torch.empty(img.shape[:2], dtype=torch.float32).pin_memory()
        rid = srv.submit_edit(j, disks, out)
        outs[rid] = out
        expected[rid] = orc.ggdt_ns(img, masks_now[j], g)

    for i, (img, mask, g) in enumerate(batch):
        out = torch.empty(img.shape[:2], dtype=torch.float32).pin_memory()
        rid = srv.submit_image(i, torch.from_numpy(img).pin_memory(), torch.from_numpy(mask).pin_memory(), g, out)
        outs[rid] = out
        expected[rid] = orc.ggdt_ns(img, mask, g)
        masks_now[i] = mask.copy()
        if i % 3 == 2:
            for j in (i, i, i - 2):
                edit(j)
    got = _drain(srv, len(outs))
    for rid, c in got.items():
        assert c["status"] == 0, c
        assert_images_eq(outs[rid], expected[rid], "request %d" % rid)
    st = srv.stats()
    assert st["completed"] == len(outs) and st["failed"] == 0
    if not live:
        assert st["waves"] >= len(outs) // 2
    srv.close()


@BOTH
def test_failed_wave_fails_its_requests_only(live):
    """A wave whose tile queue stalls (host-side injection: one phantom queued tile, short no-progress limit;
    no device fault) completes its requests with DTB_ERR_TIMEOUT and drops its new image; the engine keeps
    serving, and requests before and after it are exact.  Live: the stalled request is the next one the running
    kernel claims; the kernel ends on its watchdog and the next request launches it again."""
    rng = np.random.default_rng(9)
    batch = _images(35, 3, smin=60, smax=200)
    ctx = dtb.Context(0)
    srv = dtb.Server(128 << 20, ctx=ctx, live=live)

    def new_image(i):
        img, mask, g = batch[i]
        out = torch.empty(img.shape[:2], dtype=torch.float32)
        rid = srv.submit_image(i, torch.from_numpy(img), torch.from_numpy(mask), g, out)
        return _drain(srv, 1)[rid]["status"], out

    status, out0 = new_image(0)
    assert status == 0
    assert_images_eq(out0, orc.ggdt_ns(*batch[0]), "before the stall")
    ctx.inject_queue_stall(100)
    status, _ = new_image(1)
    assert status == 4  # DTB_ERR_TIMEOUT
    out = torch.empty(batch[1][0].shape[:2], dtype=torch.float32)
    rid = srv.submit_edit(1, [(5, 5, 3)], out)
    assert _drain(srv, 1)[rid]["status"] == 1  # the failed image was not kept
    status, out2 = new_image(2)
    assert status == 0
    assert_images_eq(out2, orc.ggdt_ns(*batch[2]), "after the stall")
    img, mask, g = batch[0]
    disks = _disks(rng, img, 2)
    out = torch.empty(img.shape[:2], dtype=torch.float32)
    rid = srv.submit_edit(0, disks, out)
    assert _drain(srv, 1)[rid]["status"] == 0
    assert_images_eq(out, orc.ggdt_ns(img, _mask_with(mask, disks), g), "edit after the stall")
    st = srv.stats()
    assert st["failed"] == 2
    srv.close()
    ctx.close()


def test_waves_split_at_their_limits_allocate_nothing_and_report_phase_times():
    """Waves run in buffers sized at create time: a per-wave limit closes a wave while requests are left (they
    wait for the next wave), every result stays exact, the device's free memory does not change while the waves
    run, the statistics say where the time went, and an image larger than a whole wave may be is rejected."""
    batch = _images(57, 14, smin=100, smax=400)
    # one request per wave: a burst of submissions leaves requests waiting at an admission, which then closes
    # the wave at the limit; images have at most 13 x 13 tiles, under the tile limit
    srv = dtb.Server(256 << 20, max_wave_requests=1, max_wave_tiles=200, wave_stage_bytes=4 << 20)
    outs, expected = {}, {}
    hosts = [(torch.from_numpy(i).pin_memory(), torch.from_numpy(m).pin_memory()) for i, m, _ in batch]
    bufs = [torch.empty(i.shape[:2], dtype=torch.float32).pin_memory() for i, _, _ in batch]
    refs = [orc.ggdt_ns(img, mask, g) for img, mask, g in batch]  # before the burst: submissions back to back
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k, ((img, mask, g), (hi, hm)) in enumerate(zip(batch, hosts)):
        rid = srv.submit_image(500 + k, hi, hm, g, bufs[k])
        outs[rid] = bufs[k]
        expected[rid] = refs[k]
    got = _drain(srv, len(outs))
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for rid, c in got.items():
        assert c["status"] == 0, c
        assert_images_eq(outs[rid], expected[rid], "split-wave request %d" % rid)
    st = srv.stats()
    assert st["failed"] == 0 and st["waves"] == len(batch) and st["waves_split"] >= 1, st
    assert st["kernel_ms"] > 0 and st["copy_in_ms"] > 0 and st["copy_out_ms"] > 0 and st["host_prep_ms"] > 0, st
    assert st["queue_wait_max_ms"] >= st["queue_wait_ms"] / max(1, st["completed"])
    # an image alone above the per-wave tile limit is rejected, and the server keeps serving
    big = np.zeros((600, 600), np.uint8)
    out = torch.empty((600, 600), dtype=torch.float32)
    rid = srv.submit_image(900, torch.from_numpy(big), torch.from_numpy(big), 0.1, out)
    assert _drain(srv, 1)[rid]["status"] == 7  # DTB_ERR_CAPACITY: 19 x 19 tiles > 200
    img, mask, g = batch[0]
    out = torch.empty(img.shape[:2], dtype=torch.float32)
    rid = srv.submit_image(901, torch.from_numpy(img), torch.from_numpy(mask), g, out)
    assert _drain(srv, 1)[rid]["status"] == 0
    assert_images_eq(out, orc.ggdt_ns(img, mask, g), "after a rejected request")
    srv.close()


def test_live_request_admitted_while_another_runs_finishes_first():
    """Live admission: small requests submitted while a long one (the 4096 x 4096 maze, many re-activation
    rounds) is on the GPU are claimed by the running kernel and complete before it, all in one launch; each map
    equals its run alone (the small ones against the oracle, the maze against a one-shot call)."""
    maze, mmask, mg = wl.config1()
    small = _images(61, 6, smin=64, smax=200)
    srv = dtb.Server(1 << 30, live=True, live_idle_us=200000)
    order = []
    out_m = torch.empty(maze.shape, dtype=torch.float32).pin_memory()
    hm, hmm = torch.from_numpy(maze).pin_memory(), torch.from_numpy(mmask).pin_memory()
    small_in = [(torch.from_numpy(i).pin_memory(), torch.from_numpy(m).pin_memory()) for i, m, _ in small]
    outs = [torch.empty(i.shape[:2], dtype=torch.float32).pin_memory() for i, _, _ in small]
    rid_m = srv.submit_image(1, hm, hmm, mg, out_m)
    time.sleep(0.002)  # the maze is claimed and running
    rids = [srv.submit_image(10 + k, hi, hk, g, outs[k]) for k, ((hi, hk), (_, _, g)) in enumerate(zip(small_in, small))]
    t0 = time.time()
    while len(order) < 1 + len(rids):
        for c in srv.poll(wait_ms=50):
            assert c["status"] == 0, c
            order.append(c["request_id"])
        assert time.time() - t0 < 60
    assert order.index(rid_m) == len(order) - 1, order  # every small request ended before the maze
    st = srv.stats()
    assert st["waves"] == 1, st  # one launch served them all
    srv.close()
    for k, (img, mask, g) in enumerate(small):
        assert_images_eq(outs[k], orc.ggdt_ns(img, mask, g), "small request %d" % k)
    ref = dtb.geodesic_distance_transform(torch.from_numpy(maze).cuda(), torch.from_numpy(mmask).cuda(), mg)
    assert_images_eq(out_m, ref.cpu().numpy(), "maze, live vs one-shot")


def test_live_kernel_ends_when_idle_relaunches_and_allocates_nothing():
    """The live kernel ends after its idle time; the next request launches it again.  Serving allocates no
    device memory (free memory unchanged across requests and launches), and edits stay exact across launches."""
    rng = np.random.default_rng(3)
    batch = _images(62, 4, smin=80, smax=300)
    srv = dtb.Server(256 << 20, live=True, live_idle_us=2000)
    hosts = [(torch.from_numpy(i).pin_memory(), torch.from_numpy(m).pin_memory()) for i, m, _ in batch]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    masks_now = {}
    for k, ((img, mask, g), (hi, hm)) in enumerate(zip(batch, hosts)):
        out = torch.empty(img.shape[:2], dtype=torch.float32).pin_memory()
        rid = srv.submit_image(k, hi, hm, g, out)
        assert _drain(srv, 1)[rid]["status"] == 0
        assert_images_eq(out, orc.ggdt_ns(img, mask, g), "image %d" % k)
        masks_now[k] = mask.copy()
        time.sleep(0.05)  # well past the idle time: the kernel has ended
    for k in (0, 2, 0):
        img, _, g = batch[k]
        disks = _disks(rng, img, 2)
        masks_now[k] = _mask_with(masks_now[k], disks)
        out = torch.empty(img.shape[:2], dtype=torch.float32).pin_memory()
        rid = srv.submit_edit(k, disks, out)
        assert _drain(srv, 1)[rid]["status"] == 0
        assert_images_eq(out, orc.ggdt_ns(img, masks_now[k], g), "edit of image %d" % k)
        time.sleep(0.05)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    st = srv.stats()
    assert st["failed"] == 0 and st["waves"] >= 7, st  # a launch per request after each idle end
    assert st["tile_visits"] > 0 and st["kernel_ms"] > 0
    srv.close()


@BOTH
def test_odd_shapes_and_their_edits_match_the_oracle(live):
    """Edge shapes through both engines: one-pixel and one-row / one-column images, sides that are not multiples
    of the 32-pixel tile or of 16 bytes, and a 1023 x 8 rgb8 image whose staged rows do not fit its distance plane
    (live engine: the copy goes straight into place instead); each new image and one edit of it equal the
    oracle's map."""
    rng = np.random.default_rng(11)
    shapes = [(1, 1, 1), (33, 1, 1), (1, 57, 1), (1023, 8, 3), (257, 3, 3), (31, 95, 1), (65, 33, 3)]
    srv = dtb.Server(64 << 20, live=live)
    for k, (w, h, c) in enumerate(shapes):
        img = (wl.blobs_gray(100 + k, w, h) if c == 1 else wl.voronoi_rgb(100 + k, w, h))
        mask = np.zeros((h, w), np.uint8)
        mask[int(rng.integers(0, h)), int(rng.integers(0, w))] = 1
        g = 0.1
        out = torch.empty((h, w), dtype=torch.float32)
        rid = srv.submit_image(k, torch.from_numpy(img), torch.from_numpy(mask), g, out)
        assert _drain(srv, 1)[rid]["status"] == 0
        assert_images_eq(out, orc.ggdt_ns(img, mask, g), "image %dx%dx%d" % (w, h, c))
        disks = [(int(rng.integers(0, w)), int(rng.integers(0, h)), 1)]
        out2 = torch.empty((h, w), dtype=torch.float32)
        rid = srv.submit_edit(k, disks, out2)
        assert _drain(srv, 1)[rid]["status"] == 0
        assert_images_eq(out2, orc.ggdt_ns(img, _mask_with(mask, disks), g), "edit of %dx%dx%d" % (w, h, c))
    assert srv.stats()["failed"] == 0
    srv.close()
