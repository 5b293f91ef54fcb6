"""GPU parity tests: the CUDA path against the oracle, bit for bit.

Mirrors the reference's tests/distance_transform.cpp: the two golden tensors (:14-281, :283-476) through all
three entry points, and cross-variant equality on random images (:485-559) -- here seeded, and against the
oracle rather than against another GPU variant.  Full-size workloads are checked through the exact fixpoint
characterisation of tests/helpers.py.
"""
import os

import numpy as np
import pytest
import torch

import distance_transform_benchmarks_b200 as dtb
from distance_transform_benchmarks_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import assert_images_eq, ns_fixpoint_violations

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_goldens.npz"))
VARIANTS = {
    "raster": dtb.generalised_distance_transform,
    "blocks": dtb.generalised_distance_transform_blocks,
    "task": dtb.generalised_distance_transform_task,
}


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


# ---------------------------------------------------------------------------------------------------
# ref-mode (reference weight, C8)
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("name", ["euclid", "geodesic"])
def test_reference_goldens(ctx, variant, name):
    img, mask, ref = GOLD[name + "_img"], GOLD[name + "_mask"], GOLD[name + "_ref"]
    d = VARIANTS[variant](cuda(img), cuda(mask), float(GOLD[name + "_lambda"]), ctx=ctx)
    assert_images_eq(d, ref, "%s %s" % (variant, name))


REF_SIZES = [(1, 1), (1, 37), (37, 1), (31, 33), (32, 32), (64, 64), (100, 300), (230, 250)]


def _ref_case(h, w, seed):
    rng = np.random.default_rng(seed)
    img = rng.integers(0, 256, (h, w), dtype=np.uint8)
    mask = np.zeros((h, w), np.uint8)
    mask[h // 2, w // 2] = 1
    for _ in range(2):
        mask[rng.integers(0, h), rng.integers(0, w)] = 1
    return img, mask


@pytest.mark.parametrize("h,w", REF_SIZES)
@pytest.mark.parametrize("lam", [0.0, 0.5, 1.0, 0.3])
def test_ref_random_vs_oracle(ctx, h, w, lam):
    img, mask = _ref_case(h, w, h * 1000 + w)
    ref = orc.ggdt_ref(img, mask, lam, fma=True)
    for variant in ("task", "blocks"):
        d = VARIANTS[variant](cuda(img), cuda(mask), lam, ctx=ctx)
        assert_images_eq(d, ref, "ref %s %dx%d lambda=%g" % (variant, w, h, lam))


@pytest.mark.parametrize("lam", [0.3, 0.77])
def test_ref_no_fma_vs_oracle(ctx, lam):
    img, mask = _ref_case(90, 70, 5)
    ref = orc.ggdt_ref(img, mask, lam, fma=False)
    d = dtb.generalised_distance_transform(cuda(img), cuda(mask), lam, ctx=ctx, fma=False)
    assert_images_eq(d, ref, "ref no-fma lambda=%g" % lam)


def test_ref_smooth_image_multi_seed(ctx):
    img = wl.blobs_gray(17, 200, 150)
    mask = wl.random_disks(np.random.default_rng(4), 200, 150, 6, 1, 4)
    ref = orc.ggdt_ref(img, mask, 0.5)
    assert_images_eq(dtb.generalised_distance_transform(cuda(img), cuda(mask), 0.5, ctx=ctx), ref, "ref blobs")


# ---------------------------------------------------------------------------------------------------
# ns-mode (C4, sqrt(1 + gamma^2 dI^2))
# ---------------------------------------------------------------------------------------------------
def _ns_check(ctx, img, mask, gamma, v=1e10, what="", rounds=(False, True)):
    ref = orc.ggdt_ns(img, mask, gamma, v=v)
    for r in rounds:
        d = dtb.geodesic_distance_transform(cuda(img), cuda(mask), gamma, v=v, rounds=r, ctx=ctx)
        assert_images_eq(d, ref, "%s rounds=%s" % (what, r))
    return ref


def test_ns_config0(ctx):
    img, mask, gamma = wl.config0()
    _ns_check(ctx, img, mask, gamma, what="config0")


@pytest.mark.parametrize("h,w", [(1, 1), (1, 50), (50, 1), (33, 65), (129, 97), (256, 256)])
@pytest.mark.parametrize("rgb", [False, True])
def test_ns_odd_sizes_random(ctx, h, w, rgb):
    rng = np.random.default_rng(h * 7 + w)
    img = rng.integers(0, 256, (h, w, 3) if rgb else (h, w), dtype=np.uint8)
    mask = np.zeros((h, w), np.uint8)
    mask[rng.integers(0, h), rng.integers(0, w)] = 1
    _ns_check(ctx, img, mask, 0.2, what="random %dx%d rgb=%s" % (w, h, rgb))


def test_ns_voronoi_rgb(ctx):
    img = wl.voronoi_rgb(21, 333, 250)
    mask = wl.random_disks(np.random.default_rng(9), 333, 250, 8, 5, 5)
    _ns_check(ctx, img, mask, 0.02, what="voronoi")


def test_ns_maze_crop(ctx):
    img, (sx, sy) = wl.maze_gray(31, 512, 512)
    mask = np.zeros(img.shape, np.uint8)
    mask[sy, sx] = 1
    _ns_check(ctx, img, mask, 0.5, what="maze 512")


def test_ns_no_seeds_all_v(ctx):
    img = wl.blobs_gray(3, 100, 70)
    mask = np.zeros(img.shape, np.uint8)
    d = dtb.geodesic_distance_transform(cuda(img), cuda(mask), 0.1, v=55.0, ctx=ctx)
    assert bool((d == 55.0).all())


def test_ns_all_seeds_zero(ctx):
    img = wl.blobs_gray(3, 70, 100)
    mask = np.ones(img.shape, np.uint8)
    d = dtb.geodesic_distance_transform(cuda(img), cuda(mask), 0.1, ctx=ctx)
    assert bool((d == 0).all())


def test_ns_corner_seeds_and_inf_v(ctx):
    img = wl.blobs_gray(8, 97, 131)
    mask = np.zeros(img.shape, np.uint8)
    mask[0, 0] = mask[-1, -1] = 1
    _ns_check(ctx, img, mask, 1.0, v=float("inf"), what="corners inf-v")


def test_ns_unaligned_pitch_is_staged(ctx):
    img = wl.blobs_gray(12, 37, 29)  # 37-byte rows: not TMA-aligned, staged by the library
    mask = np.zeros(img.shape, np.uint8)
    mask[3, 4] = 1
    _ns_check(ctx, img, mask, 0.3, what="unaligned", rounds=(False,))


def test_ns_padded_views(ctx):
    big = cuda(wl.blobs_gray(13, 160, 90))
    img = big[:, 16:144]  # pitch 160, offset 16 bytes: aligned sub-view
    mask = torch.zeros((90, 128), dtype=torch.uint8, device="cuda")
    mask[40, 60] = 1
    dist_big = torch.full((90, 200), -1.0, device="cuda")
    dist = dist_big[:, 8:136]
    dtb.geodesic_distance_transform(img, mask, 0.1, dist=dist, ctx=ctx)
    ref = orc.ggdt_ns(img.cpu().numpy(), mask.cpu().numpy(), 0.1)
    assert_images_eq(dist, ref, "padded view")
    assert bool((dist_big[:, :8] == -1).all()) and bool((dist_big[:, 136:] == -1).all())


def test_ns_host_buffers(ctx):
    img, mask, gamma = wl.config0(seed=5, w=300, h=200)
    dist = torch.empty((200, 300), dtype=torch.float32)
    dtb.geodesic_distance_transform(torch.from_numpy(img), torch.from_numpy(mask), gamma, dist=dist, ctx=ctx)
    assert_images_eq(dist, orc.ggdt_ns(img, mask, gamma), "host buffers")


def test_ns_repeated_calls_are_identical(ctx):
    img, mask, gamma = wl.config0(seed=6)
    a = dtb.geodesic_distance_transform(cuda(img), cuda(mask), gamma, ctx=ctx)
    for _ in range(3):
        b = dtb.geodesic_distance_transform(cuda(img), cuda(mask), gamma, ctx=ctx)
        assert_images_eq(b, a.cpu().numpy(), "repeat")


FP64_TOL = 1e-5  # stated bound on the relative error of the fp32 maps against exact-sum shortest paths


@pytest.mark.parametrize("which", ["config0", "config1", "config2"])
def test_ns_fp64_relative_error(ctx, which):
    """Max relative error of the GPU map against the FP64 Dijkstra on the same C4 graph, per configuration
    (512^2 gray blobs, 4096^2 gray maze, 8192^2 rgb8 Voronoi)."""
    img, mask, gamma = getattr(wl, which)()
    d = dtb.geodesic_distance_transform(cuda(img), cuda(mask), gamma, ctx=ctx).cpu().numpy().astype(np.float64)
    dj = orc.dijkstra_ns_f64(img, mask, gamma)
    sel = dj > 0
    rel = float((np.abs(d[sel] - dj[sel]) / dj[sel]).max())
    assert rel < FP64_TOL, rel


# ---------------------------------------------------------------------------------------------------
# ragged batch
# ---------------------------------------------------------------------------------------------------
def test_batch_vs_oracle_and_single(ctx):
    batch = wl.config3(seed=11, n=24, smin=16, smax=300)
    imgs = [cuda(i) for i, _, _ in batch]
    masks = [cuda(m) for _, m, _ in batch]
    gammas = [g for _, _, g in batch]
    dists = dtb.geodesic_distance_transform_batch(imgs, masks, gammas, ctx=ctx)
    for k, ((img, mask, g), d) in enumerate(zip(batch, dists)):
        assert_images_eq(d, orc.ggdt_ns(img, mask, g), "batch image %d %s" % (k, img.shape))
    st = ctx.stats()
    assert st["tiles"] == sum(((i.shape[0] + 31) // 32) * ((i.shape[1] + 31) // 32) for i, _, _ in batch)
    assert st["tile_visits"] >= 1 and st["device_error"] == 0
    plain = dtb.geodesic_distance_transform_batch(imgs, masks, gammas, rounds=True, ctx=ctx)
    for k, (a, b) in enumerate(zip(dists, plain)):
        assert_images_eq(b, a.cpu().numpy(), "plain per-image vs batch %d" % k)


def test_host_pipeline_many_chunks_padded_rows_and_empty_images():
    c = dtb.Context(0)
    c.set_tuning(host_chunk_kpx=24)  # ~24k pixels per chunk: many chunks, all overlapping
    batch = wl.config3(seed=13, n=17, smin=20, smax=240)
    imgs = [torch.from_numpy(i) for i, _, _ in batch]
    masks = [torch.from_numpy(m) for _, m, _ in batch]
    # a host image with padded rows (2-D copy path) and an empty image
    big = torch.from_numpy(np.ascontiguousarray(np.pad(batch[0][0], ((0, 0), (0, 5)) + (((0, 0),) if batch[0][0].ndim == 3 else ()))))
    imgs[0] = big[:, :batch[0][0].shape[1]]
    imgs.append(torch.zeros((0, 7), dtype=torch.uint8))
    masks.append(torch.zeros((0, 7), dtype=torch.uint8))
    gammas = [g for _, _, g in batch] + [0.1]
    dists = dtb.geodesic_distance_transform_batch(imgs, masks, gammas, ctx=c)
    assert c.stats()["rounds"] > 3  # chunks
    for k, (img, mask, g) in enumerate(batch):
        assert_images_eq(dists[k], orc.ggdt_ns(img, mask, g), "pipeline image %d" % k)
    assert dists[-1].shape == (0, 7)
    c.close()


@pytest.mark.parametrize("chunk_kpx", [16, 32768])
def test_host_pipeline_arena_runs(chunk_kpx):
    """Batch in one host arena per plane kind: adjacent packed planes move as one copy per chunk; odd widths put
    most planes off 16-byte boundaries (repitched on the device); small chunks split the runs; one image outside
    the arena breaks a run."""
    c = dtb.Context(0)
    c.set_tuning(host_chunk_kpx=chunk_kpx)
    rng = np.random.default_rng(21)
    batch = []
    for k in range(23):
        w, h = int(rng.integers(1, 180)), int(rng.integers(1, 150))
        img = wl.voronoi_rgb(k, w, h) if k % 3 == 0 else wl.blobs_gray(k, w, h)
        batch.append((img, wl.random_disks(rng, w, h, 2, 1, 4), float(rng.choice([0.01, 0.1, 1.0]))))
    iv, mv, dv = dtb.host_batch_arena([i for i, _, _ in batch], [m for _, m, _ in batch])
    iv[11] = torch.from_numpy(batch[11][0].copy())  # outside the arena: its own copy
    dtb.geodesic_distance_transform_batch(iv, mv, [g for _, _, g in batch], dists=dv, ctx=c)
    for k, (img, mask, g) in enumerate(batch):
        assert_images_eq(dv[k], orc.ggdt_ns(img, mask, g), "arena image %d" % k)
    if chunk_kpx == 16:
        assert c.stats()["rounds"] > 3
    c.close()


def test_host_pipeline_asynchronous_calls():
    """Back-to-back asynchronous host batches (a call's copies in overlap the previous call's copies out) and one
    dtb_sync for all of them; a stalled call among them is reported by that sync, and the context recovers."""
    c = dtb.Context(0)
    c.set_tuning(host_chunk_kpx=64)
    batches = [wl.config3(seed=30 + k, n=9, smin=20, smax=200) for k in range(3)]
    arenas = [dtb.host_batch_arena([i for i, _, _ in b], [m for _, m, _ in b]) for b in batches]
    for b, (iv, mv, dv) in zip(batches, arenas):
        dtb.geodesic_distance_transform_batch(iv, mv, [g for _, _, g in b], dists=dv, ctx=c, asynchronous=True)
    c.sync()
    for b, (_, _, dv) in zip(batches, arenas):
        for k, (img, mask, g) in enumerate(b):
            assert_images_eq(dv[k], orc.ggdt_ns(img, mask, g), "async batch image %d" % k)
    st = c.stats()
    assert st["tiles"] == sum(sum(((i.shape[0] + 31) // 32) * ((i.shape[1] + 31) // 32) for i, _, _ in b) for b in batches)
    # A stalled call in the middle: the sync raises; the next synchronous call is correct.
    iv, mv, dv = arenas[0]
    gam = [g for _, _, g in batches[0]]
    dtb.geodesic_distance_transform_batch(iv, mv, gam, dists=dv, ctx=c, asynchronous=True)
    c.inject_queue_stall(100)
    dtb.geodesic_distance_transform_batch(iv, mv, gam, dists=dv, ctx=c, asynchronous=True)
    with pytest.raises(dtb.DtbError) as e:
        c.sync()
    assert e.value.status == 4
    dtb.geodesic_distance_transform_batch(iv, mv, gam, dists=dv, ctx=c)
    for k, (img, mask, g) in enumerate(batches[0]):
        assert_images_eq(dv[k], orc.ggdt_ns(img, mask, g), "after stall, image %d" % k)
    c.close()


def test_host_pipeline_alternate_buffer_sets():
    """Successive host-buffer calls use alternate sets of device staging: calls of growing size (each set grows
    while the other may be in flight), with a device-resident call and a synchronous host call between
    asynchronous ones, all correct after one sync."""
    c = dtb.Context(0)
    c.set_tuning(host_chunk_kpx=32)
    batches = [wl.config3(seed=40 + k, n=5 + 3 * k, smin=16, smax=120 + 60 * k) for k in range(5)]
    arenas = [dtb.host_batch_arena([i for i, _, _ in b], [m for _, m, _ in b]) for b in batches]
    dev_batch = wl.config3(seed=49, n=4, smin=30, smax=150)
    dev_out = None
    for k, (b, (iv, mv, dv)) in enumerate(zip(batches, arenas)):
        sync_call = k == 3
        dtb.geodesic_distance_transform_batch(iv, mv, [g for _, _, g in b], dists=dv, ctx=c, asynchronous=not sync_call)
        if k == 1:
            dev_out = dtb.geodesic_distance_transform_batch([cuda(i) for i, _, _ in dev_batch],
                                                            [cuda(m) for _, m, _ in dev_batch],
                                                            [g for _, _, g in dev_batch], ctx=c)
    c.sync()
    for j, (b, (_, _, dv)) in enumerate(zip(batches, arenas)):
        for k, (img, mask, g) in enumerate(b):
            assert_images_eq(dv[k], orc.ggdt_ns(img, mask, g), "call %d image %d" % (j, k))
    for k, ((img, mask, g), d) in enumerate(zip(dev_batch, dev_out)):
        assert_images_eq(d, orc.ggdt_ns(img, mask, g), "device call image %d" % k)
    c.close()


def test_host_pipeline_reports_bytes_moved():
    """dtb_stats of a host-buffer batch counts the bytes copied each way: images and masks (plus the descriptor
    tables) in, maps out."""
    c = dtb.Context(0)
    c.set_tuning(host_chunk_kpx=256)
    batch = wl.config3(seed=42, n=12, smin=40, smax=400)
    imgs = [torch.from_numpy(i) for i, _, _ in batch]
    masks = [torch.from_numpy(m) for _, m, _ in batch]
    dists = dtb.geodesic_distance_transform_batch(imgs, masks, [g for _, _, g in batch], ctx=c)
    st = c.stats()
    planes_in = sum(i.numel() + m.numel() for i, m in zip(imgs, masks))
    assert planes_in < st["h2d_bytes"] < planes_in + (1 << 20)
    assert st["d2h_bytes"] == sum(d.numel() * 4 for d in dists)
    c.close()


def test_batch_host_buffers(ctx):
    batch = wl.config3(seed=12, n=6, smin=40, smax=200)
    dists = dtb.geodesic_distance_transform_batch([torch.from_numpy(i) for i, _, _ in batch],
                                                  [torch.from_numpy(m) for _, m, _ in batch],
                                                  [g for _, _, g in batch], ctx=ctx)
    for (img, mask, g), d in zip(batch, dists):
        assert not d.is_cuda
        assert_images_eq(d, orc.ggdt_ns(img, mask, g), "batch host")


# ---------------------------------------------------------------------------------------------------
# full-size configurations: exact fixpoint characterisation (size independent)
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("which", ["config1", "config2"])
def test_full_size_fixpoint(ctx, which):
    img, mask, gamma = getattr(wl, which)()
    ti, tm = cuda(img), cuda(mask)
    d = dtb.geodesic_distance_transform(ti, tm, gamma, ctx=ctx)
    va, vb, dmax = ns_fixpoint_violations(ti, tm, gamma, 1e10, d)
    assert dmax < 2 ** 23, dmax
    assert va == 0 and vb == 0, (va, vb)
    assert ctx.stats()["device_error"] == 0


def test_pitched_allocation_layout():
    t = dtb.pitched_empty(5, 37, 3)
    assert t.shape == (5, 37, 3) and t.stride() == (128, 3, 1)
    f = dtb.pitched_empty(4, 33, 1, torch.float32)
    assert f.stride() == (64, 1)  # 33 floats -> 256-byte rows


def test_plan_rejects_unaligned_buffers(ctx):
    img = torch.zeros((10, 37), dtype=torch.uint8, device="cuda")  # 37-byte pitch
    with pytest.raises(dtb.DtbError):
        dtb.BatchPlan([img], [img.clone()], [0.1], ctx=ctx)


# ---------------------------------------------------------------------------------------------------
# batch plans (CUDA graph) and the autotuner
# ---------------------------------------------------------------------------------------------------
def test_plan_graph_runs_match_oracle_and_autotune_keeps_results(ctx):
    batch = wl.config3(seed=21, n=20, smin=24, smax=260)
    imgs = [dtb.pitched_from(i) for i, _, _ in batch]
    masks = [dtb.pitched_from(m) for _, m, _ in batch]
    dists = [dtb.pitched_empty(i.shape[0], i.shape[1], 1, torch.float32).fill_(-1.0) for i, _, _ in batch]
    plan = dtb.BatchPlan(imgs, masks, [g for _, _, g in batch], dists=dists, ctx=ctx)
    refs = [orc.ggdt_ns(i, m, g) for i, m, g in batch]
    for run in range(2):
        for d in dists:
            d.fill_(-1.0)
        plan.run()
        st = plan.wait()
        assert st["device_error"] == 0 and st["tile_visits"] >= 1
        for k, (d, ref) in enumerate(zip(dists, refs)):
            assert_images_eq(d, ref, "plan run %d image %d" % (run, k))
    chosen = plan.autotune(reps=1)
    assert (chosen["ctas_per_sm"], chosen["warps_per_cta"]) in SHAPES and 1 <= chosen["grid_percent"] <= 100
    for d in dists:
        d.fill_(-1.0)
    plan.run()
    plan.wait()
    for k, (d, ref) in enumerate(zip(dists, refs)):
        assert_images_eq(d, ref, "tuned plan image %d" % k)
    plan.close()


SHAPES = {(2, 4), (3, 4), (4, 4), (6, 2), (2, 6), (2, 8)}  # (CTAs per SM, warps per CTA) of the tile kernel

TUNINGS = [  # (ctas_per_sm, grid_percent, staging, queue_buckets, bucket_width_pct, warps_per_cta)
    (3, 100, 1, 8, 50, 4), (4, 50, 1, 8, 50, 4), (2, 25, 1, 8, 50, 4),    # launch shapes, self-staging visits
    (6, 100, 1, 8, 25, 2), (2, 100, 1, 8, 25, 6), (2, 60, 1, 1, 50, 8),   # other warps per CTA
    (3, 100, 2, 8, 50, 4), (2, 75, 2, 16, 25, 4),                         # next tile staged ahead
    (3, 100, 1, 1, 50, 4), (3, 100, 2, 1, 50, 4),                         # FIFO queue
    (3, 100, 1, 16, 100, 4), (3, 100, 2, 2, 400, 4), (3, 100, 2, 4, 1, 4),  # bucket counts and widths
]


@pytest.mark.parametrize("ctas,pct,staging,buckets,width,wpc", TUNINGS)
def test_every_tuning_gives_the_same_map(ctas, pct, staging, buckets, width, wpc):
    """Launch shape, staging and queue policy change the visit order only: every one gives the oracle's map,
    on a single image and on a ragged batch (gray and rgb8, seeds in several tiles)."""
    c = dtb.Context(0)
    c.set_tuning(ctas_per_sm=ctas, grid_percent=pct, staging=staging, queue_buckets=buckets, bucket_width_pct=width,
                 warps_per_cta=wpc)
    assert c.get_tuning() == {"ctas_per_sm": ctas, "grid_percent": pct, "host_chunk_kpx": 16384,
                              "queue_buckets": buckets, "bucket_width_pct": width, "staging": staging,
                              "warps_per_cta": wpc}
    img, mask, gamma = wl.config0(seed=9)
    d = dtb.geodesic_distance_transform(cuda(img), cuda(mask), gamma, ctx=c)
    what = "tuning %s" % ((ctas, pct, staging, buckets, width, wpc),)
    assert_images_eq(d, orc.ggdt_ns(img, mask, gamma), what)
    batch = wl.config3(seed=31, n=20, smin=48, smax=700)
    dists = dtb.geodesic_distance_transform_batch([cuda(i) for i, _, _ in batch], [cuda(m) for _, m, _ in batch],
                                                  [g for _, _, g in batch], ctx=c)
    for k, ((i, m, g), dk) in enumerate(zip(batch, dists)):
        assert_images_eq(dk, orc.ggdt_ns(i, m, g), "%s batch image %d" % (what, k))
    assert c.stats()["device_error"] == 0
    c.close()


def test_invalid_tunings_are_rejected():
    c = dtb.Context(0)
    for kw in ({"ctas_per_sm": 4, "staging": 2}, {"ctas_per_sm": 5}, {"queue_buckets": 3}, {"queue_buckets": 32},
               {"bucket_width_pct": 6401}, {"staging": 3}, {"grid_percent": 101}, {"warps_per_cta": 3},
               {"ctas_per_sm": 3, "warps_per_cta": 8}, {"ctas_per_sm": 6, "warps_per_cta": 2, "staging": 2}):
        with pytest.raises(dtb.DtbError):
            c.set_tuning(**kw)
    c.close()


def test_autotuner_cache_round_trip(tmp_path):
    """dtb_plan_autotune writes its choice to the JSON cache; a new context that loads the cache starts plans
    of the same size class from it."""
    import json
    path = tmp_path / "autotune.json"
    batch = wl.config3(seed=41, n=12, smin=64, smax=400)
    imgs = [dtb.pitched_from(i) for i, _, _ in batch]  # plans take TMA-aligned device rows
    masks = [dtb.pitched_from(m) for _, m, _ in batch]
    gammas = [g for _, _, g in batch]
    c = dtb.Context(0)
    c.set_tuning_cache(path)
    plan = dtb.BatchPlan(imgs, masks, gammas, ctx=c)
    chosen = plan.autotune(reps=1)
    plan.run()
    plan.wait()
    for k, (i, m, g) in enumerate(batch):
        assert_images_eq(plan.dists[k], orc.ggdt_ns(i, m, g), "autotuned image %d" % k)
    plan.close()
    c.close()
    doc = json.loads(path.read_text())
    assert doc["format"] == "dtb-autotune-1" and len(doc["entries"]) == 1
    e = doc["entries"][0]
    assert e["gpu"] == torch.cuda.get_device_name(0)
    assert {k: e[k] for k in chosen if k != "host_chunk_kpx"} == {k: v for k, v in chosen.items() if k != "host_chunk_kpx"}
    c2 = dtb.Context(0)
    c2.set_tuning_cache(path)
    plan2 = dtb.BatchPlan(imgs, masks, gammas, ctx=c2)
    assert plan2.tuning() == chosen
    plan2.close()
    c2.close()


def test_staged_ahead_batch_runs_are_bit_identical_under_load():
    """The staged-ahead kernel under load: a tile popped ahead is claimed only when its visit starts, so an
    activation that reaches it while it waits must still be covered.  Repeated full-grid runs of a ragged batch,
    each compared with the first, the first with the oracle."""
    c = dtb.Context(0)
    c.set_tuning(ctas_per_sm=3, staging=2, grid_percent=100)
    batch = wl.config3(seed=23, n=120, smin=64, smax=1536)
    imgs = [cuda(i) for i, _, _ in batch]
    masks = [cuda(m) for _, m, _ in batch]
    gammas = [g for _, _, g in batch]
    dists = dtb.geodesic_distance_transform_batch(imgs, masks, gammas, ctx=c)
    for k in range(0, len(batch), 6):
        img, mask, g = batch[k]
        assert_images_eq(dists[k], orc.ggdt_ns(img, mask, g), "ahead batch image %d %s" % (k, img.shape))
    first = torch.cat([d.flatten() for d in dists])
    for rep in range(30):
        dtb.geodesic_distance_transform_batch(imgs, masks, gammas, dists=dists, ctx=c)
        assert torch.equal(torch.cat([d.flatten() for d in dists]), first), rep
    assert c.stats()["device_error"] == 0
    c.close()


# ---------------------------------------------------------------------------------------------------
# concurrency: the fixpoint does not depend on the visit order, so every run is bit-identical
# ---------------------------------------------------------------------------------------------------
def test_batch_runs_are_bit_identical_under_load(ctx):
    """Many full-grid runs of a ragged batch: a lost wake-up between concurrently visited neighbour tiles
    (e.g. an activation seen before the activating tile's VISITED bit) leaves a few pixels above the
    fixpoint in a rare run, so each run is compared with the first, and the first with the oracle."""
    batch = wl.config3(seed=21, n=160, smin=64, smax=1536)
    imgs = [cuda(i) for i, _, _ in batch]
    masks = [cuda(m) for _, m, _ in batch]
    gammas = [g for _, _, g in batch]
    dists = dtb.geodesic_distance_transform_batch(imgs, masks, gammas, ctx=ctx)
    for k in range(0, len(batch), 8):
        img, mask, g = batch[k]
        assert_images_eq(dists[k], orc.ggdt_ns(img, mask, g), "batch image %d %s" % (k, img.shape))
    first = torch.cat([d.flatten() for d in dists])
    bad = []
    for rep in range(60):
        dtb.geodesic_distance_transform_batch(imgs, masks, gammas, dists=dists, ctx=ctx)
        if not torch.equal(torch.cat([d.flatten() for d in dists]), first):
            off = 0
            for k, d in enumerate(dists):
                n = d.numel()
                if not torch.equal(d.flatten(), first[off:off + n]):
                    va, vb, _ = ns_fixpoint_violations(imgs[k], masks[k], gammas[k], 1e10, d)
                    bad.append((rep, k, int((d.flatten() != first[off:off + n]).sum()), va, vb))
                off += n
    assert not bad, bad[:8]
    assert ctx.stats()["device_error"] == 0


def test_ref_runs_are_bit_identical_under_load(ctx):
    img, mask = _ref_case(2048, 2048, 22)
    ti, tm = cuda(img), cuda(mask)
    a = dtb.generalised_distance_transform(ti, tm, 0.5, ctx=ctx)
    assert_images_eq(a, orc.ggdt_ref(img, mask, 0.5), "ref 2048")
    d = torch.empty_like(a)
    for rep in range(30):
        dtb.generalised_distance_transform(ti, tm, 0.5, dist=d, ctx=ctx)
        assert torch.equal(d, a), (rep, int((d != a).sum()))


@pytest.mark.parametrize("kind,h,w,gamma", [("gray", 2048, 1536, 0.0), ("rgb8", 1500, 2100, 0.0),
                                            ("const", 4096, 4096, 1.0)])
def test_ns_unit_weights_are_city_block_distance(ctx, kind, h, w, gamma):
    """Oracle-free check at sizes the CPU restatement is slow on: with every C4 edge weighing exactly 1
    (gamma = 0, or an image without intensity steps) the map is the integer city-block distance to the nearest
    seed, which scipy computes independently."""
    from scipy import ndimage
    rng = np.random.default_rng(17)
    if kind == "const":
        img = np.full((h, w), 77, np.uint8)
    elif kind == "gray":
        img = rng.integers(0, 256, (h, w), dtype=np.uint8)
    else:
        img = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    mask = wl.random_disks(rng, w, h, 5, 1, 6)
    d = dtb.geodesic_distance_transform(cuda(img), cuda(mask), gamma, ctx=ctx)
    expect = ndimage.distance_transform_cdt(mask == 0, metric="taxicab").astype(np.float32)
    assert_images_eq(d, expect, "unit weights, %s %dx%d" % (kind, h, w))


@pytest.mark.parametrize("which", ["config1", "config2"])
def test_full_size_union_of_seed_sets_is_elementwise_min(ctx, which):
    """The map is the minimum, over paths from any seed, of the path's fp32 sum, and a path's sum does not depend
    on which other seeds exist: T(A | B) == min(T(A), T(B)) bit for bit, at the full sizes of the 4096^2 maze
    and the 8192^2 rgb8 workload."""
    img, mask_a, gamma = getattr(wl, which)()
    h, w = mask_a.shape
    mask_b = wl.random_disks(np.random.default_rng(23), w, h, 7, 2, 6)
    ti = cuda(img)
    da = dtb.geodesic_distance_transform(ti, cuda(mask_a), gamma, ctx=ctx)
    db = dtb.geodesic_distance_transform(ti, cuda(mask_b), gamma, ctx=ctx)
    du = dtb.geodesic_distance_transform(ti, cuda(mask_a | mask_b), gamma, ctx=ctx)
    expect = torch.minimum(da, db)
    assert torch.equal(du, expect), int((du != expect).sum())
    assert ctx.stats()["device_error"] == 0


@pytest.mark.parametrize("lam", [0.0, 0.5, 1.0])
def test_ref_union_of_seed_sets_is_elementwise_min_full_size(ctx, lam):
    """ref-mode at the reference benchmark's image size (3648 x 2432 gray): T(A | B) == min(T(A), T(B))."""
    rng = np.random.default_rng(29)
    h, w = 2432, 3648
    img = cuda(wl.blobs_gray(31, w, h))
    a = cuda(wl.random_disks(rng, w, h, 8, 2, 6))
    b = cuda(wl.random_disks(rng, w, h, 5, 2, 6))
    da = dtb.generalised_distance_transform(img, a, lam, ctx=ctx)
    db = dtb.generalised_distance_transform(img, b, lam, ctx=ctx)
    du = dtb.generalised_distance_transform(img, a | b, lam, ctx=ctx)
    expect = torch.minimum(da, db)
    assert torch.equal(du, expect), int((du != expect).sum())
