#!/usr/bin/env python
"""Benchmark: converged GGDT Mpixel/s on the ragged batch (1024 images, sides log-uniform in [64, 2048],
half gray blobs / half rgb8 Voronoi, 1-8 seed disks, gamma in {0.01, 0.1, 1.0}), one persistent launch per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  Under torchrun every rank processes its own batch (different seed, no data-path
collective: images are independent), so per-GPU work is fixed (weak scaling); the step time is the max over
ranks.  `value` times the batch on device-resident inputs; `e2e` times the same call through the C ABI with
pinned host buffers (host->device copies of images and masks and the device->host copy of the distance
maps inside the timed region).  `--impl reference` times the CPU restatement of the reference algorithm
(the reference has no CPU implementation of this path) on the host cores.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged GGDT Mpixel/s, batched vs per-image on one B200; serve p50/p99 ms"
UNIT = "Mpixel/s"
PLAIN_SUBSET = 64          # images of the batch timed through the plain per-image path
REF_STEP_MPX = 24.0        # CPU legs (reference arm, cpu_baseline): pixels of the stratified sample per step
PARITY_LARGE = 16          # oracle parity sample: images of the batch with a side >= 1536 ...
PARITY_SPREAD = 16         # ... plus images at evenly spaced size quantiles
FP64_TOL = 1e-5            # stated bound on the relative error against the FP64 Dijkstra


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--images", type=int, default=1024)
    p.add_argument("--seed", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--serve-requests", type=int, default=5000)
    p.add_argument("--serve-rate", type=float, default=500.0, help="Poisson arrival rate (requests / s)")
    p.add_argument("--serve-saturated", type=int, default=1000,
                   help="requests of the same mix submitted at once after the paced phase (capacity)")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-ref-mode", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the single-image C0 / C1 / C2 leg")
    p.add_argument("--ref-mpx", type=float, default=REF_STEP_MPX, help="reference arm: pixels per step (millions)")
    return p.parse_args()


# ---------------------------------------------------------------------------------------------------------
# distributed plumbing (timing only: the max of the step times over ranks)
# ---------------------------------------------------------------------------------------------------------
from distance_transform_benchmarks_b200.replicas import ReplicaGroup as Dist  # noqa: E402


# ---------------------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.proc = None
        self.path = None
        try:
            uuid = str(torch.cuda.get_device_properties(device).uuid)
            self.sel = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            self.sel = str(device)

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.sel, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.15)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic_bytes_per_px():
    """DRAM bytes per pixel of the tile kernel from the committed ncu summary (a smaller capture of the same
    workload, scaled by pixels), or None."""
    path = os.path.join(ROOT, "profiles", "ggdt_persistent_batch.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_pixel:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------------------------------------
def link_floor(h2d, d2h, e2e_ms, nchunks):
    """The host link's own time for one e2e step, copies only, pinned memory, CUDA events: the step's h2d bytes
    in and d2h bytes out concurrently on two streams as one copy each way (copy_floor_ms), as `nchunks` copies
    each way like the host-buffer pipeline (chunked_copy_floor_ms), and with chunk k's copy out waiting for
    chunk k + 2's copy in, a stand-in for the tile runs between them (pipelined_copy_floor_ms); and each
    direction alone."""
    hin = torch.empty(h2d, dtype=torch.uint8).pin_memory()
    hout = torch.empty(d2h, dtype=torch.uint8).pin_memory()
    din = torch.empty(h2d, dtype=torch.uint8, device="cuda")
    dout = torch.empty(d2h, dtype=torch.uint8, device="cuda")
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    n = max(1, nchunks)
    ci = [(k * h2d // n, (k + 1) * h2d // n) for k in range(n)]
    co = [(k * d2h // n, (k + 1) * d2h // n) for k in range(n)]

    def timed(do_in, do_out, reps=3, chunks=1, lag=None):
        best = None
        for _ in range(reps):
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            torch.cuda.synchronize()
            a.record(s_in)
            s_out.wait_event(a)
            if chunks == 1:
                if do_in:
                    with torch.cuda.stream(s_in):
                        din.copy_(hin, non_blocking=True)
                if do_out:
                    with torch.cuda.stream(s_out):
                        hout.copy_(dout, non_blocking=True)
            elif lag is None:
                for (x, y), (u, v) in zip(ci, co):
                    with torch.cuda.stream(s_in):
                        din[x:y].copy_(hin[x:y], non_blocking=True)
                    with torch.cuda.stream(s_out):
                        hout[u:v].copy_(dout[u:v], non_blocking=True)
            else:
                ev = []
                for x, y in ci:
                    with torch.cuda.stream(s_in):
                        din[x:y].copy_(hin[x:y], non_blocking=True)
                    e = torch.cuda.Event()
                    e.record(s_in)
                    ev.append(e)
                for k, (u, v) in enumerate(co):
                    s_out.wait_event(ev[min(k + lag, n - 1)])
                    with torch.cuda.stream(s_out):
                        hout[u:v].copy_(dout[u:v], non_blocking=True)
            b.record(s_out)
            s_in.wait_event(b)
            c.record(s_in)
            torch.cuda.synchronize()
            t = a.elapsed_time(c)
            best = t if best is None else min(best, t)
        return best

    both = timed(True, True)
    chunked = timed(True, True, chunks=n)
    lagged = timed(True, True, chunks=n, lag=2)
    t_in = timed(True, False)
    t_out = timed(False, True)
    return {"copy_floor_ms": both, "frac": both / e2e_ms, "chunks": n, "chunked_copy_floor_ms": chunked,
            "pipelined_copy_floor_ms": lagged, "frac_of_pipelined": lagged / e2e_ms,
            "h2d_alone_gbs": h2d / t_in / 1e6, "d2h_alone_gbs": d2h / t_out / 1e6, "e2e_d2h_gbs": d2h / e2e_ms / 1e6,
            "note": "copies only, pinned, concurrent in/out: one copy per direction; the pipeline's chunk count; "
                    "and chunk k out after chunk k+2 in"}


def bench_config(args, specs):
    """The `config` object of the JSON line: the same dict in both arms (the workload, not how an arm samples
    it)."""
    return {"workload": "ragged batch of %d images per GPU, sides log-U[64,2048], half gray blobs / half rgb8 "
                        "Voronoi, 1-8 seed disks r 2-6, gamma in {0.01,0.1,1.0}, seed %d" % (args.images, args.seed),
            "pixels_per_gpu": int(sum(s[1] * s[2] for s in specs)), "parallelism": "replicas (independent images "
            "per rank)", "l2": "inputs larger than L2 (no flush needed)"}


def sample_desc(idx, specs):
    px = sum(specs[i][1] * specs[i][2] for i in idx)
    stride = idx[1] - idx[0] if len(idx) > 1 else 1
    return "every %d-th image of the batch (%d images, %.1f Mpx, gray and rgb8 alternating)" % (stride, len(idx),
                                                                                                  px / 1e6), px


def parity_indices(specs):
    """The oracle parity sample: the first PARITY_LARGE images with a side >= 1536 and PARITY_SPREAD images at
    evenly spaced quantiles of the pixel count."""
    large = [i for i, s in enumerate(specs) if max(s[1], s[2]) >= 1536][:PARITY_LARGE]
    order = sorted(range(len(specs)), key=lambda i: specs[i][1] * specs[i][2])
    spread = [order[int(round(q * (len(order) - 1) / max(1, PARITY_SPREAD - 1)))] for q in range(PARITY_SPREAD)]
    return sorted(set(large) | set(spread))


def cpu_legs(batch, specs, sample_idx, maps, config_maps):
    """The CPU legs, rank 0 of a one-GPU run: the oracle (CPU restatement of the reference raster algorithm) on
    the host cores, timed on the reference arm's stratified sample; the same oracle as the bit-exact checker of
    the GPU maps of that sample and of the parity sample; and the FP64 Dijkstra as the accuracy bound per
    configuration.  `maps[i]`: the GPU map of batch image i (host numpy); `config_maps`: name -> (img, mask,
    gamma, GPU map) of the single-image configurations.  Returns (cpu_baseline, parity)."""
    from oracle import oracle as orc
    desc, px = sample_desc(sample_idx, specs)
    mism = {}
    t_oracle = 0.0
    for i in sample_idx:
        img, mask, g = batch[i]
        t0 = time.perf_counter()
        ref = orc.ggdt_ns(img, mask, g)
        t_oracle += time.perf_counter() - t0
        mism[i] = int(np.count_nonzero(ref.view(np.uint32) != maps[i].view(np.uint32)))
    out = {"value": px / t_oracle / 1e6, "unit": UNIT, "cores": orc.max_threads(), "kind": "port",
           "sample": desc + ", %.1f s" % t_oracle}
    sample = [batch[i] for i in sample_idx]

    def rate(fn, seconds):
        px, t0 = 0, time.perf_counter()
        for img, mask, g in sample:
            fn(img, mask, g)
            px += img.shape[0] * img.shape[1]
            if time.perf_counter() - t0 > seconds:
                break
        return px / (time.perf_counter() - t0) / 1e6

    # For information (same images, a few seconds each): one host thread, the FP64 Dijkstra on the same graph
    # (one thread), and the reference weight (C8, lambda 0.5; the raster restatement is single-threaded).
    out["single_thread_mpx_s"] = rate(lambda i, m, g: orc.ggdt_ns(i, m, g, nthreads=1), 3.0)
    out["dijkstra_f64_mpx_s"] = rate(lambda i, m, g: orc.dijkstra_ns_f64(i, m, g), 3.0)
    gray = [(i, m, g) for i, m, g in sample if i.ndim == 2]
    px_r, t0 = 0, time.perf_counter()
    for img, mask, _ in gray:
        orc.ggdt_ref(img, mask, 0.5)
        px_r += img.size
        if time.perf_counter() - t0 > 3.0:
            break
    out["ref_mode_lambda05_single_thread_mpx_s"] = px_r / (time.perf_counter() - t0) / 1e6

    # Parity: the oracle sample (large and size-spread images) beside the stratified one.
    extra = [i for i in parity_indices(specs) if i not in mism]
    for i in extra:
        img, mask, g = batch[i]
        mism[i] = int(np.count_nonzero(orc.ggdt_ns(img, mask, g).view(np.uint32) != maps[i].view(np.uint32)))
    checked = sorted(mism)

    def rel64(img, mask, g, d32):
        d64 = orc.dijkstra_ns_f64(img, mask, g)
        sel = d64 > 0
        return float((np.abs(d32[sel].astype(np.float64) - d64[sel]) / d64[sel]).max()) if sel.any() else 0.0

    fp64 = {name: rel64(*cm) for name, cm in config_maps.items()}
    fp64["C3_first64"] = max(rel64(*batch[i], maps[i]) for i in range(min(64, len(batch))))
    parity = {"oracle_images": len(checked),
              "oracle_images_side_ge_1536": sum(1 for i in checked if max(specs[i][1], specs[i][2]) >= 1536),
              "oracle_pixels": int(sum(specs[i][1] * specs[i][2] for i in checked)),
              "oracle_mismatches": int(sum(mism.values())),
              "oracle_sample": "the cpu_baseline sample, the first %d images with a side >= 1536 and %d images at "
                               "evenly spaced size quantiles; bit-exact comparison" % (PARITY_LARGE, PARITY_SPREAD),
              "fp64_max_rel": fp64, "fp64_tol": FP64_TOL,
              "fp64_within_tol": all(v < FP64_TOL for v in fp64.values())}
    return out, parity


SERVE_POOL = 48                 # distinct synthetic images behind the new-image requests
SERVE_BUDGET = 120 << 30        # device-memory budget of the serving engine (bytes)


# The reference's own benchmark (benchmarks/distance_transform.cpp): reference weight (C8, lambda blend) on
# ~8.9 Mpx gray photographs, lambda in {0, 0.5, 1}, one call per image timed whole (allocation and setup
# included).  Published throughput on its (unrecorded) GPU, Mpixel/s: raster 55.8 / 28.0 / 25.1, blocks
# 375 / 324 / 323, task 613 / 555 / 560 for lambda 0 / 0.5 / 1.  The photographs are not available: a seeded
# 3648 x 2432 (8.87 Mpx) gray blob image with 8 seed disks stands in for them.
REF_MODE_W, REF_MODE_H = 3648, 2432
REF_PUBLISHED = {"raster": [55.8, 28.0, 25.1], "blocks": [375.0, 324.0, 323.0], "task": [613.0, 555.0, 560.0]}


def run_ref_mode(args, ctx, stream):
    import distance_transform_benchmarks_b200 as dtb
    from distance_transform_benchmarks_b200 import workloads as wl
    img = wl.blobs_gray(args.seed + 77, REF_MODE_W, REF_MODE_H)
    mask = wl.random_disks(np.random.default_rng(args.seed + 78), REF_MODE_W, REF_MODE_H, 8, 2, 6)
    ti, tm = torch.from_numpy(img).cuda(), torch.from_numpy(mask).cuda()
    px = REF_MODE_W * REF_MODE_H
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {}
    variants = (("task", dtb.generalised_distance_transform_task), ("blocks", dtb.generalised_distance_transform_blocks))
    for name, fn in variants:
        vals = []
        for lam in (0.0, 0.5, 1.0):
            fn(ti, tm, lam, ctx=ctx, stream=stream)  # warm-up (scratch growth, module load)
            reps = 3
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(reps):
                fn(ti, tm, lam, ctx=ctx, stream=stream)  # allocating call, as the reference benchmark times it
            e1.record(stream)
            torch.cuda.synchronize()
            vals.append(px / 1e6 / (e0.elapsed_time(e1) / reps / 1e3))
        out[name] = vals
    return {"image": "%dx%d gray blobs, 8 seed disks r 2-6 (stands in for the reference's ~8.9 Mpx photographs)"
                     % (REF_MODE_W, REF_MODE_H),
            "lambdas": [0.0, 0.5, 1.0], "mpx_s": out, "unit": UNIT,
            "reference_published_mpx_s": REF_PUBLISHED,
            "note": "whole call timed on the stream (allocation + setup + transform), inputs resident on the device; "
                    "task = persistent tile queue (the raster variant returns the same map through the same path)"}


def run_configs(ctx, stream):
    """The single-image configurations, inputs resident on the device, one call each (3 timed): C0 (512^2 gray
    blobs), C1 (4096^2 gray maze: the worst case for raster passes, paths wind through the whole image) and C2
    (8192^2 rgb8 Voronoi), with the tile visits and sweep phases behind each figure.  Returns the figures and,
    per configuration, (img, mask, gamma, map) for the FP64 error of the CPU legs."""
    import distance_transform_benchmarks_b200 as dtb
    from distance_transform_benchmarks_b200 import workloads as wl
    out, maps = {}, {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, gen in (("C0", wl.config0), ("C1", wl.config1), ("C2", wl.config2)):
        img, mask, gamma = gen()
        ti, tm = dtb.pitched_from(img), dtb.pitched_from(mask)
        d = dtb.pitched_empty(img.shape[0], img.shape[1], 1, torch.float32)
        dtb.geodesic_distance_transform(ti, tm, gamma, dist=d, ctx=ctx, stream=stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            dtb.geodesic_distance_transform(ti, tm, gamma, dist=d, ctx=ctx, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        st = ctx.stats()
        out[name] = {"shape": list(img.shape), "ms": ms, "mpx_s": img.shape[0] * img.shape[1] / 1e3 / ms,
                     "visits_per_tile": st["tile_visits"] / max(1, st["tiles"]),
                     "phases_per_visit": st["phases"] / max(1, st["tile_visits"]),
                     "activations_per_tile": st["activations"] / max(1, st["tiles"])}
        maps[name] = (img, mask, gamma, d.cpu().numpy())
        del ti, tm, d
    return out, maps


def serve_pool():
    """The serving workload's images: sides log-uniform in [256, 4096], gray blobs or rgb8 Voronoi, 1-8 seed
    disks, pinned host buffers (an output map per image, shared by its requests)."""
    import math
    from distance_transform_benchmarks_b200 import workloads as wl

    rng = np.random.default_rng(4)
    pool = []
    for i in range(SERVE_POOL):
        w = int(round(math.exp(rng.uniform(math.log(256), math.log(4096)))))
        h = int(round(math.exp(rng.uniform(math.log(256), math.log(4096)))))
        g = float(np.float32(rng.choice([0.01, 0.1, 1.0])))
        img, mask, g = wl.make_image(("gray" if i % 2 == 0 else "rgb8", w, h, g, 1000 + i))
        out = torch.empty((h, w), dtype=torch.float32).pin_memory()  # shared by the pool image's requests
        pool.append((torch.from_numpy(img).pin_memory(), torch.from_numpy(mask).pin_memory(), g, out))
    return pool


def run_serve(args, dev, pool, live=False):
    """Serving workload: Poisson arrivals; 60 % new images (the pool's), 40 % seed edits (1-3 disks of radius 3)
    of a resident image, warm-started from its map.  Latency is measured by the engine from submit to the map
    being in host memory.  live: requests join the tile queue of one running kernel instead of waves (the same
    request stream, seeded alike)."""
    import distance_transform_benchmarks_b200 as dtb

    rng = np.random.default_rng(5)
    srv = dtb.Server(SERVE_BUDGET, device=dev, live=live)
    n = args.serve_requests
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n))
    kinds = rng.random(n) < 0.6
    created = []       # image ids created so far
    pool_of = {}
    next_id = 0

    def submit(new_image):
        """One request of the mix; returns its pixels."""
        nonlocal next_id
        if new_image or not created:
            p = next_id % SERVE_POOL
            img, mask, g, out = pool[p]
            srv.submit_image(next_id, img, mask, g, out)
            created.append(next_id)
            pool_of[next_id] = p
            next_id += 1
        else:
            iid = created[int(rng.integers(max(0, len(created) - 256), len(created)))]
            img, _, _, out = pool[pool_of[iid]]
            hh, ww = img.shape[:2]
            disks = [(int(rng.integers(0, ww)), int(rng.integers(0, hh)), 3) for _ in range(int(rng.integers(1, 4)))]
            srv.submit_edit(iid, disks, out)
        return int(img.shape[0]) * int(img.shape[1])

    def drain(lat, count, deadline):
        while len(lat) < count:
            for c in srv.poll(wait_ms=100):
                lat.append(c["latency_ms"])
            if time.perf_counter() > deadline:
                break

    lat, px, submitted = [], 0, 0
    t0 = time.perf_counter()
    for k in range(n):
        while time.perf_counter() - t0 < arrivals[k]:
            for c in srv.poll(wait_ms=0):
                lat.append(c["latency_ms"])
            time.sleep(0.0002)
        px += submit(kinds[k])
        submitted += 1
    drain(lat, submitted, t0 + arrivals[-1] + 120)
    elapsed = time.perf_counter() - t0
    st = srv.stats()

    def phases(a, b):
        """Where the time of the waves between stats a and b went (per wave: host preparation, copies in, tile
        run, copies out on their streams; per request: queueing before its wave's preparation).  Live engine:
        per request, host clock: publish, publish to its completion word (copy in + tile work), copy out;
        "waves" counts kernel launches."""
        r = max(1, b["completed"] - a["completed"])
        if live:
            return {"launches": int(b["waves"] - a["waves"]),
                    "launch_ends": {k: int(b["live_ended_" + k] - a["live_ended_" + k])
                                    for k in ("idle", "lifetime", "error", "stop")},
                    "host_prep_ms_per_request": (b["host_prep_ms"] - a["host_prep_ms"]) / r,
                    "in_and_kernel_ms_per_request": (b["kernel_ms"] - a["kernel_ms"]) / r,
                    "copy_out_ms_per_request": (b["copy_out_ms"] - a["copy_out_ms"]) / r,
                    "queue_wait_mean_ms": (b["queue_wait_ms"] - a["queue_wait_ms"]) / r,
                    "queue_wait_max_ms": b["queue_wait_max_ms"],
                    "tile_visits_per_tile": (b["tile_visits"] - a["tile_visits"]) / max(1, b["tiles"] - a["tiles"])}
        w = max(1, b["waves"] - a["waves"])
        return {"waves": int(b["waves"] - a["waves"]), "waves_split": int(b["waves_split"] - a["waves_split"]),
                "host_prep_ms_per_wave": (b["host_prep_ms"] - a["host_prep_ms"]) / w,
                "copy_in_ms_per_wave": (b["copy_in_ms"] - a["copy_in_ms"]) / w,
                "kernel_ms_per_wave": (b["kernel_ms"] - a["kernel_ms"]) / w,
                "copy_out_ms_per_wave": (b["copy_out_ms"] - a["copy_out_ms"]) / w,
                "queue_wait_mean_ms": (b["queue_wait_ms"] - a["queue_wait_ms"]) / r,
                "queue_wait_max_ms": b["queue_wait_max_ms"]}

    zero = {k: 0 for k in st}
    # Saturated phase: the same mix submitted at once; throughput = the engine's capacity.
    ns = args.serve_saturated
    saturated = None
    if ns > 0:
        lat2, px2 = [], 0
        t1 = time.perf_counter()
        for k in range(ns):
            px2 += submit(rng.random() < 0.6)
        drain(lat2, ns, t1 + 300)
        el2 = time.perf_counter() - t1
        st2 = srv.stats()
        lat2 = np.array(lat2)
        saturated = {"requests": ns, "completed": len(lat2), "failed": int(st2["failed"] - st["failed"]),
                     "throughput_rps": len(lat2) / el2, "mpx_s": px2 / 1e6 / el2,
                     "waves": int(st2["waves"] - st["waves"]), "p50_ms": float(np.percentile(lat2, 50)),
                     "p99_ms": float(np.percentile(lat2, 99)), "phases": phases(st, st2),
                     "note": "all requests submitted at t=0 (latency includes queueing behind earlier requests)"}
    srv.close()
    lat = np.array(lat)
    return {"engine": "live admission into one running tile kernel" if live else "waves (two in flight)",
            "requests": n, "rate_rps": args.serve_rate, "new_fraction": 0.6, "completed": int(st["completed"]),
            "failed": int(st["failed"]), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "throughput_rps": len(lat) / elapsed, "mpx_s": px / 1e6 / elapsed,
            "waves": int(st["waves"]), "requests_per_wave": len(lat) / max(1, st["waves"]),
            "hbm_budget_gb": SERVE_BUDGET / 2 ** 30, "evictions": int(st["evictions"]), "phases": phases(zero, st),
            "images": "sides log-U[256,4096], half gray blobs / half rgb8 Voronoi, %d distinct" % SERVE_POOL,
            "saturated": saturated}


def run_reference(args, dist):
    """The reference arm: the oracle (the reference's raster algorithm restated on the CPU; the reference itself
    has no CPU implementation of the path) on all host cores, each step one pass over the stratified sample of
    the batch.  The inputs come from the oracle's build of the workload generators, so this process loads only
    libraries under oracle/."""
    if dist.rank != 0:
        return
    from distance_transform_benchmarks_b200 import workloads as wl
    from oracle import oracle as orc
    wl.use_generator(orc.workload_generator_path())
    specs = wl.config3_specs(seed=args.seed, n=args.images)
    idx = wl.stratified_indices(specs, args.ref_mpx)
    desc, px = sample_desc(idx, specs)
    sample = [wl.make_image(specs[i]) for i in idx]
    for _ in range(args.warmup):
        for img, mask, g in sample[:4]:
            orc.ggdt_ns(img, mask, g)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for img, mask, g in sample:
            orc.ggdt_ns(img, mask, g)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = px / 1e6 / (ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(args, specs),
            "sample": desc,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": orc.max_threads(), "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, dist):
    import distance_transform_benchmarks_b200 as dtb
    from distance_transform_benchmarks_b200 import workloads as wl
    from distance_transform_benchmarks_b200.verify import ns_fixpoint_violations

    dev = dist.local
    torch.cuda.set_device(dev)
    ctx = dtb.Context(dev)
    stream = torch.cuda.current_stream()

    specs = wl.config3_specs(seed=dist.seed(args.seed), n=args.images)
    batch = [wl.make_image(sp) for sp in specs]
    px = wl.pixels(batch)
    alg_bytes = sum(img.shape[0] * img.shape[1] * wl.bytes_per_pixel(img) for img, _, _ in batch)
    imgs = [dtb.pitched_from(i) for i, _, _ in batch]
    masks = [dtb.pitched_from(m) for _, m, _ in batch]
    gammas = [g for _, _, g in batch]
    dists = [dtb.pitched_empty(i.shape[0], i.shape[1], 1, torch.float32) for i, _, _ in batch]

    # The batched persistent form: a plan (descriptors, tensor maps and scratch prepared once) whose run is one
    # CUDA graph (queue reset, seed scan, the cooperative persistent tile kernel, finalize), autotuned first.
    plan = dtb.BatchPlan(imgs, masks, gammas, dists=dists, ctx=ctx)
    tuning = plan.autotune(reps=2, stream=stream)
    for _ in range(max(3, args.warmup)):
        plan.run(stream)
        stats = plan.wait(stream)

    clocks = Clocks(dev)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.run(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    stats = plan.wait(stream)
    dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = dist.max(ms, "cuda")
    px_all = dist.sum(px, "cuda")
    value = px_all / 1e6 / (ms_max / 1e3)

    # Parity of the timed workload itself: every map of the last timed step satisfies the exact fixpoint
    # characterisation (no edge can lower a value, every value is realised); the oracle compares a sample bit for
    # bit in the CPU legs below.
    viol = 0
    for k in range(len(batch)):
        va, vb, _ = ns_fixpoint_violations(imgs[k], masks[k], gammas[k], dtb.DEFAULT_V, dists[k])
        viol += va + vb
    maps = [d.cpu().numpy() for d in dists]

    # The reference arm's stratified sample through the same path (plan, graph launch, device-resident), so the
    # two arms can also be compared on identical pixels.
    ref_idx = wl.stratified_indices(specs, args.ref_mpx)
    ref_desc, ref_px = sample_desc(ref_idx, specs)
    sub_plan = dtb.BatchPlan([imgs[i] for i in ref_idx], [masks[i] for i in ref_idx], [gammas[i] for i in ref_idx],
                             dists=[dists[i] for i in ref_idx], ctx=ctx)
    for _ in range(3):
        sub_plan.run(stream)
    sub_plan.wait(stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        sub_plan.run(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    sub_plan.wait(stream)
    ref_sample_ours = ref_px / 1e6 / (e0.elapsed_time(e1) / args.steps / 1e3)
    sub_plan.close()

    # The same batch through the one-shot call (descriptors and tensor maps rebuilt per call, no graph; the
    # context reuses the autotuned launch).  Its DTB_FLAG_TIMING events, recorded on the launching stream
    # around the tile kernel, give the kernel's device time for the roofline.
    kernel_ms = []
    for _ in range(2):
        dtb.geodesic_distance_transform_batch(imgs, masks, gammas, dists=dists, ctx=ctx, stream=stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(max(3, min(args.steps, 10))):
        dtb.geodesic_distance_transform_batch(imgs, masks, gammas, dists=dists, ctx=ctx, stream=stream, timing=True)
        kernel_ms.append(ctx.stats()["kernel_ms"])
    e1.record(stream)
    torch.cuda.synchronize()
    one_shot = px / 1e6 / (e0.elapsed_time(e1) / len(kernel_ms) / 1e3)

    # The per-image forms on the first PLAIN_SUBSET images: the plain path (host-driven rounds, one call per
    # image, the structure of the reference's blocks variant), the persistent kernel called once per image, and
    # the same images as one batched call.
    sub = list(range(min(PLAIN_SUBSET, len(batch))))
    px_sub = sum(batch[k][0].shape[0] * batch[k][0].shape[1] for k in sub)

    def per_image(rounds):
        for k in sub:
            dtb.geodesic_distance_transform(imgs[k], masks[k], gammas[k], dist=dists[k], ctx=ctx, stream=stream,
                                            rounds=rounds)

    def batched():
        dtb.geodesic_distance_transform_batch([imgs[k] for k in sub], [masks[k] for k in sub], [gammas[k] for k in sub],
                                              dists=[dists[k] for k in sub], ctx=ctx, stream=stream)

    rates = {}
    for name, fn in (("plain", lambda: per_image(True)), ("persistent", lambda: per_image(False)), ("batched", batched)):
        fn()
        torch.cuda.synchronize()
        best = None
        for _ in range(3):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
            best = t if best is None else min(best, t)
        rates[name] = px_sub / 1e6 / best

    # End to end through the C ABI with pinned host buffers.
    e2e = None
    himgs = hmasks = hdists = None
    if not args.no_e2e:
        # The batch as a data loader would hand it over: one pinned arena per plane kind (images, masks, maps).
        himgs, hmasks, hdists = dtb.host_batch_arena([i for i, _, _ in batch], [m for _, m, _ in batch])
        h2d = sum(t.numel() * t.element_size() for t in himgs + hmasks)
        d2h = sum(t.numel() * t.element_size() for t in hdists)

        def estep(last=False):
            # Asynchronous calls: a call's host-side preparation and copies in overlap the previous call's run and
            # copies out.  The last call is synchronous: `stream` then waits for the end of every call before e1
            # (an asynchronous host batch does not make `stream` wait for it).
            dtb.geodesic_distance_transform_batch(himgs, hmasks, gammas, dists=hdists, ctx=ctx, stream=stream,
                                                  asynchronous=not last)

        for _ in range(2):
            estep()
        ctx.sync(stream)
        dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for k in range(args.steps):
            estep(last=k == args.steps - 1)
        e1.record(stream)
        ctx.sync(stream)  # raises on a device error of any step
        torch.cuda.synchronize()
        ems = dist.max(e0.elapsed_time(e1) / args.steps, "cuda")
        e2e = {"value": px_all / 1e6 / (ems / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": ems}
        e2e["maps_equal_device_run"] = bool(all(np.array_equal(hd.numpy().view(np.uint32), m.view(np.uint32))
                                                for hd, m in zip(hdists, maps)))
        e2e["host_layout"] = "one pinned arena per plane kind (images, masks, distance maps)"
        e2e["calls"] = "asynchronous, the last one synchronous (the timed region ends with the last copy out)"
        est = ctx.stats()  # the K timed calls (the last, synchronous one reports them all)
        e2e["library_bytes_per_step"] = {"h2d": est["h2d_bytes"] // max(1, args.steps),
                                         "d2h": est["d2h_bytes"] // max(1, args.steps),
                                         "note": "bytes the host pipeline copied (h2d includes its descriptor tables)"}
        if dist.world == 1:
            e2e["link"] = link_floor(h2d, d2h, ems, int(est["rounds"]) // max(1, args.steps))
    if e2e is not None and dist.world == 1:
        # The same batch from separate pinned buffers per image (one copy per plane and direction).
        simgs = [torch.from_numpy(i).pin_memory() for i, _, _ in batch]
        smasks = [torch.from_numpy(m).pin_memory() for _, m, _ in batch]
        sdists = [torch.empty(i.shape[:2], dtype=torch.float32).pin_memory() for i, _, _ in batch]
        dtb.geodesic_distance_transform_batch(simgs, smasks, gammas, dists=sdists, ctx=ctx, stream=stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            dtb.geodesic_distance_transform_batch(simgs, smasks, gammas, dists=sdists, ctx=ctx, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e["separate_buffers_mpx_s"] = px / 1e6 / (e0.elapsed_time(e1) / 3 / 1e3)
        simgs = smasks = sdists = None

    kms = statistics.mean(kernel_ms) if kernel_ms and kernel_ms[0] > 0 else None
    peak, peak_kind = measured_peak_gbs()
    roofline = None
    if kms:
        achieved = alg_bytes / (kms / 1e3) / 1e9
        bpp = profiled_traffic_bytes_per_px()
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_kind": peak_kind, "kernel": "ggdt_persistent", "kernel_ms": kms,
                    "algorithmic_bytes": alg_bytes, "traffic": (bpp * px) if bpp else None}

    # The reference-shape, single-image and serving legs run in single-GPU runs only (with N ranks every rank
    # would repeat them on its own GPU; the job's line reports the batch and e2e legs, reduced over ranks).
    one_gpu = dist.world == 1
    ref_mode = None if (args.no_ref_mode or not one_gpu) else run_ref_mode(args, ctx, stream)
    configs, config_maps = (None, {}) if (args.no_configs or not one_gpu) else run_configs(ctx, stream)
    cpu = parity = None
    if dist.rank == 0 and one_gpu and not args.no_cpu_baseline:
        cpu, parity = cpu_legs(batch, specs, ref_idx, maps, config_maps)
    config_maps = None
    if parity is None:
        parity = {}
    parity.update({"fixpoint_images": len(batch), "fixpoint_violations": viol,
                   "fixpoint_check": "every map of the timed batch: no edge lowers a value and every value is "
                                     "realised (exact greatest-fixpoint characterisation, on the GPU)"})
    serve = serve_live = None
    if not args.no_serve and one_gpu:
        himgs = hmasks = hdists = None  # release pinned host memory of the e2e leg
        pool = serve_pool()
        serve = run_serve(args, dev, pool)
        serve_live = run_serve(args, dev, pool, live=True)
        pool = None

    if dist.rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": bench_config(args, specs),
                "launch": "one CUDA graph per step: queue reset, seed scan, persistent tile kernel, finalize",
                "parity": parity,
                "reference_sample": {"sample": ref_desc, "ours_mpx_s": ref_sample_ours,
                                     "note": "the reference arm's per-step sample through the same graph-launched "
                                             "plan, device-resident"},
                "per_image": {"subset": "first %d images of the batch (%.1f Mpx)" % (len(sub), px_sub / 1e6),
                              "plain_per_image_mpx_s": rates["plain"],
                              "persistent_per_image_mpx_s": rates["persistent"],
                              "batched_mpx_s": rates["batched"],
                              "batched_vs_plain": rates["batched"] / rates["plain"],
                              "batched_vs_persistent_per_image": rates["batched"] / rates["persistent"],
                              "note": "plain = host-driven rounds (the reference's blocks-variant structure), one "
                                      "call per image; persistent = one persistent-kernel call per image; batched = "
                                      "the same images in one call; wall clock, best of 3"},
                "full_batch_graph_vs_plain_per_image": value / rates["plain"],
                "one_shot_call_mpx_s": one_shot, "autotuned": tuning,
                "tile_stats": {"tiles": stats["tiles"], "visits_per_tile": stats["tile_visits"] / max(1, stats["tiles"]),
                               "phases_per_visit": stats["phases"] / max(1, stats["tile_visits"])},
                "gpu_launches": 3 * args.steps,
                "clocks": clk, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "serve": serve,
                "serve_live": serve_live,
                "ref_mode": ref_mode, "configs": configs}
        print(json.dumps(line), flush=True)
    plan.close()
    ctx.close()


def main():
    args = parse()
    dist = Dist()
    if dist.world > 1 and "OMP_NUM_THREADS" not in os.environ:
        # The ranks share the host: split its cores for the input generators.
        os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or 1) // dist.world))
    if args.impl == "reference":
        run_reference(args, dist)  # rank 0 only; the other ranks exit without work
        return
    dist.init("nccl")
    try:
        run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
