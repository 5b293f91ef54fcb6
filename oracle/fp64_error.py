"""Relative error of the fp32 map against the FP64 Dijkstra on the same C4 graph, per workload.

TEST INFRASTRUCTURE: the oracle's fp32 fixpoint equals the CUDA path's map bit for bit (tests/test_gpu_parity.py),
so its error against exact-sum shortest paths is the error of the library's maps.  Run from the repository root:

    python oracle/fp64_error.py [config0 config1 config2 config3]
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from distance_transform_benchmarks_b200 import workloads as wl  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def rel_error(img, mask, gamma):
    d32 = orc.ggdt_ns(img, mask, gamma).astype(np.float64)
    d64 = orc.dijkstra_ns_f64(img, mask, gamma)
    sel = d64 > 0
    rel = np.abs(d32[sel] - d64[sel]) / d64[sel]
    return float(rel.max()), float(rel.mean())


def main(names):
    for name in names:
        t0 = time.perf_counter()
        if name == "config3":  # the ragged batch: its first 64 images
            worst, means = 0.0, []
            for img, mask, g in wl.config3(n=64):
                mx, mn = rel_error(img, mask, g)
                worst = max(worst, mx)
                means.append(mn)
            mx, mn = worst, float(np.mean(means))
        else:
            mx, mn = rel_error(*getattr(wl, name)())
        print("%s: max relative error %.3e, mean %.3e (%.1f s)" % (name, mx, mn, time.perf_counter() - t0), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["config0", "config1", "config2", "config3"])
