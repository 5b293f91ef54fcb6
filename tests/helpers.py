"""Shared checks of the test suite (the oracle is the checker; nothing here computes a distance map)."""
import numpy as np
import torch


def assert_images_eq(got, ref, what=""):
    """Bit-exact comparison (reference tests/helpers.hpp:25-33 compares with !=), with a useful message."""
    got = got.detach().cpu().numpy() if isinstance(got, torch.Tensor) else np.asarray(got)
    ref = np.asarray(ref)
    assert got.shape == ref.shape, "%s: shape %s != %s" % (what, got.shape, ref.shape)
    bad = got.view(np.uint32) != ref.view(np.uint32)
    if bad.any():
        ys, xs = np.nonzero(bad)
        k = 0
        raise AssertionError("%s: %d of %d values differ; first at (x=%d, y=%d): got %r, expected %r" % (
            what, int(bad.sum()), bad.size, xs[k], ys[k], float(got[ys[k], xs[k]]), float(ref[ys[k], xs[k]])))


# The fixpoint characterisation lives in the package (bench.py checks every map of its timed batch with it).
from distance_transform_benchmarks_b200.verify import ns_fixpoint_violations  # noqa: E402,F401
from distance_transform_benchmarks_b200.verify import ns_weights as ns_weights_torch  # noqa: E402,F401
