"""Command line transform of one image file, the counterpart of the reference's bin/distance_transform.cpp:

    python -m distance_transform_benchmarks_b200.cli input lambda output [mask]

reads a gray 8-bit image (PNG / PGM / JPEG), seeds it at the non-zero pixels of `mask` (default: the centre pixel),
runs the reference-weight transform (C8, lambda blend) on the GPU and writes the map normalised to 0..255 as a
gray image (the reference colours it with the inferno map, which is not part of this library).  With
``--c4 GAMMA`` it runs the C4 geodesic weight sqrt(1 + gamma^2 |dI|^2) instead (gray or, with ``--rgb``, rgb8
input).  ``--raw FILE`` also stores the float map (numpy .npy).
"""
import argparse
import sys

import numpy as np
import torch


def normalize_u8(d):
    """dt::normalize<uint8_t> (reference dt/include/dt/normalize.hpp:36-53): (v - min) / (max - min) * 255."""
    d = d.astype(np.float64)
    lo, hi = d.min(), d.max()
    rng = hi - lo
    if rng == 0:
        return np.zeros(d.shape, np.uint8)
    return ((d - lo) / rng * 255.0).astype(np.uint8)


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("input")
    p.add_argument("lam", type=float, help="lambda in [0, 1] (reference weight)")
    p.add_argument("output")
    p.add_argument("mask", nargs="?", default=None)
    p.add_argument("--c4", type=float, default=None, metavar="GAMMA", help="C4 geodesic weight with this gamma")
    p.add_argument("--rgb", action="store_true", help="rgb8 input (with --c4)")
    p.add_argument("--raw", default=None, help="also save the float map as .npy")
    a = p.parse_args(argv)

    import distance_transform_benchmarks_b200 as dtb
    channels = 3 if (a.rgb and a.c4 is not None) else 1
    img = dtb.imread(a.input, channels)
    h, w = img.shape[:2]
    if a.mask is not None:
        mask = dtb.imread(a.mask, 1)
        if mask.shape != (h, w):
            print("Invalid mask shape (Got (w: %d h: %d), expected (w: %d h: %d))" % (mask.shape[1], mask.shape[0], w, h),
                  file=sys.stderr)
            return 1
    else:
        mask = np.zeros((h, w), np.uint8)
        mask[h // 2, w // 2] = 1
    if not (0.0 <= a.lam <= 1.0):
        print("Lambda argument must be in the range [0.0 - 1.0] (Got %g)" % a.lam, file=sys.stderr)
        return 1
    ti, tm = torch.from_numpy(img).cuda(), torch.from_numpy(mask).cuda()
    if a.c4 is not None:
        d = dtb.geodesic_distance_transform(ti, tm, a.c4)
    else:
        d = dtb.generalised_distance_transform(ti, tm, a.lam)
    d = d.cpu().numpy()
    if a.raw:
        np.save(a.raw, d)
    dtb.imsave(a.output, normalize_u8(d))
    return 0


if __name__ == "__main__":
    sys.exit(main())
