"""JPEG fixtures and the reference decoder's output for them: tests/golden/jpeg/*.jpg and jpeg_goldens.npz.

The reference reads its benchmark inputs with dt::imread (dt/src/imread.cpp:10-31), i.e. stbi_load(path, &w, &h,
&n, 0) of the stb_image it vendors, and accepts only 1-component files.  This script encodes small seeded synthetic
images with OpenCV's JPEG encoder in the modes that decoder handles (baseline and progressive frames, optimised
Huffman tables, restart intervals, 4:4:4 / 4:2:2 / 4:2:0 / 4:1:1 / 4:4:0 chroma), decodes every file with stb_image
built from the reference's own source (oracle/_ref/libstb_ref.so, `make -C oracle stb-ref REF_ROOT=...`) and stores
what it returns: the gray samples for 1-component files, stbi_load(..., 3) for colour files.

Usage: python tests/golden/make_jpeg_golden.py   (after building oracle/_ref/libstb_ref.so)
"""
import os
import sys

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as orc  # noqa: E402

SUB = {"444": cv2.IMWRITE_JPEG_SAMPLING_FACTOR_444, "422": cv2.IMWRITE_JPEG_SAMPLING_FACTOR_422,
       "420": cv2.IMWRITE_JPEG_SAMPLING_FACTOR_420, "411": cv2.IMWRITE_JPEG_SAMPLING_FACTOR_411,
       "440": cv2.IMWRITE_JPEG_SAMPLING_FACTOR_440}

# name: (height, width, channels, quality, progressive, restart interval (MCUs), optimised tables, chroma)
CASES = {
    "gray_base_q90": (45, 67, 1, 90, 0, 0, 0, None),
    "gray_prog_q75": (45, 67, 1, 75, 1, 0, 0, None),
    "gray_rst2_opt_q50": (17, 129, 1, 50, 0, 2, 1, None),
    "gray_prog_rst1_q100": (64, 64, 1, 100, 1, 1, 0, None),
    "gray_1x1_q90": (1, 1, 1, 90, 0, 0, 0, None),
    "gray_base_q20": (8, 200, 1, 20, 0, 0, 1, None),
    "rgb_420_q90": (45, 67, 3, 90, 0, 0, 0, "420"),
    "rgb_422_prog_q80": (37, 53, 3, 80, 1, 0, 0, "422"),
    "rgb_444_rst3_q95": (24, 40, 3, 95, 0, 3, 0, "444"),
    "rgb_411_q85": (21, 70, 3, 85, 0, 0, 1, "411"),
    "rgb_440_prog_q70": (50, 35, 3, 70, 1, 0, 0, "440"),
}


def synthetic(h, w, c, seed):
    """Smooth shading, a checker of hard edges and sensor-like noise: every DCT band carries energy."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    planes = []
    for k in range(c):
        base = 128 + 90 * np.sin(x / (5.0 + 2 * k) + k) * np.cos(y / 7.0)
        base += 40 * (((x // 11) + (y // 6) + k) % 2) - 20
        planes.append(base + rng.normal(0, 14, (h, w)))
    return np.clip(np.stack(planes, -1), 0, 255).astype(np.uint8)


def encode(name):
    h, w, c, q, prog, rst, opt, sub = CASES[name]
    img = synthetic(h, w, c, seed=sum(map(ord, name)))
    params = [cv2.IMWRITE_JPEG_QUALITY, q, cv2.IMWRITE_JPEG_PROGRESSIVE, prog, cv2.IMWRITE_JPEG_RST_INTERVAL, rst,
              cv2.IMWRITE_JPEG_OPTIMIZE, opt]
    if sub:
        params += [cv2.IMWRITE_JPEG_SAMPLING_FACTOR, SUB[sub]]
    ok, buf = cv2.imencode(".jpg", img[..., ::-1] if c == 3 else img[..., 0], params)  # OpenCV takes BGR
    assert ok, name
    return buf.tobytes()


def main():
    if not orc.stb_ref_available():
        sys.exit("oracle/_ref/libstb_ref.so is missing: make -C oracle stb-ref REF_ROOT=<reference root>")
    out_dir = os.path.join(HERE, "jpeg")
    os.makedirs(out_dir, exist_ok=True)
    goldens = {}
    for name, case in CASES.items():
        path = os.path.join(out_dir, name + ".jpg")
        with open(path, "wb") as f:
            f.write(encode(name))
        gray = case[2] == 1
        got = orc.stb_ref_load(path, 0 if gray else 3)
        assert got is not None, name
        pixels, n = got
        assert n == case[2], (name, n)
        goldens[name] = pixels[..., 0] if gray else pixels
    np.savez_compressed(os.path.join(HERE, "jpeg_goldens.npz"), **goldens)
    print("wrote %d fixtures" % len(goldens))


if __name__ == "__main__":
    main()
