"""Extract the reference's golden GGDT tensors into tests/golden/ref_goldens.npz.

Reads tests/distance_transform.cpp of the reference project as text (it is never compiled or run):

* ``DistanceTransform.EuclidianFastGeodis`` (tests/distance_transform.cpp:14-281): 50x40 zero image,
  seed rectangle x in [20, 43), y in [20, 30) (:267-273), lambda = 0, expected ``ref_data``.
* ``DistanceTransform.GeodesicFastGeodis`` (tests/distance_transform.cpp:283-476): 36x34 ``img_data``,
  single seed at (width / 2, height / 2) (:468), lambda = 1, expected ``ref_data``.

Both calls use the API default v = 1e10 (dt/include/dt/generalised_distance_transform.hpp:8,11).
The float literals are converted the way the C++ compiler does: decimal -> double -> float.

Usage: python tests/golden/make_golden.py path/to/reference/tests/distance_transform.cpp
       (or set DTB_REFERENCE_ROOT to the reference project's root)
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _test_body(text, name):
    m = re.search(r"TEST\(DistanceTransform,\s*%s\)\s*\{" % name, text)
    if not m:
        raise RuntimeError("test %s not found" % name)
    depth, i = 1, m.end()
    while depth:
        c = text[i]
        depth += c == "{"
        depth -= c == "}"
        i += 1
    return text[m.end():i - 1]


def _array(body, ctype, name):
    m = re.search(r"%s\s+%s\[\]\s*=\s*\{(.*?)\};" % (re.escape(ctype), name), body, flags=re.S)
    if not m:
        raise RuntimeError("array %s not found" % name)
    return [tok.strip() for tok in m.group(1).split(",") if tok.strip()]


def _int_const(body, name):
    m = re.search(r"constexpr\s+int\s+%s\s*=\s*(\d+)\s*;" % name, body)
    return int(m.group(1))


def main(src):
    text = _strip_comments(open(src).read())

    b1 = _test_body(text, "EuclidianFastGeodis")
    w1, h1 = _int_const(b1, "WIDTH"), _int_const(b1, "HEIGHT")
    ref1 = np.array([np.float32(float(t)) for t in _array(b1, "float", "ref_data")], np.float32).reshape(h1, w1)
    img1 = np.zeros((h1, w1), np.uint8)
    m = re.search(r"for \(int y = (\d+); y < (\d+); y\+\+\)\s*\{\s*for \(int x = (\d+); x < (\d+); x\+\+\)", b1)
    y0, y1, x0, x1 = map(int, m.groups())
    mask1 = np.zeros((h1, w1), np.uint8)
    mask1[y0:y1, x0:x1] = 1
    lam1 = float(re.search(r"generalised_distance_transform\(d_img, d_mask, ([0-9.]+)f?\)", b1).group(1))

    b2 = _test_body(text, "GeodesicFastGeodis")
    w2, h2 = _int_const(b2, "WIDTH"), _int_const(b2, "HEIGHT")
    img2 = np.array([int(t) for t in _array(b2, "std::uint8_t", "img_data")], np.uint8).reshape(h2, w2)
    ref2 = np.array([np.float32(float(t)) for t in _array(b2, "float", "ref_data")], np.float32).reshape(h2, w2)
    assert "mask(img.width() / 2, img.height() / 2) = 1" in b2
    mask2 = np.zeros((h2, w2), np.uint8)
    mask2[h2 // 2, w2 // 2] = 1
    lam2 = float(re.search(r"generalised_distance_transform\(d_img, d_mask, ([0-9.]+)f?\)", b2).group(1))

    out = os.path.join(HERE, "ref_goldens.npz")
    np.savez_compressed(
        out,
        euclid_img=img1, euclid_mask=mask1, euclid_ref=ref1, euclid_lambda=np.float32(lam1),
        geodesic_img=img2, geodesic_mask=mask2, geodesic_ref=ref2, geodesic_lambda=np.float32(lam2),
        v=np.float32(1e10),
    )
    print("wrote", out, ref1.shape, ref2.shape, "lambdas", lam1, lam2, "rect", (x0, x1, y0, y1))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("DTB_REFERENCE_ROOT"):
        main(os.path.join(os.environ["DTB_REFERENCE_ROOT"], "tests", "distance_transform.cpp"))
    else:
        sys.exit("usage: make_golden.py <reference>/tests/distance_transform.cpp (or set DTB_REFERENCE_ROOT)")
