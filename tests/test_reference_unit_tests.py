"""The reference's own unit tests of the path, compiled unchanged against this repository's C++ layer.

oracle/Makefile `ref-tests` compiles the reference's tests/{image_view,image2d,c4,rgb8,transfert,
distance_transform}.cpp with include/dt (this repository's namespace dt headers), libdtb and a GoogleTest stand-in
(oracle/gtest_shim).  tests/distance_transform.cpp holds the reference's golden tensors (lambda 0 and 1) and its
raster == blocks == task equality tests on random 250x230 images; passing it is the drop-in check of the C++
boundary.  The binaries exist only where the reference source tree was present at build time.
"""
import subprocess

import pytest

from oracle import oracle as orc


def _run(name, cwd=None):
    exe = orc.ref_test_binary(name)
    if exe is None:
        pytest.skip("oracle/_ref/test_%s not built (reference source tree absent at build time)" % name)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600, cwd=cwd)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 failed" in r.stdout, r.stdout
    return r.stdout


@pytest.mark.parametrize("name", ["image_view", "image2d", "c4", "rgb8", "io"])
def test_reference_host_unit_tests(name, tmp_path):
    _run(name, cwd=str(tmp_path))  # io writes its file into the working directory


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["transfert", "distance_transform"])
def test_reference_device_unit_tests(name):
    out = _run(name)
    if name == "distance_transform":
        for t in ("EuclidianFastGeodis", "GeodesicFastGeodis", "EuclidianBlocks", "GeodesicBlocks", "EuclidianTask",
                  "GeodesicTask"):
            assert "OK ] DistanceTransform." + t in out, out
