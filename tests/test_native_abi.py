"""CPU tests of the native boundary: the libraries load and export every symbol include/dtb.h declares,
and the host-side entry points behave without a GPU."""
import ctypes
import os
import re

import pytest

from distance_transform_benchmarks_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"DTB_API\s+[\w\s\*]+?\b(dtb_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert _declared("dtb.h") == sorted(_native.DTB_SYMBOLS)


def test_libdtb_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.LIBDTB_PATH)
    for name in _declared("dtb.h"):
        assert hasattr(lib, name), name


def test_abi_version_and_status_strings():
    lib = _native.lib()
    assert lib.dtb_abi_version() == 1
    assert lib.dtb_status_string(0) == b"ok"
    assert lib.dtb_status_string(4) == b"device wait timed out"
    assert lib.dtb_status_string(99) == b"unknown status"


def test_context_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = _native.lib().dtb_context_create(0, ctypes.byref(h))
    assert st == 6 and not h.value  # DTB_ERR_NO_DEVICE


def test_invalid_arguments_are_rejected_before_any_device_work():
    lib = _native.lib()
    assert lib.dtb_gdt(None, None, None, None, 1.0, 1.0, 0, None) == 1
    assert lib.dtb_host_to_device(None, None, None) == 1
    a = _native.DtbImage(None, 4, 4, 4, 1, 0)
    b = _native.DtbImage(None, 4, 4, 4, 1, 0)  # both CPU: not a host->device pair
    assert lib.dtb_host_to_device(ctypes.byref(a), ctypes.byref(b), None) == 1
    assert lib.dtb_gdt_ref_blocks(None, None, None, None, 0.5, 1.0, None, 0, None) == 1
    assert lib.dtb_debug_inject_queue_stall(None, 100) == 1


def test_host_image_allocation_without_gpu():
    """dtb_image_alloc / dtb_image_free of CPU images: packed rows like the reference's CPU image2d."""
    lib = _native.lib()
    im = _native.DtbImage()
    assert lib.dtb_image_alloc(7, 5, 3, 0, ctypes.byref(im)) == 0
    assert (im.width, im.height, im.pitch, im.elem_size, im.memory_kind) == (7, 5, 21, 3, 0) and im.buffer
    ctypes.memset(im.buffer, 0xAB, im.pitch * im.height)
    assert lib.dtb_image_free(ctypes.byref(im)) == 0 and not im.buffer
    assert lib.dtb_image_alloc(-1, 5, 1, 0, ctypes.byref(im)) == 1
    assert lib.dtb_image_alloc(4, 4, 1, 7, ctypes.byref(im)) == 1
    assert lib.dtb_image_free(None) == 1


def test_host_library_exports():
    lib = ctypes.CDLL(_native.LIBHOST_PATH)
    for name in ["dtbg_blobs_gray", "dtbg_voronoi_rgb", "dtbg_maze_gray", "dtbg_draw_disks"]:
        assert hasattr(lib, name)
