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
    assert lib.dtb_abi_version() == _native.ABI_VERSION == 3
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


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every struct of include/dtb.h, compiled as C: size and member offsets equal the ctypes mirror's."""
    import shutil
    import subprocess
    nat = _native
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"dtb_image": nat.DtbImage, "dtb_stats": nat.DtbStats, "dtb_tuning": nat.DtbTuning,
               "dtb_serve_config": nat.DtbServeConfig, "dtb_serve_request": nat.DtbServeRequest,
               "dtb_serve_completion": nat.DtbServeCompletion, "dtb_serve_stats": nat.DtbServeStats}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "dtb.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append('  printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for field, _ in py._fields_:
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, field, cname, field))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([cc, "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, what, val = line.split()
        got[(cname, what)] = int(val)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)
