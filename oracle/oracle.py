"""ctypes front end of the CPU oracle (oracle/ggdt_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
reference legs, as the checker.  The product path (distance_transform_benchmarks_b200) never imports it.
See ggdt_oracle.c for what is pinned against the reference (ref-mode: the two golden tensors of
tests/distance_transform.cpp) and what is not (ns-mode: parity unpinned with respect to the reference).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
WORKLOADS_PATH = os.path.join(HERE, "libworkloads.so")
REF_PASSES_PATH = os.path.join(HERE, "_ref", "libref_passes.so")
_lib = None
_ref_lib = None


def build(force=False):
    """Builds liboracle.so and libworkloads.so (make's own dependency check decides what is stale)."""
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []), check=True)
    return LIB_PATH


def workload_generator_path():
    """The oracle's build of the package's seeded workload generators (csrc/datagen.cpp): the same pixels as
    libdtb_host.so, for processes that must not load a library of the package (bench.py's reference arm)."""
    if not os.path.exists(WORKLOADS_PATH):
        build()
    return WORKLOADS_PATH


REF_TESTS = ("image_view", "image2d", "c4", "rgb8", "io", "transfert", "distance_transform")


def build_ref(ref_root, force=False):
    """Builds, from the reference source tree at `ref_root`, into _ref/: the reference's tile-pass device
    functions (libref_passes.so, see ref_passes_driver.cu), the reference's image decoder (libstb_ref.so, the
    reference's dt/src/stb_image_implementation.c) and the reference's own unit tests compiled against include/dt
    and libdtb (test_<name>, see gtest_shim/).  libdtb must be built first.  Returns False if
    `ref_root` is absent."""
    if not os.path.isdir(os.path.join(ref_root, "dt", "src")):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", "stb-ref", "ref-tests", "REF_ROOT=" + ref_root] +
                   (["-B"] if force else []), check=True)
    return True


STB_REF_PATH = os.path.join(HERE, "_ref", "libstb_ref.so")


def stb_ref_available():
    return os.path.exists(STB_REF_PATH)


def stb_ref_load(path, req_comp=0):
    """The reference's image decoder (stb_image, built by build_ref from the reference's own source) on a file:
    stbi_load(path, &w, &h, &n, req_comp) as dt::imread calls it (dt/src/imread.cpp:14, req_comp = 0).  Returns
    (uint8 array [h, w, n'], n) with n' = req_comp or n, or None when stb_image rejects the file."""
    lib = ctypes.CDLL(STB_REF_PATH)
    lib.stbi_load.restype = ctypes.POINTER(ctypes.c_uint8)
    lib.stbi_load.argtypes = [ctypes.c_char_p] + [ctypes.POINTER(ctypes.c_int)] * 3 + [ctypes.c_int]
    w, h, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    p = lib.stbi_load(str(path).encode(), ctypes.byref(w), ctypes.byref(h), ctypes.byref(n), int(req_comp))
    if not p:
        return None
    try:
        ch = req_comp or n.value
        a = np.ctypeslib.as_array(p, shape=(h.value * w.value * ch,)).reshape(h.value, w.value, ch).copy()
    finally:
        lib.stbi_image_free(ctypes.cast(p, ctypes.c_void_p))
    return a, n.value


def ref_test_binary(name):
    """Path of the reference unit test `name` built by build_ref, or None if it was not built."""
    p = os.path.join(HERE, "_ref", "test_" + name)
    return p if os.path.exists(p) else None


def ref_passes_available():
    return os.path.exists(REF_PASSES_PATH)


def ref_passes(imgs, masks, lam, v=1e10):
    """The reference's compiled ref-mode arithmetic (dt/src/dt_block_passes.cuh:12-127) run to quiescence on the
    GPU, for a stack of n images of at most 32x32 pixels (uint8 [n, h, w] image and seed mask).  Needs a GPU
    and _ref/libref_passes.so."""
    global _ref_lib
    if _ref_lib is None:
        L = ctypes.CDLL(REF_PASSES_PATH)
        P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.refp_gdt_tiles.restype = I
        L.refp_gdt_tiles.argtypes = [P, P, P, I, I, I, F, F]
        _ref_lib = L
    imgs = _c(np.asarray(imgs, dtype=np.uint8))
    masks = _c(np.asarray(masks, dtype=np.uint8))
    n, h, w = imgs.shape
    assert masks.shape == imgs.shape
    out = np.empty((n, h, w), dtype=np.float32)
    rc = _ref_lib.refp_gdt_tiles(imgs.ctypes.data, masks.ctypes.data, out.ctypes.data, n, w, h, float(lam), float(v))
    if rc != 0:
        raise RuntimeError("refp_gdt_tiles failed with code %d" % rc)
    return out


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P, I, F, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.oracle_ggdt_ref.restype = I
        L.oracle_ggdt_ref.argtypes = [P, I, P, I, P, I, I, F, F, I, I]
        L.oracle_ggdt_ns.restype = I
        L.oracle_ggdt_ns.argtypes = [P, I, I, P, I, P, I, I, F, F, I, I]
        L.oracle_ggdt_ns_warm.restype = I
        L.oracle_ggdt_ns_warm.argtypes = [P, I, I, P, I, P, I, I, F, I, I]
        L.oracle_ggdt_ns_serial.restype = I
        L.oracle_ggdt_ns_serial.argtypes = [P, I, I, P, I, P, I, I, F, F, I]
        L.oracle_dijkstra_ns_f64.restype = I
        L.oracle_dijkstra_ns_f64.argtypes = [P, I, I, P, I, P, I, I, D, D]
        L.oracle_max_threads.restype = I
        _lib = L
    return _lib


MAX_ROUNDS = 1 << 30


def _c(a):
    return np.ascontiguousarray(a)


def g2_of(gamma):
    """fl32(gamma * gamma), the squaring the CUDA path performs."""
    g = np.float32(gamma)
    return np.float32(g * g)


def ggdt_ref(img, mask, lam, v=1e10, fma=True):
    """ref-mode fixpoint (C8, lambda blend), gray uint8 [H, W]."""
    img, mask = _c(img), _c(mask)
    h, w = img.shape
    d = np.empty((h, w), np.float32)
    r = lib().oracle_ggdt_ref(img.ctypes.data, w, mask.ctypes.data, w, d.ctypes.data, w, h, float(lam), float(v),
                              1 if fma else 0, MAX_ROUNDS)
    if r < 0:
        raise RuntimeError("oracle did not converge")
    return d


def ggdt_ns(img, mask, gamma, v=1e10, nthreads=0, serial=False):
    """ns-mode fixpoint (C4, sqrt(1 + g2 dI^2)), gray [H, W] or rgb8 [H, W, 3]."""
    img, mask = _c(img), _c(mask)
    h, w = img.shape[:2]
    ch = 3 if img.ndim == 3 else 1
    d = np.empty((h, w), np.float32)
    g2 = float(g2_of(gamma))
    if serial:
        r = lib().oracle_ggdt_ns_serial(img.ctypes.data, w * ch, ch, mask.ctypes.data, w, d.ctypes.data, w, h, g2,
                                        float(v), MAX_ROUNDS)
    else:
        r = lib().oracle_ggdt_ns(img.ctypes.data, w * ch, ch, mask.ctypes.data, w, d.ctypes.data, w, h, g2, float(v),
                                 int(nthreads), MAX_ROUNDS)
    if r < 0:
        raise RuntimeError("oracle did not converge")
    return d


def ggdt_ns_warm(img, new_seeds, prev, gamma, nthreads=0):
    """Warm start from a previous ns-mode map with added seeds."""
    img, new_seeds = _c(img), _c(new_seeds)
    h, w = img.shape[:2]
    ch = 3 if img.ndim == 3 else 1
    d = np.array(prev, np.float32, copy=True, order="C")
    r = lib().oracle_ggdt_ns_warm(img.ctypes.data, w * ch, ch, new_seeds.ctypes.data, w, d.ctypes.data, w, h,
                                  float(g2_of(gamma)), int(nthreads), MAX_ROUNDS)
    if r < 0:
        raise RuntimeError("oracle did not converge")
    return d


def dijkstra_ns_f64(img, mask, gamma, v=1e10):
    """Exact-sum FP64 Dijkstra on the ns-mode graph (weights evaluated in double from g2 = fl32(gamma^2))."""
    img, mask = _c(img), _c(mask)
    h, w = img.shape[:2]
    ch = 3 if img.ndim == 3 else 1
    d = np.empty((h, w), np.float64)
    r = lib().oracle_dijkstra_ns_f64(img.ctypes.data, w * ch, ch, mask.ctypes.data, w, d.ctypes.data, w, h,
                                     float(g2_of(gamma)), float(v))
    if r != 0:
        raise MemoryError("dijkstra allocation failed")
    return d


def max_threads():
    return lib().oracle_max_threads()
