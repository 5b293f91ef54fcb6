"""ctypes declarations of the native libraries (include/dtb.h and the generator library).

Loading fails loudly: there is no Python or CPU fallback for the distance transform.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDTB_PATH = os.path.join(HERE, "libdtb.so")
LIBHOST_PATH = os.path.join(HERE, "libdtb_host.so")

DTB_CPU = 0
DTB_GPU = 1

DTB_FLAG_ASYNC = 0x1
DTB_FLAG_ROUNDS = 0x2
DTB_FLAG_REF_NO_FMA = 0x4
DTB_FLAG_TIMING = 0x8

STATUS_NAMES = {
    0: "DTB_OK", 1: "DTB_ERR_INVALID_ARG", 2: "DTB_ERR_CUDA", 3: "DTB_ERR_OUT_OF_MEMORY", 4: "DTB_ERR_TIMEOUT",
    5: "DTB_ERR_DEVICE", 6: "DTB_ERR_NO_DEVICE", 7: "DTB_ERR_CAPACITY", 8: "DTB_ERR_IO",
}

# Every symbol include/dtb.h declares (checked by the CPU test suite).
DTB_SYMBOLS = [
    "dtb_abi_version", "dtb_status_string", "dtb_context_create", "dtb_context_destroy", "dtb_context_message",
    "dtb_last_stats", "dtb_sync", "dtb_gdt_ref", "dtb_gdt", "dtb_gdt_batch", "dtb_gdt_noalloc", "dtb_host_to_device",
    "dtb_device_to_host", "dtb_context_set_tuning", "dtb_context_get_tuning", "dtb_plan_create", "dtb_plan_run",
    "dtb_plan_wait", "dtb_plan_autotune", "dtb_plan_destroy", "dtb_serve_create", "dtb_serve_submit", "dtb_serve_poll",
    "dtb_serve_release", "dtb_serve_get_stats", "dtb_serve_destroy", "dtb_gdt_ref_blocks", "dtb_image_alloc",
    "dtb_image_free", "dtb_debug_inject_queue_stall", "dtb_image_read", "dtb_image_write", "dtb_plan_get_tuning",
    "dtb_context_set_tuning_cache",
]

DTB_REQ_IMAGE = 0
DTB_REQ_EDIT = 1


class DtbImage(ctypes.Structure):
    """dtb_image: the fields of dt::image2d_view<void> (reference dt/include/dt/image2d_view.hpp:117-123)."""
    _fields_ = [
        ("buffer", ctypes.c_void_p),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("pitch", ctypes.c_int32),
        ("elem_size", ctypes.c_int32),
        ("memory_kind", ctypes.c_int32),
    ]


class DtbStats(ctypes.Structure):
    _fields_ = [
        ("tiles", ctypes.c_uint64),
        ("tile_visits", ctypes.c_uint64),
        ("phases", ctypes.c_uint64),
        ("activations", ctypes.c_uint64),
        ("rounds", ctypes.c_uint64),
        ("device_error", ctypes.c_uint32),
        ("device_error_info", ctypes.c_uint32),
        ("kernel_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
    ]


class DtbTuning(ctypes.Structure):
    _fields_ = [("ctas_per_sm", ctypes.c_int32), ("grid_percent", ctypes.c_int32), ("host_chunk_kpx", ctypes.c_int32),
                ("queue_buckets", ctypes.c_int32), ("bucket_width_pct", ctypes.c_int32), ("staging", ctypes.c_int32),
                ("warps_per_cta", ctypes.c_int32)]


class DtbServeConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_wave_requests", ctypes.c_int32), ("v", ctypes.c_float),
                ("max_wave_tiles", ctypes.c_uint32), ("wave_stage_bytes", ctypes.c_uint64), ("live", ctypes.c_int32),
                ("live_idle_us", ctypes.c_uint32)]


class DtbServeRequest(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("image_id", ctypes.c_int64), ("img", DtbImage), ("mask", DtbImage),
                ("gamma", ctypes.c_float), ("n_disks", ctypes.c_int32), ("disks", ctypes.POINTER(ctypes.c_int32)),
                ("out", DtbImage)]


class DtbServeCompletion(ctypes.Structure):
    _fields_ = [("request_id", ctypes.c_int64), ("status", ctypes.c_int32), ("latency_ms", ctypes.c_double)]


class DtbServeStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("submitted", "completed", "failed", "waves", "evictions", "pending",
                                             "resident_images")] + \
               [(n, ctypes.c_uint64) for n in ("resident_bytes", "tiles", "tile_visits")] + \
               [(n, ctypes.c_double) for n in ("host_prep_ms", "copy_in_ms", "kernel_ms", "copy_out_ms", "queue_wait_ms",
                                               "queue_wait_max_ms")] + \
               [("waves_split", ctypes.c_int64)] + \
               [(n, ctypes.c_int64) for n in ("live_ended_idle", "live_ended_lifetime", "live_ended_error",
                                             "live_ended_stop")]


class DtbError(RuntimeError):
    """A dtb_* call returned a non-zero status (the reference throws std::runtime_error in these cases)."""

    def __init__(self, status, message):
        self.status = status
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))


_lib = None
_host = None
ABI_VERSION = 3  # the struct layouts mirrored here (include/dtb.h DTB_ABI_VERSION)


def lib():
    """The CUDA library; raises if it was not built (run __graft_entry__.build())."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBDTB_PATH):
            raise RuntimeError("libdtb.so is missing at %s: build it with __graft_entry__.build()" % LIBDTB_PATH)
        L = ctypes.CDLL(LIBDTB_PATH)
        P, I32, U32, F = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32, ctypes.c_float
        IMG = ctypes.POINTER(DtbImage)
        L.dtb_abi_version.restype = I32
        if L.dtb_abi_version() != ABI_VERSION:
            raise RuntimeError("libdtb.so has ABI version %d, this package mirrors %d: rebuild it with "
                               "__graft_entry__.build()" % (L.dtb_abi_version(), ABI_VERSION))
        L.dtb_status_string.restype = ctypes.c_char_p
        L.dtb_status_string.argtypes = [I32]
        L.dtb_context_create.restype = I32
        L.dtb_context_create.argtypes = [I32, ctypes.POINTER(P)]
        L.dtb_context_destroy.restype = None
        L.dtb_context_destroy.argtypes = [P]
        L.dtb_context_message.restype = ctypes.c_char_p
        L.dtb_context_message.argtypes = [P]
        L.dtb_last_stats.restype = I32
        L.dtb_last_stats.argtypes = [P, ctypes.POINTER(DtbStats)]
        L.dtb_sync.restype = I32
        L.dtb_sync.argtypes = [P, P]
        L.dtb_gdt_ref.restype = I32
        L.dtb_gdt_ref.argtypes = [P, IMG, IMG, IMG, F, F, U32, P]
        L.dtb_gdt.restype = I32
        L.dtb_gdt.argtypes = [P, IMG, IMG, IMG, F, F, U32, P]
        L.dtb_gdt_ref_blocks.restype = I32
        L.dtb_gdt_ref_blocks.argtypes = [P, IMG, IMG, IMG, F, F, P, U32, P]
        L.dtb_image_alloc.restype = I32
        L.dtb_image_alloc.argtypes = [I32, I32, I32, I32, ctypes.POINTER(DtbImage)]
        L.dtb_debug_inject_queue_stall.restype = I32
        L.dtb_debug_inject_queue_stall.argtypes = [P, U32]
        L.dtb_image_read.restype = I32
        L.dtb_image_read.argtypes = [ctypes.c_char_p, I32, ctypes.POINTER(DtbImage)]
        L.dtb_image_write.restype = I32
        L.dtb_image_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(DtbImage)]
        L.dtb_image_free.restype = I32
        L.dtb_image_free.argtypes = [ctypes.POINTER(DtbImage)]
        L.dtb_gdt_batch.restype = I32
        L.dtb_gdt_batch.argtypes = [P, I32, IMG, IMG, IMG, ctypes.POINTER(F), F, U32, P]
        L.dtb_context_set_tuning.restype = I32
        L.dtb_context_set_tuning.argtypes = [P, ctypes.POINTER(DtbTuning)]
        L.dtb_context_get_tuning.restype = I32
        L.dtb_context_get_tuning.argtypes = [P, ctypes.POINTER(DtbTuning)]
        L.dtb_plan_create.restype = I32
        L.dtb_plan_create.argtypes = [P, I32, IMG, IMG, IMG, ctypes.POINTER(F), F, U32, ctypes.POINTER(P)]
        L.dtb_plan_run.restype = I32
        L.dtb_plan_run.argtypes = [P, P]
        L.dtb_plan_wait.restype = I32
        L.dtb_plan_wait.argtypes = [P, P, ctypes.POINTER(DtbStats)]
        L.dtb_plan_autotune.restype = I32
        L.dtb_plan_autotune.argtypes = [P, P, I32, ctypes.POINTER(DtbTuning)]
        L.dtb_plan_get_tuning.restype = I32
        L.dtb_plan_get_tuning.argtypes = [P, ctypes.POINTER(DtbTuning)]
        L.dtb_context_set_tuning_cache.restype = I32
        L.dtb_context_set_tuning_cache.argtypes = [P, ctypes.c_char_p]
        L.dtb_plan_destroy.restype = None
        L.dtb_plan_destroy.argtypes = [P]
        L.dtb_serve_create.restype = I32
        L.dtb_serve_create.argtypes = [P, ctypes.POINTER(DtbServeConfig), ctypes.POINTER(P)]
        L.dtb_serve_submit.restype = I32
        L.dtb_serve_submit.argtypes = [P, ctypes.POINTER(DtbServeRequest), ctypes.POINTER(ctypes.c_int64)]
        L.dtb_serve_poll.restype = I32
        L.dtb_serve_poll.argtypes = [P, ctypes.POINTER(DtbServeCompletion), I32, I32]
        L.dtb_serve_release.restype = I32
        L.dtb_serve_release.argtypes = [P, ctypes.c_int64]
        L.dtb_serve_get_stats.restype = I32
        L.dtb_serve_get_stats.argtypes = [P, ctypes.POINTER(DtbServeStats)]
        L.dtb_serve_destroy.restype = None
        L.dtb_serve_destroy.argtypes = [P]
        L.dtb_gdt_noalloc.restype = I32
        L.dtb_gdt_noalloc.argtypes = [IMG, IMG, IMG, F, F, P]
        L.dtb_host_to_device.restype = I32
        L.dtb_host_to_device.argtypes = [IMG, IMG, P]
        L.dtb_device_to_host.restype = I32
        L.dtb_device_to_host.argtypes = [IMG, IMG, P]
        _lib = L
    return _lib


def declare_generator(H):
    """Declares the argument types of the generator entry points (csrc/datagen.cpp) on a loaded library."""
    P, I, I64, U64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
    H.dtbg_blobs_gray.restype = None
    H.dtbg_blobs_gray.argtypes = [U64, I, I, I, D, D, D, D, D, P, I64]
    H.dtbg_voronoi_rgb.restype = None
    H.dtbg_voronoi_rgb.argtypes = [U64, I, I, I, D, P, I64]
    H.dtbg_maze_gray.restype = I
    H.dtbg_maze_gray.argtypes = [U64, I, I, I, I, I, P, I64, ctypes.POINTER(I), ctypes.POINTER(I)]
    H.dtbg_draw_disks.restype = None
    H.dtbg_draw_disks.argtypes = [P, I64, I, I, I, P, P, P]
    return H


def host():
    """The host-only generator library."""
    global _host
    if _host is None:
        if not os.path.exists(LIBHOST_PATH):
            raise RuntimeError("libdtb_host.so is missing at %s: build it with __graft_entry__.build()" % LIBHOST_PATH)
        _host = declare_generator(ctypes.CDLL(LIBHOST_PATH))
    return _host
