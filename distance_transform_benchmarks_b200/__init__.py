"""B200-native generalised geodesic distance transform (GGDT).

Python mirror of the reference library's entry points (namespace ``dt``,
dt/include/dt/generalised_distance_transform.hpp:7-27 and dt/include/dt/transfert.hpp:9-17) over the C ABI
of include/dtb.h.  Torch tensors serve as containers (device memory, streams); every distance is computed by
the CUDA kernels in libdtb.so -- there is no fallback path.

Images are ``uint8`` tensors of shape ``[H, W]`` (gray) or ``[H, W, 3]`` (rgb8), seed masks ``uint8 [H, W]``
(non-zero = seed), distances ``float32 [H, W]``.  Rows may be padded (``stride(0)`` is the pitch).  Inputs on the
CPU are staged to the device by the library, as the reference's ``host_to_device`` does for its callers.
"""
import ctypes
import threading

import numpy as np
import torch

from ._native import (DTB_CPU, DTB_FLAG_ASYNC, DTB_FLAG_REF_NO_FMA, DTB_FLAG_ROUNDS, DTB_FLAG_TIMING, DTB_GPU,
                      DTB_REQ_EDIT, DTB_REQ_IMAGE, DtbError, DtbImage, DtbServeCompletion, DtbServeConfig,
                      DtbServeRequest, DtbServeStats, DtbStats, DtbTuning, lib)

__all__ = [
    "Context", "DtbError", "default_context", "generalised_distance_transform", "imread", "imsave",
    "generalised_distance_transform_blocks", "generalised_distance_transform_task", "geodesic_distance_transform",
    "geodesic_distance_transform_batch", "host_to_device", "device_to_host", "image_view", "DEFAULT_V", "BatchPlan",
    "pitched_empty", "pitched_from", "Server",
]

DEFAULT_V = 1e10  # reference default, generalised_distance_transform.hpp:8


class Context:
    """A dtb_context: owns the device scratch of the calls made through it."""

    def __init__(self, device=None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = int(device)
        self._h = ctypes.c_void_p()
        st = lib().dtb_context_create(self.device, ctypes.byref(self._h))
        if st != 0:
            raise DtbError(st, "dtb_context_create(%d) failed (an sm_100 device is required)" % self.device)

    @property
    def handle(self):
        return self._h

    def check(self, status):
        if status != 0:
            raise DtbError(status, lib().dtb_context_message(self._h).decode())

    def stats(self):
        s = DtbStats()
        self.check(lib().dtb_last_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in DtbStats._fields_}

    def set_tuning(self, ctas_per_sm=0, grid_percent=0, host_chunk_kpx=0, queue_buckets=0, bucket_width_pct=0, staging=0,
                   warps_per_cta=0):
        """dtb_context_set_tuning: 0 keeps a field (see include/dtb.h for the ranges)."""
        t = DtbTuning(ctas_per_sm, grid_percent, host_chunk_kpx, queue_buckets, bucket_width_pct, staging, warps_per_cta)
        self.check(lib().dtb_context_set_tuning(self._h, ctypes.byref(t)))

    def get_tuning(self):
        t = DtbTuning()
        self.check(lib().dtb_context_get_tuning(self._h, ctypes.byref(t)))
        return _tuning_dict(t)

    def set_tuning_cache(self, path):
        """dtb_context_set_tuning_cache: load this GPU's autotuner results from the JSON file at `path` and save
        new ones there (None turns the cache off)."""
        self.check(lib().dtb_context_set_tuning_cache(self._h, None if path is None else str(path).encode()))

    def sync(self, stream=None):
        self.check(lib().dtb_sync(self._h, ctypes.c_void_p(_stream_ptr(stream))))

    def inject_queue_stall(self, timeout_ms):
        """Failure-detection self-test: the next tile run of this context waits on a tile that is never queued,
        so its bounded queue wait (``timeout_ms``) ends the run with DTB_ERR_TIMEOUT (dtb_debug_inject_queue_stall)."""
        self.check(lib().dtb_debug_inject_queue_stall(self._h, int(timeout_ms)))

    def close(self):
        if self._h:
            lib().dtb_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _tuning_dict(t):
    return {f: getattr(t, f) for f, _ in DtbTuning._fields_}


_ctx_lock = threading.Lock()
_contexts = {}


def default_context(device=None):
    if device is None:
        device = torch.cuda.current_device()
    with _ctx_lock:
        c = _contexts.get(device)
        if c is None:
            c = _contexts[device] = Context(device)
        return c


def _stream_ptr(stream):
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def image_view(t, elem_size=None):
    """dtb_image view of a tensor ([H, W] or [H, W, C], rows contiguous)."""
    if isinstance(t, np.ndarray):
        t = torch.from_numpy(t)
    if t.dim() == 3:
        h, w, c = t.shape
        if t.stride(2) != 1 or t.stride(1) != c:
            raise ValueError("pixels of a [H, W, C] image must be contiguous")
    elif t.dim() == 2:
        h, w = t.shape
        c = 1
        if t.stride(1) != 1 and w > 1:
            raise ValueError("rows must be contiguous")
    else:
        raise ValueError("expected a [H, W] or [H, W, C] tensor")
    es = t.element_size() * c
    if elem_size is not None and es != elem_size:
        raise ValueError("element size %d, expected %d" % (es, elem_size))
    pitch = t.stride(0) * t.element_size() if h > 1 else w * es
    kind = DTB_GPU if t.is_cuda else DTB_CPU
    return DtbImage(t.data_ptr() if t.numel() else None, w, h, pitch, es, kind)


# dtb_image as a numpy record (same layout: 8-byte pointer, five int32, padded to 32 bytes).
_VIEW_DTYPE = np.dtype([("buffer", "<u8"), ("width", "<i4"), ("height", "<i4"), ("pitch", "<i4"), ("elem_size", "<i4"),
                        ("memory_kind", "<i4")], align=True)
assert _VIEW_DTYPE.itemsize == ctypes.sizeof(DtbImage)


def _batch_views(tensors, elem_sizes):
    """dtb_image array for a list of tensors (the same checks as image_view, one pass, no ctypes objects per
    image: a 1024-image batch costs about a third of building image_view structs one by one).  `elem_sizes`:
    the bytes per pixel allowed (e.g. (1, 3) for gray or rgb8 images)."""
    rows = []
    for t in tensors:
        shp = t.shape
        st = t.stride()
        nd = len(shp)
        if nd == 3:
            h, w, c = shp
            if st[2] != 1 or st[1] != c:
                raise ValueError("pixels of a [H, W, C] image must be contiguous")
        elif nd == 2:
            h, w = shp
            c = 1
            if st[1] != 1 and w > 1:
                raise ValueError("rows must be contiguous")
        else:
            raise ValueError("expected a [H, W] or [H, W, C] tensor")
        es = t.element_size()
        if es * c not in elem_sizes:
            raise ValueError("element size %d, expected one of %s" % (es * c, elem_sizes))
        rows.append((t.data_ptr() if h * w else 0, w, h, st[0] * es if h > 1 else w * es * c, es * c,
                     DTB_GPU if t.is_cuda else DTB_CPU))
    arr = np.array(rows, dtype=_VIEW_DTYPE)
    return arr, arr.ctypes.data_as(ctypes.POINTER(DtbImage))


PITCH_ALIGN = 128  # bytes; cudaMallocPitch-style rows, as the reference's GPU image2d (image2d_data_gpu.hpp:28)


def pitched_empty(height, width, channels=1, dtype=torch.uint8, device="cuda"):
    """Uninitialised [H, W] (or [H, W, C]) tensor whose rows start every PITCH_ALIGN bytes: the layout the TMA
    path reads without staging (the reference allocates GPU images the same way)."""
    es = torch.empty((), dtype=dtype).element_size()
    row = width * channels * es
    pitch_elems = (-(-max(row, 1) // PITCH_ALIGN) * PITCH_ALIGN) // es
    store = torch.empty((max(height, 1), pitch_elems), dtype=dtype, device=device)
    if channels == 1:
        return store[:height, :width]
    return torch.as_strided(store, (height, width, channels), (pitch_elems, channels, 1))


def host_batch_arena(imgs, masks, pin=True):
    """Packs a batch's host images and masks back to back into one (pinned) buffer per plane kind and allocates the
    distance maps back to back in a third one; returns (img_views, mask_views, dist_views), tensors viewing the
    arenas.  Adjacent packed planes are what the host-buffer pipeline moves as one copy per chunk and direction
    (a data loader that fills such arenas gets the full copy-engine bandwidth in both directions)."""
    imgs = [_as_tensor(i) for i in imgs]
    masks = [_as_tensor(m) for m in masks]

    def arena(shapes, dtype):
        sizes = [int(np.prod(shp)) for shp in shapes]
        buf = torch.empty(max(1, sum(sizes)), dtype=dtype)
        if pin:
            buf = buf.pin_memory()
        views, off = [], 0
        for shp, n in zip(shapes, sizes):
            views.append(buf[off:off + n].view(*shp))
            off += n
        return views

    iv = arena([tuple(t.shape) for t in imgs], torch.uint8)
    mv = arena([tuple(t.shape) for t in masks], torch.uint8)
    dv = arena([tuple(t.shape[:2]) for t in imgs], torch.float32)
    for a, b in zip(iv, imgs):
        a.copy_(b)
    for a, b in zip(mv, masks):
        a.copy_(b)
    return iv, mv, dv


def pitched_from(arr, device="cuda"):
    """Copy of a [H, W] / [H, W, C] array into a pitched device tensor."""
    t = _as_tensor(arr)
    c = t.shape[2] if t.dim() == 3 else 1
    out = pitched_empty(t.shape[0], t.shape[1], c, t.dtype, device)
    out.copy_(t)
    return out


def _as_tensor(x):
    if isinstance(x, np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(x))
    return x


def _dist_like(img, dist):
    if dist is not None:
        return dist
    h, w = img.shape[0], img.shape[1]
    return torch.empty((h, w), dtype=torch.float32, device=img.device)


def _ctx_for(t, ctx):
    if ctx is not None:
        return ctx
    dev = t.device.index if t.is_cuda else None
    return default_context(dev)


def _ref_call(img, mask, lam, v, dist, rounds, ctx, stream, fma, round_per_blocks=None):
    img, mask = _as_tensor(img), _as_tensor(mask)
    dist = _dist_like(img, dist)
    ctx = _ctx_for(img, ctx)
    if stream is None and img.is_cuda:
        stream = torch.cuda.current_stream(img.device)
    vi, vm, vd = image_view(img, 1), image_view(mask, 1), image_view(dist, 4)
    flags = (DTB_FLAG_ROUNDS if rounds else 0) | (0 if fma else DTB_FLAG_REF_NO_FMA)
    if round_per_blocks is not None:
        tiles = ((img.shape[1] + 31) // 32) * ((img.shape[0] + 31) // 32)
        if (round_per_blocks.dtype != torch.int32 or not round_per_blocks.is_contiguous()
                or round_per_blocks.numel() != tiles):
            raise ValueError("round_per_blocks must be a contiguous int32 tensor of %d tile counters" % tiles)
        ctx.check(lib().dtb_gdt_ref_blocks(ctx.handle, ctypes.byref(vi), ctypes.byref(vm), ctypes.byref(vd), float(lam),
                                           float(v), ctypes.c_void_p(round_per_blocks.data_ptr()), flags,
                                           ctypes.c_void_p(_stream_ptr(stream))))
        return dist
    ctx.check(lib().dtb_gdt_ref(ctx.handle, ctypes.byref(vi), ctypes.byref(vm), ctypes.byref(vd), float(lam), float(v),
                                flags, ctypes.c_void_p(_stream_ptr(stream))))
    return dist


def generalised_distance_transform(img, mask, lam, v=DEFAULT_V, dist=None, *, ctx=None, stream=None, fma=True):
    """Reference weight (C8, lambda blend): dt::generalised_distance_transform
    (reference dt/src/generalised_distance_transform.cu:101-148).  Returns ``dist`` (allocated if None)."""
    return _ref_call(img, mask, lam, v, dist, False, ctx, stream, fma)


def generalised_distance_transform_blocks(img, mask, lam, v=DEFAULT_V, dist=None, round_per_blocks=None, *, ctx=None,
                                          stream=None, fma=True):
    """dt::generalised_distance_transform_blocks (reference _blocks.cu:114-184): host-driven rounds over active
    tiles.  Same result as the other two variants.  ``round_per_blocks``: optional int32 tensor (host or device)
    of ceil(W/32)*ceil(H/32) counters, incremented once per round in which the tile was visited."""
    return _ref_call(img, mask, lam, v, dist, True, ctx, stream, fma, round_per_blocks)


def generalised_distance_transform_task(img, mask, lam, v=DEFAULT_V, dist=None, *, ctx=None, stream=None, fma=True):
    """dt::generalised_distance_transform_task (reference _task.cu:152-207): persistent tile queue."""
    return _ref_call(img, mask, lam, v, dist, False, ctx, stream, fma)


def geodesic_distance_transform(img, mask, gamma, v=DEFAULT_V, dist=None, *, rounds=False, ctx=None, stream=None):
    """C4 geodesic distance with w = sqrt(1 + gamma^2 |dI|^2), gray or rgb8 (dtb_gdt)."""
    img, mask = _as_tensor(img), _as_tensor(mask)
    dist = _dist_like(img, dist)
    ctx = _ctx_for(img, ctx)
    if stream is None and img.is_cuda:
        stream = torch.cuda.current_stream(img.device)
    es = 3 if img.dim() == 3 else 1
    vi, vm, vd = image_view(img, es), image_view(mask, 1), image_view(dist, 4)
    ctx.check(lib().dtb_gdt(ctx.handle, ctypes.byref(vi), ctypes.byref(vm), ctypes.byref(vd), float(gamma), float(v),
                            DTB_FLAG_ROUNDS if rounds else 0, ctypes.c_void_p(_stream_ptr(stream))))
    return dist


def geodesic_distance_transform_batch(imgs, masks, gammas, v=DEFAULT_V, dists=None, *, rounds=False, ctx=None,
                                      stream=None, asynchronous=False, timing=False):
    """Ragged batch in one persistent launch over a shared tile queue (dtb_gdt_batch).  With host tensors the
    batch streams through the host-buffer pipeline.  ``asynchronous``: return after enqueueing (device tensors,
    or all-host batches); ``ctx.sync(stream)`` waits and raises on a device error; the tensors must stay alive
    and untouched until then."""
    n = len(imgs)
    imgs = [_as_tensor(t) for t in imgs]
    masks = [_as_tensor(t) for t in masks]
    if dists is None:
        dists = [_dist_like(t, None) for t in imgs]
    if n == 0:
        return dists
    ctx = _ctx_for(imgs[0], ctx)
    if stream is None and imgs[0].is_cuda:
        stream = torch.cuda.current_stream(imgs[0].device)
    if len(masks) != n or len(dists) != n or len(gammas) != n:
        raise ValueError("imgs, masks, gammas and dists must have the same length")
    keep_i, vi = _batch_views(imgs, (1, 3))
    keep_m, vm = _batch_views(masks, (1,))
    keep_d, vd = _batch_views(dists, (4,))
    g = np.asarray(gammas, dtype=np.float32)
    flags = (DTB_FLAG_ROUNDS if rounds else 0) | (DTB_FLAG_ASYNC if asynchronous else 0) | \
        (DTB_FLAG_TIMING if timing else 0)
    ctx.check(lib().dtb_gdt_batch(ctx.handle, n, vi, vm, vd, g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(v),
                                  flags, ctypes.c_void_p(_stream_ptr(stream))))
    return dists


def imread(path, channels=1):
    """dt::imread (reference dt/src/imread.cpp): an 8-bit PNG / PGM / PPM / JPEG file as a uint8 array, [H, W] for
    channels=1 (the file must be gray), [H, W, 3] for channels=3 (rgb, palette or colour JPEG).  Gray JPEG samples
    are identical to those of stb_image, the reference's decoder."""
    im = DtbImage()
    st = lib().dtb_image_read(str(path).encode(), int(channels), ctypes.byref(im))
    if st != 0:
        raise DtbError(st, "cannot read %s as a %d-channel 8-bit image" % (path, channels))
    try:
        buf = (ctypes.c_uint8 * (im.pitch * im.height)).from_address(im.buffer)
        a = np.frombuffer(buf, dtype=np.uint8).reshape(im.height, im.pitch)[:, :im.width * channels]
        out = a.reshape(im.height, im.width, channels).copy() if channels == 3 else a.copy()
    finally:
        lib().dtb_image_free(ctypes.byref(im))
    return out


def imsave(path, img):
    """dt::imsave (reference dt/src/imsave.cpp): a uint8 [H, W] or [H, W, 3] array (or tensor) to .png, .pgm
    (gray) or .ppm (rgb8)."""
    t = _as_tensor(img)
    if t.is_cuda:
        t = t.cpu()
    t = t.contiguous()
    view = image_view(t, 3 if t.dim() == 3 else 1)
    st = lib().dtb_image_write(str(path).encode(), ctypes.byref(view))
    if st != 0:
        raise DtbError(st, "cannot write %s" % path)


def host_to_device(t, stream=None):
    """dt::host_to_device (reference dt/src/transfert.cpp:10-18): pitched copy into new device memory."""
    t = _as_tensor(t)
    out = torch.empty_like(t, device="cuda")
    es = t.element_size() * (t.shape[2] if t.dim() == 3 else 1)
    st = lib().dtb_host_to_device(ctypes.byref(image_view(t, es)), ctypes.byref(image_view(out, es)),
                                  ctypes.c_void_p(_stream_ptr(stream)))
    if st != 0:
        raise DtbError(st, "Unable to transfert host to device")
    return out


def device_to_host(t, stream=None):
    """dt::device_to_host (reference dt/src/transfert.cpp:20-28)."""
    out = torch.empty_like(t, device="cpu")
    es = t.element_size() * (t.shape[2] if t.dim() == 3 else 1)
    st = lib().dtb_device_to_host(ctypes.byref(image_view(t, es)), ctypes.byref(image_view(out, es)),
                                  ctypes.c_void_p(_stream_ptr(stream)))
    if st != 0:
        raise DtbError(st, "Unable to transfert device to host")
    return out


class BatchPlan:
    """dtb_plan: a ragged batch of device tensors prepared once (descriptors, TMA tensor maps, scratch) and
    captured in a CUDA graph; run() launches the graph, wait() returns the device status and counters."""

    def __init__(self, imgs, masks, gammas, v=DEFAULT_V, dists=None, *, ctx=None):
        n = len(imgs)
        if dists is None:
            dists = [_dist_like(t, None) for t in imgs]
        self.imgs, self.masks, self.dists = list(imgs), list(masks), list(dists)  # keep the buffers alive
        self.ctx = ctx if ctx is not None else _ctx_for(imgs[0], None)
        vi = (DtbImage * n)(*[image_view(t, 3 if t.dim() == 3 else 1) for t in self.imgs])
        vm = (DtbImage * n)(*[image_view(t, 1) for t in self.masks])
        vd = (DtbImage * n)(*[image_view(t, 4) for t in self.dists])
        g = (ctypes.c_float * n)(*[float(x) for x in gammas])
        self._h = ctypes.c_void_p()
        self.ctx.check(lib().dtb_plan_create(self.ctx.handle, n, vi, vm, vd, g, float(v), 0, ctypes.byref(self._h)))

    def run(self, stream=None):
        if stream is None:
            stream = torch.cuda.current_stream()
        self.ctx.check(lib().dtb_plan_run(self._h, ctypes.c_void_p(_stream_ptr(stream))))

    def wait(self, stream=None):
        if stream is None:
            stream = torch.cuda.current_stream()
        s = DtbStats()
        self.ctx.check(lib().dtb_plan_wait(self._h, ctypes.c_void_p(_stream_ptr(stream)), ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in DtbStats._fields_}

    def autotune(self, reps=3, stream=None):
        if stream is None:
            stream = torch.cuda.current_stream()
        t = DtbTuning()
        self.ctx.check(lib().dtb_plan_autotune(self._h, ctypes.c_void_p(_stream_ptr(stream)), int(reps), ctypes.byref(t)))
        return _tuning_dict(t)

    def tuning(self):
        t = DtbTuning()
        self.ctx.check(lib().dtb_plan_get_tuning(self._h, ctypes.byref(t)))
        return _tuning_dict(t)

    def close(self):
        if self._h:
            lib().dtb_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """dtb_server: continuous batching of new-image and seed-edit requests (see include/dtb.h).  Inputs and the
    output map are host tensors (pinned memory copies fastest); they are kept alive here until the request's
    completion has been polled.  live=True: requests join the tile queue of one persistent kernel that keeps
    running (live admission) instead of running in waves."""

    def __init__(self, hbm_budget_bytes, *, max_wave_requests=0, v=DEFAULT_V, max_wave_tiles=0, wave_stage_bytes=0,
                 live=False, live_idle_us=0, ctx=None, device=0):
        self.ctx = ctx if ctx is not None else default_context(device)
        cfg = DtbServeConfig(int(hbm_budget_bytes), int(max_wave_requests), float(v), int(max_wave_tiles),
                             int(wave_stage_bytes), 1 if live else 0, int(live_idle_us))
        self._h = ctypes.c_void_p()
        st = lib().dtb_serve_create(self.ctx.handle, ctypes.byref(cfg), ctypes.byref(self._h))
        if st != 0:
            raise DtbError(st, "dtb_serve_create failed")
        self._alive = {}

    def _submit(self, req, keep):
        rid = ctypes.c_int64()
        st = lib().dtb_serve_submit(self._h, ctypes.byref(req), ctypes.byref(rid))
        if st != 0:
            raise DtbError(st, "dtb_serve_submit rejected the request")
        self._alive[rid.value] = keep
        return rid.value

    def submit_image(self, image_id, img, mask, gamma, out):
        img, mask = _as_tensor(img), _as_tensor(mask)
        req = DtbServeRequest()
        req.kind = DTB_REQ_IMAGE
        req.image_id = int(image_id)
        req.img = image_view(img, 3 if img.dim() == 3 else 1)
        req.mask = image_view(mask, 1)
        req.gamma = float(gamma)
        req.out = image_view(out, 4)
        return self._submit(req, (img, mask, out))

    def submit_edit(self, image_id, disks, out):
        arr = (ctypes.c_int32 * (3 * len(disks)))(*[int(v) for d in disks for v in d])
        req = DtbServeRequest()
        req.kind = DTB_REQ_EDIT
        req.image_id = int(image_id)
        req.n_disks = len(disks)
        req.disks = ctypes.cast(arr, ctypes.POINTER(ctypes.c_int32))
        req.out = image_view(out, 4)
        return self._submit(req, (out,))

    def poll(self, max_items=256, wait_ms=0):
        buf = (DtbServeCompletion * max_items)()
        k = lib().dtb_serve_poll(self._h, buf, max_items, int(wait_ms))
        out = []
        for c in buf[:k]:
            self._alive.pop(c.request_id, None)
            out.append({"request_id": c.request_id, "status": c.status, "latency_ms": c.latency_ms})
        return out

    def release(self, image_id):
        return lib().dtb_serve_release(self._h, int(image_id))

    def stats(self):
        s = DtbServeStats()
        lib().dtb_serve_get_stats(self._h, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in DtbServeStats._fields_}

    def close(self):
        if self._h:
            lib().dtb_serve_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._alive.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
