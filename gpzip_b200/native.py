"""ctypes binding of the C ABI in include/gpz.h (libgpz.so, built for sm_100a).

There is no fallback: if the shared library is missing or no CUDA device is
usable, loading or creating a context raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpz.so")

GPZ_OK = 0
STATUS = {0: "GPZ_OK", 1: "GPZ_E_NOMEM", 2: "GPZ_E_ADMISSION", 3: "GPZ_E_TIMEOUT", 4: "GPZ_E_CUDA",
          5: "GPZ_E_ARG", 6: "GPZ_E_SPACE", 7: "GPZ_E_INTERNAL", 8: "GPZ_E_BUSY", 9: "GPZ_E_PENDING",
          10: "GPZ_E_DATA", 11: "GPZ_E_SINK"}
GPZ_E_DATA = 10
GPZ_E_SINK = 11
# gpz_sink_fn / gpz_chunk_fn
SINK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t)
CHUNK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t,
                            ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t))
GPZ_E_PENDING = 9
GPZ_E_BUSY = 8
GPZ_E_ADMISSION = 2
GPZ_E_TIMEOUT = 3
GPZ_CODEC_GZIP = 0
GPZ_CODEC_ZSTD = 1
GPZ_FLAG_NO_GRAPHS = 1
GPZ_FLAG_NO_AUTOTUNE = 2
GPZ_FLAG_STAGE_TIMING = 4
GPZ_FLAG_SM_PARTITION = 8
GPZ_FLAG_FIXED_BLOCKS = 16
# gpz_stage_times order (GPZ_STAGES values): the kernels each stage covers
STAGE_NAMES = ["k_segtab", "k_lookup", "k_walk", "k_huff", "k_emit"]
# the same stages of a zstd context (the last two: blocks + placement, copy)
STAGE_NAMES_ZSTD = ["k_segtab", "k_lookup", "k_walk", "k_zblock", "k_zcopy"]

# Every symbol include/gpz.h declares.
EXPORTS = [
    "gpz_config_default", "gpz_create", "gpz_destroy", "gpz_bound", "gpz_bound_ctx", "gpz_compress_chunk",
    "gpz_compress_batch", "gpz_compress_batch_plain", "gpz_compress_device", "gpz_frame_host",
    "gpz_debug_chunk", "gpz_submit", "gpz_poll", "gpz_serve_stats_get", "gpz_strerror", "gpz_last_error",
    "gpz_get_shape", "gpz_set_shape", "gpz_last_launches", "gpz_stage_times", "gpz_compress_member_static",
    "gpz_serve_reset_stats", "gpz_submit_ref", "gpz_host_times", "gpz_serve_lane_stats",
    "gpz_inflate_size", "gpz_inflate", "gpz_inflate_device_ms",
    "gpz_writer_open", "gpz_writer_open_fn", "gpz_writer_write", "gpz_writer_flush", "gpz_writer_finish",
    "gpz_writer_close", "gpz_set_wait_ms", "gpz_hybrid_config_default", "gpz_hybrid_create", "gpz_hybrid_chunk",
    "gpz_hybrid_stats", "gpz_hybrid_destroy", "gpz_cpu_gzip_chunk",
]


class GpzError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("member_bytes", ctypes.c_size_t), ("pool_bytes", ctypes.c_size_t),
                ("batch_bytes", ctypes.c_size_t), ("streams", ctypes.c_int), ("flags", ctypes.c_int),
                ("wait_ms", ctypes.c_int), ("codec", ctypes.c_int)]


class HybridConfig(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("device", ctypes.c_int), ("level", ctypes.c_int),
                ("gpu_permits", ctypes.c_size_t), ("warmup_chunks", ctypes.c_size_t), ("cpu_fn", ctypes.c_void_p),
                ("cpu_user", ctypes.c_void_p), ("gpu_fn", ctypes.c_void_p), ("gpu_user", ctypes.c_void_p)]


class Desc(ctypes.Structure):
    _fields_ = [("in_", ctypes.c_void_p), ("n", ctypes.c_size_t), ("level", ctypes.c_int)]


class Out(ctypes.Structure):
    _fields_ = [("out", ctypes.c_void_p), ("out_cap", ctypes.c_size_t), ("out_len", ctypes.c_size_t),
                ("status", ctypes.c_int)]


class Shape(ctypes.Structure):
    _fields_ = [("lookup_threads", ctypes.c_int), ("lookup_grid", ctypes.c_int), ("walk_threads", ctypes.c_int),
                ("walk_grid", ctypes.c_int), ("emit_threads", ctypes.c_int), ("emit_grid", ctypes.c_int)]


class ServeStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("p999_ms", ctypes.c_double),
                ("max_queue_ms", ctypes.c_double), ("bytes_in", ctypes.c_uint64), ("bytes_out", ctypes.c_uint64),
                ("completed_small", ctypes.c_uint64), ("p50_small_ms", ctypes.c_double),
                ("p99_small_ms", ctypes.c_double), ("p999_small_ms", ctypes.c_double),
                ("queued_bytes", ctypes.c_uint64)]


class LaneStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_uint64), ("units", ctypes.c_uint64), ("bytes", ctypes.c_uint64),
                ("queue_ms", ctypes.c_double), ("submit_ms", ctypes.c_double), ("h2d_ms", ctypes.c_double),
                ("kernel_ms", ctypes.c_double), ("wait_ms", ctypes.c_double), ("complete_ms", ctypes.c_double),
                ("max_queue_ms", ctypes.c_double), ("max_batch_ms", ctypes.c_double)]


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libgpz.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m gpzip_b200.build`")
    L = ctypes.CDLL(path)
    vp, sz, u64p = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)
    L.gpz_config_default.argtypes = [ctypes.POINTER(Config)]
    L.gpz_config_default.restype = None
    L.gpz_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
    L.gpz_create.restype = ctypes.c_int
    L.gpz_destroy.argtypes = [vp]
    L.gpz_destroy.restype = None
    L.gpz_bound.argtypes = [sz]
    L.gpz_bound.restype = sz
    L.gpz_bound_ctx.argtypes = [vp, sz]
    L.gpz_bound_ctx.restype = sz
    L.gpz_compress_chunk.argtypes = [vp, vp, sz, ctypes.c_int, vp, sz, ctypes.POINTER(sz)]
    L.gpz_compress_chunk.restype = ctypes.c_int
    L.gpz_compress_batch.argtypes = [vp, ctypes.POINTER(Desc), sz, ctypes.POINTER(Out)]
    L.gpz_compress_batch.restype = ctypes.c_int
    L.gpz_compress_batch_plain.argtypes = [vp, ctypes.POINTER(Desc), sz, ctypes.POINTER(Out)]
    L.gpz_compress_batch_plain.restype = ctypes.c_int
    L.gpz_compress_device.argtypes = [vp, vp, u64p, u64p, sz, vp, sz, u64p, vp]
    L.gpz_compress_device.restype = ctypes.c_int
    L.gpz_frame_host.argtypes = [vp, vp, sz]
    L.gpz_frame_host.restype = ctypes.c_int
    L.gpz_debug_chunk.argtypes = [vp, vp, sz, vp, vp, ctypes.POINTER(sz), vp, sz, ctypes.POINTER(sz)]
    L.gpz_debug_chunk.restype = ctypes.c_int
    L.gpz_submit.argtypes = [vp, ctypes.POINTER(Desc), ctypes.POINTER(ctypes.c_uint64)]
    L.gpz_submit.restype = ctypes.c_int
    L.gpz_poll.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(Out), ctypes.c_int]
    L.gpz_poll.restype = ctypes.c_int
    L.gpz_serve_stats_get.argtypes = [vp, ctypes.POINTER(ServeStats)]
    L.gpz_serve_stats_get.restype = ctypes.c_int
    L.gpz_serve_reset_stats.argtypes = [vp]
    L.gpz_serve_reset_stats.restype = ctypes.c_int
    L.gpz_submit_ref.argtypes = [vp, ctypes.POINTER(Desc), ctypes.POINTER(ctypes.c_uint64)]
    L.gpz_submit_ref.restype = ctypes.c_int
    L.gpz_serve_lane_stats.argtypes = [vp, ctypes.c_int, ctypes.POINTER(LaneStats)]
    L.gpz_serve_lane_stats.restype = ctypes.c_int
    L.gpz_host_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    L.gpz_host_times.restype = ctypes.c_int
    L.gpz_inflate_size.argtypes = [vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz)]
    L.gpz_inflate_size.restype = ctypes.c_int
    L.gpz_inflate.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(sz)]
    L.gpz_inflate.restype = ctypes.c_int
    L.gpz_inflate_device_ms.argtypes = [vp]
    L.gpz_inflate_device_ms.restype = ctypes.c_float
    L.gpz_writer_open.argtypes = [vp, sz, sz, SINK_FN, vp, ctypes.POINTER(vp)]
    L.gpz_writer_open.restype = ctypes.c_int
    L.gpz_writer_open_fn.argtypes = [CHUNK_FN, vp, sz, sz, SINK_FN, vp, ctypes.POINTER(vp)]
    L.gpz_writer_open_fn.restype = ctypes.c_int
    L.gpz_writer_write.argtypes = [vp, vp, sz]
    L.gpz_writer_write.restype = ctypes.c_int
    for f in (L.gpz_writer_flush, L.gpz_writer_finish):
        f.argtypes = [vp]
        f.restype = ctypes.c_int
    L.gpz_writer_close.argtypes = [vp]
    L.gpz_writer_close.restype = None
    L.gpz_strerror.argtypes = [ctypes.c_int]
    L.gpz_strerror.restype = ctypes.c_char_p
    L.gpz_last_error.argtypes = [vp]
    L.gpz_last_error.restype = ctypes.c_char_p
    L.gpz_get_shape.argtypes = [vp, ctypes.POINTER(Shape)]
    L.gpz_get_shape.restype = ctypes.c_int
    L.gpz_set_shape.argtypes = [vp, ctypes.POINTER(Shape)]
    L.gpz_set_shape.restype = ctypes.c_int
    L.gpz_last_launches.argtypes = [vp]
    L.gpz_last_launches.restype = ctypes.c_uint64
    L.gpz_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.gpz_stage_times.restype = ctypes.c_int
    L.gpz_compress_member_static.argtypes = [vp, sz, vp, sz, ctypes.POINTER(sz), vp]
    L.gpz_compress_member_static.restype = ctypes.c_int
    L.gpz_set_wait_ms.argtypes = [vp, ctypes.c_int]
    L.gpz_set_wait_ms.restype = ctypes.c_int
    L.gpz_hybrid_config_default.argtypes = [ctypes.POINTER(HybridConfig)]
    L.gpz_hybrid_config_default.restype = None
    L.gpz_hybrid_create.argtypes = [ctypes.POINTER(HybridConfig), ctypes.POINTER(vp)]
    L.gpz_hybrid_create.restype = ctypes.c_int
    L.gpz_hybrid_chunk.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(sz)]
    L.gpz_hybrid_chunk.restype = ctypes.c_int
    L.gpz_hybrid_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.gpz_hybrid_stats.restype = ctypes.c_int
    L.gpz_hybrid_destroy.argtypes = [vp]
    L.gpz_hybrid_destroy.restype = None
    L.gpz_cpu_gzip_chunk.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(sz)]
    L.gpz_cpu_gzip_chunk.restype = ctypes.c_int
    _lib = L
    return L


def _u8(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
    return np.frombuffer(bytes(data), dtype=np.uint8)


def inflate_size(data):
    """(members, output bytes) of a gzip stream written by gpzip, from its
    headers and ISIZE trailers (host only).  Raises GpzError (GPZ_E_DATA)
    when the stream does not start with gpzip's header."""
    L = load()
    a = _u8(data)
    m, t = ctypes.c_size_t(), ctypes.c_size_t()
    rc = L.gpz_inflate_size(_p(a), a.size, ctypes.byref(m), ctypes.byref(t))
    if rc:
        raise GpzError(rc, "gpz_inflate_size")
    return m.value, t.value


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a.size else ctypes.c_void_p(0)


class Context:
    """One gpz_ctx (device pool, streams, launch shapes) on one CUDA device."""

    def __init__(self, device: int = 0, member_bytes: int = 128 * 1024, pool_bytes: int = 0,
                 batch_bytes: int = 0, flags: int = 0, wait_ms: int = 0, codec: int = GPZ_CODEC_GZIP):
        L = load()
        cfg = Config()
        L.gpz_config_default(ctypes.byref(cfg))
        cfg.device, cfg.member_bytes, cfg.pool_bytes = device, member_bytes, pool_bytes
        cfg.batch_bytes, cfg.flags, cfg.wait_ms, cfg.codec = batch_bytes, flags, wait_ms, codec
        h = ctypes.c_void_p()
        rc = L.gpz_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != GPZ_OK:
            raise GpzError(rc, "gpz_create")
        self._h = h
        self.member_bytes = member_bytes
        self.L = L

    def close(self):
        if getattr(self, "_h", None):
            self.L.gpz_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != GPZ_OK:
            raise GpzError(rc, f"{what}: {self.L.gpz_last_error(self._h).decode()}")

    def bound(self, n: int) -> int:
        return self.L.gpz_bound_ctx(self._h, n)

    def set_wait_ms(self, ms: int):
        """Bound of every wait for the device (0: give up at once unless the
        work is done; such a call raises GpzError with GPZ_E_TIMEOUT)."""
        self._check(self.L.gpz_set_wait_ms(self._h, ms), "gpz_set_wait_ms")

    def compress_chunk(self, data, level: int = 5) -> bytes:
        a = _u8(data)
        cap = self.bound(a.size)
        out = np.empty(cap, dtype=np.uint8)
        n = ctypes.c_size_t()
        self._check(self.L.gpz_compress_chunk(self._h, _p(a), a.size, level, _p(out), cap, ctypes.byref(n)),
                    "gpz_compress_chunk")
        return out[:n.value].tobytes()

    def batch_bound(self, items) -> int:
        """Output bytes compress_batch needs for these items (sum of bounds)."""
        return max(1, sum(self.bound(len(x)) for x in items))

    def _batch(self, fn, items, level: int = 5, out=None):
        """One output buffer for all items (`out`, a uint8 array of at least
        batch_bound(items) bytes that the caller may reuse across calls, or a
        fresh allocation); results are zero-copy views into it."""
        arrs = [_u8(x) for x in items]
        k = len(arrs)
        descs = (Desc * max(k, 1))()
        outs = (Out * max(k, 1))()
        bounds = [self.bound(a.size) for a in arrs]
        if out is None:
            out = np.empty(max(1, sum(bounds)), dtype=np.uint8)
        elif out.dtype != np.uint8 or not out.flags.c_contiguous or out.size < sum(bounds):
            raise ValueError("out must be a contiguous uint8 array of at least batch_bound(items) bytes")
        base = out.ctypes.data
        off = 0
        for i, a in enumerate(arrs):
            descs[i].in_ = a.ctypes.data if a.size else None
            descs[i].n = a.size
            descs[i].level = level
            outs[i].out = base + off
            outs[i].out_cap = bounds[i]
            off += bounds[i]
        self._check(fn(self._h, descs, k, outs), fn.__name__)
        mv = memoryview(out)
        res, off = [], 0
        for i in range(k):
            res.append(mv[off:off + outs[i].out_len])
            off += bounds[i]
        return res

    def compress_batch(self, items, level: int = 5, out=None):
        return self._batch(self.L.gpz_compress_batch, items, level, out)

    def compress_batch_plain(self, items, level: int = 5, out=None):
        return self._batch(self.L.gpz_compress_batch_plain, items, level, out)

    def debug_chunk(self, data):
        """(pp, tokens, gzip bytes) of one chunk through the device path."""
        a = _u8(data)
        pp = np.zeros(max(a.size, 1), dtype=np.uint32)
        tok = np.zeros(max(a.size, 1), dtype=np.uint32)
        ntok = ctypes.c_size_t()
        cap = self.bound(a.size)
        out = np.empty(cap, dtype=np.uint8)
        olen = ctypes.c_size_t()
        self._check(self.L.gpz_debug_chunk(self._h, _p(a), a.size, _p(pp), _p(tok), ctypes.byref(ntok), _p(out),
                                           cap, ctypes.byref(olen)), "gpz_debug_chunk")
        return pp[:a.size], tok[:ntok.value], out[:olen.value].tobytes()

    def compress_device(self, d_in: int, offs, lens, d_out: int, out_cap: int, stream: int = 0):
        """Device-resident pass; returns (count+1) output offsets."""
        k = len(offs)
        o = (ctypes.c_uint64 * k)(*offs)
        l = (ctypes.c_uint64 * k)(*lens)
        r = (ctypes.c_uint64 * (k + 1))()
        self._check(self.L.gpz_compress_device(self._h, ctypes.c_void_p(d_in), o, l, k, ctypes.c_void_p(d_out),
                                               out_cap, r, ctypes.c_void_p(stream or None)), "gpz_compress_device")
        return list(r)

    def frame_host(self, host_out: np.ndarray):
        self._check(self.L.gpz_frame_host(self._h, _p(host_out), host_out.size), "gpz_frame_host")

    def get_shape(self) -> Shape:
        s = Shape()
        self._check(self.L.gpz_get_shape(self._h, ctypes.byref(s)), "gpz_get_shape")
        return s

    def set_shape(self, s: Shape):
        self._check(self.L.gpz_set_shape(self._h, ctypes.byref(s)), "gpz_set_shape")

    def last_launches(self) -> int:
        return self.L.gpz_last_launches(self._h)

    def stage_times(self):
        """Device ms of each stage of the last pass (STAGE_NAMES order)."""
        a = (ctypes.c_float * len(STAGE_NAMES))()
        self._check(self.L.gpz_stage_times(self._h, a), "gpz_stage_times")
        return list(a)

    def submit(self, data, level: int = 5) -> int:
        a = _u8(data)
        d = Desc(a.ctypes.data if a.size else None, a.size, level)
        t = ctypes.c_uint64()
        rc = self.L.gpz_submit(self._h, ctypes.byref(d), ctypes.byref(t))
        if rc != GPZ_OK:
            raise GpzError(rc, "gpz_submit")
        return t.value

    def poll(self, ticket: int, cap: int, wait_ms: int = 0):
        """The gzip stream of a submitted request, or None while pending."""
        buf = np.empty(max(cap, 1), dtype=np.uint8)
        o = Out(buf.ctypes.data, cap, 0, 0)
        rc = self.L.gpz_poll(self._h, ticket, ctypes.byref(o), wait_ms)
        if rc == GPZ_E_PENDING:
            return None
        if rc == 6:  # GPZ_E_SPACE: the result is kept; retry with the size needed
            buf = np.empty(o.out_len, dtype=np.uint8)
            o = Out(buf.ctypes.data, o.out_len, 0, 0)
            rc = self.L.gpz_poll(self._h, ticket, ctypes.byref(o), wait_ms)
        self._check(rc, "gpz_poll")
        return buf[:o.out_len].tobytes()

    def inflate(self, data, out=None):
        """Decompresses a gzip stream written by gpzip on the device (one warp
        per member).  `out`: optional reusable uint8 array of at least the
        output size; the result is a view into it.  Raises GpzError with
        GPZ_E_DATA when the stream cannot be split or a member fails."""
        a = _u8(data)
        if out is None:
            _, total = inflate_size(a)
            out = np.empty(max(total, 1), dtype=np.uint8)
        elif out.dtype != np.uint8 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous uint8 array")
        n = ctypes.c_size_t()
        self._check(self.L.gpz_inflate(self._h, _p(a), a.size, _p(out), out.size, ctypes.byref(n)), "gpz_inflate")
        return memoryview(out)[:n.value]

    def inflate_device_ms(self) -> float:
        return float(self.L.gpz_inflate_device_ms(self._h))

    def host_times(self, reset: bool = False) -> dict:
        a = (ctypes.c_double * 6)()
        self._check(self.L.gpz_host_times(self._h, a, int(reset)), "gpz_host_times")
        return dict(zip(["plan_ms", "copy_in_ms", "enqueue_ms", "wait_ms", "copy_out_ms", "passes"], list(a)))

    def serve_reset_stats(self):
        self._check(self.L.gpz_serve_reset_stats(self._h), "gpz_serve_reset_stats")

    def lane_stats(self, lane: int) -> dict:
        """Per-lane serving breakdown (lane 0: requests <= 1 MiB); times are
        per-batch means in ms, maxima per batch."""
        s = LaneStats()
        self._check(self.L.gpz_serve_lane_stats(self._h, lane, ctypes.byref(s)), "gpz_serve_lane_stats")
        d = {f: getattr(s, f) for f, _ in LaneStats._fields_}
        b = max(1, d["batches"])
        for k in ("queue_ms", "submit_ms", "h2d_ms", "kernel_ms", "wait_ms", "complete_ms"):
            d[k] = d[k] / b
        return d

    def serve_stats(self) -> dict:
        s = ServeStats()
        self._check(self.L.gpz_serve_stats_get(self._h, ctypes.byref(s)), "gpz_serve_stats_get")
        return {f: getattr(s, f) for f, _ in ServeStats._fields_}


def cpu_gzip_chunk(data, level: int = 5) -> bytes:
    """gpz_cpu_gzip_chunk: one zlib gzip member of `data` at `level` (the
    CPU chunk function of the hybrid backend)."""
    L = load()
    a = _u8(data)
    cap = L.gpz_bound(a.size)
    out = np.empty(cap, dtype=np.uint8)
    n = ctypes.c_size_t()
    lv = ctypes.c_int(level)
    rc = L.gpz_cpu_gzip_chunk(ctypes.byref(lv), _p(a), a.size, _p(out), cap, ctypes.byref(n))
    if rc:
        raise GpzError(rc, "gpz_cpu_gzip_chunk")
    return out[:n.value].tobytes()


def _py_chunk_fn(f):
    """A gpz_chunk_fn that calls f(bytes) -> bytes (a raise or a short
    buffer is a nonzero status)."""
    def call(_user, buf, n, out, cap, out_len):
        try:
            g = bytes(f(ctypes.string_at(buf, n)))
        except Exception:  # noqa: BLE001 -- the status carries the failure
            return 1
        if len(g) > cap:
            return 1
        ctypes.memmove(out, g, len(g))
        out_len[0] = len(g)
        return 0
    return CHUNK_FN(call)


class Hybrid:
    """gpz_hybrid: the `--backend auto` chunk function (CPU and GPU chunks by
    permit).  `ctx`: a Context to use for GPU chunks (None: the library makes
    one on `device` at the first GPU chunk).  `cpu_fn` / `gpu_fn`: Python
    chunk functions (bytes -> gzip bytes) that replace either side, e.g. a
    stand-in device in tests.  Pass it to Writer(hybrid=...)."""

    def __init__(self, ctx: "Context" = None, device: int = 0, level: int = 5, gpu_permits: int = 1,
                 warmup_chunks: int = 4, cpu_fn=None, gpu_fn=None):
        self.L = load()
        cfg = HybridConfig()
        self.L.gpz_hybrid_config_default(ctypes.byref(cfg))
        cfg.ctx = ctx._h.value if ctx is not None else None
        cfg.device, cfg.level, cfg.gpu_permits, cfg.warmup_chunks = device, level, gpu_permits, warmup_chunks
        self._fns = [_py_chunk_fn(f) if f is not None else None for f in (cpu_fn, gpu_fn)]  # kept alive
        if cpu_fn is not None:
            cfg.cpu_fn = ctypes.cast(self._fns[0], ctypes.c_void_p).value
        if gpu_fn is not None:
            cfg.gpu_fn = ctypes.cast(self._fns[1], ctypes.c_void_p).value
        self._ctx = ctx  # kept alive with the hybrid
        self.gpu_permits = gpu_permits
        h = ctypes.c_void_p()
        rc = self.L.gpz_hybrid_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc:
            raise GpzError(rc, "gpz_hybrid_create")
        self._h = h

    def chunk(self, data) -> bytes:
        a = _u8(data)
        cap = self.L.gpz_bound(a.size)
        out = np.empty(cap, dtype=np.uint8)
        n = ctypes.c_size_t()
        rc = self.L.gpz_hybrid_chunk(self._h, _p(a), a.size, _p(out), cap, ctypes.byref(n))
        if rc:
            raise GpzError(rc, "gpz_hybrid_chunk")
        return out[:n.value].tobytes()

    def stats(self):
        """(chunks the CPU took, chunks the GPU took)."""
        c, g = ctypes.c_uint64(), ctypes.c_uint64()
        self.L.gpz_hybrid_stats(self._h, ctypes.byref(c), ctypes.byref(g))
        return c.value, g.value

    def close(self):
        if getattr(self, "_h", None):
            self.L.gpz_hybrid_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Writer:
    """ParallelChunkedWriter over the library (gpz_writer_*): a file-like
    object whose bytes are cut into `chunk_size` chunks and written as gzip
    members, in order, to `dst` (anything with a write method).  With `ctx`
    the chunks go through the device: page-locked chunk buffers, streamed
    by the writer's thread through the context's pass loop; with `chunk_fn`
    (bytes -> gzip bytes) through that function instead, as the reference's
    writer takes any ChunkFn, and with `hybrid` (a Hybrid) through the hybrid
    CPU + GPU chunk function; in both, up to `max_in_flight` chunk calls run
    at once on the writer's worker threads.  flush() does not cut a chunk; close() writes the last
    partial chunk and raises the first error the writer met.  With sink_view, dst.write receives a
    memoryview of the library's buffer instead of a bytes copy; it is valid only during the call, so
    dst must consume it there (as a file's write does)."""

    def __init__(self, dst, ctx: "Context" = None, chunk_fn=None, chunk_size: int = 2 << 20, max_in_flight: int = 16,
                 hybrid: "Hybrid" = None, sink_view: bool = False):
        if sum(x is not None for x in (ctx, chunk_fn, hybrid)) != 1:
            raise ValueError("give exactly one of ctx, chunk_fn and hybrid")
        self.L = load()
        self._dst = dst
        self._err = None
        self._chunk_fn = chunk_fn
        self._h = None

        def sink(_user, buf, n):
            try:
                if sink_view:
                    at = ctypes.cast(buf, ctypes.c_void_p).value
                    self._dst.write(memoryview((ctypes.c_char * n).from_address(at)).cast("B") if n else b"")
                else:
                    self._dst.write(ctypes.string_at(buf, n))
                return 0
            except Exception as e:  # noqa: BLE001 -- reported by close()
                self._err = self._err or e
                return 1

        def chunk(_user, buf, n, out, cap, out_len):
            try:
                g = bytes(self._chunk_fn(ctypes.string_at(buf, n)))
                if len(g) > cap:
                    return 1
                ctypes.memmove(out, g, len(g))
                out_len[0] = len(g)
                return 0
            except Exception as e:  # noqa: BLE001 -- reported by close()
                self._err = self._err or e
                return 1

        self._sink = SINK_FN(sink)  # kept alive with the writer
        self._chunk = CHUNK_FN(chunk)
        self._hybrid = hybrid
        h = ctypes.c_void_p()
        if ctx is not None:
            rc = self.L.gpz_writer_open(ctx._h, chunk_size, max_in_flight, self._sink, None, ctypes.byref(h))
        elif hybrid is not None:
            # the library's own chunk function: no Python in the chunk calls
            fn = CHUNK_FN(ctypes.cast(self.L.gpz_hybrid_chunk, ctypes.c_void_p).value)
            self._chunk = fn
            rc = self.L.gpz_writer_open_fn(fn, hybrid._h, chunk_size, max_in_flight, self._sink, None,
                                           ctypes.byref(h))
        else:
            rc = self.L.gpz_writer_open_fn(self._chunk, None, chunk_size, max_in_flight, self._sink, None,
                                           ctypes.byref(h))
        if rc:
            raise GpzError(rc, "gpz_writer_open")
        self._h = h

    def _check(self, rc, what):
        if rc:
            raise GpzError(rc, f"{what}: {self._err!r}" if self._err else what)

    def write(self, data) -> int:
        a = _u8(data)
        self._check(self.L.gpz_writer_write(self._h, _p(a), a.size), "gpz_writer_write")
        return a.size

    def flush(self):
        self._check(self.L.gpz_writer_flush(self._h), "gpz_writer_flush")

    def close(self):
        if self._h:
            rc = self.L.gpz_writer_finish(self._h)
            self.L.gpz_writer_close(self._h)
            self._h = None
            self._check(rc, "gpz_writer_finish")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

