"""ctypes binding of the bellman-cuda C ABI (include/bellman-cuda.h).

The same class drives any library that exports that ABI: this repository's
B200 library (lib/libbellman_cuda_b200.so, the default) or a build of the
reference era-bellman-cuda, so callers and tests are written once against the
reference's interface (src/bellman-cuda.h in that project).

Host buffers are numpy arrays; device buffers are integers (device pointers)
returned by bc_malloc.  Every call checks its bc_error and raises BcError.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIBRARY = os.path.join(HERE, "lib", "libbellman_cuda_b200.so")
# BCB200_LIBRARY points the binding at another build of the same sources (experiments)
DEFAULT_LIBRARY = os.environ.get("BCB200_LIBRARY", DEFAULT_LIBRARY)

RESULT_BITS = 254
FE_BYTES = 32
AFFINE_BYTES = 64
JACOBIAN_BYTES = 96

BC_SUCCESS = 0
BC_ERROR_INVALID_VALUE = 1
BC_ERROR_MEMORY_ALLOCATION = 2
BC_ERROR_NOT_READY = 600

# msm_b200_execute_no_alloc_async limits (include/bellman-cuda-b200.h)
NO_ALLOC_MAX_COUNT = 65536
NO_ALLOC_SCRATCH_BYTES = 64 << 20


class BcError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed with bc_error {code}")
        self.code = code


class Handle(ctypes.Structure):
    """bc_stream / bc_event / bc_mem_pool: struct { void *handle; }"""

    _fields_ = [("handle", ctypes.c_void_p)]


HOST_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p)


class MsmConfiguration(ctypes.Structure):
    """msm_configuration, field for field (include/bellman-cuda.h)."""

    _fields_ = [
        ("mem_pool", Handle),
        ("stream", Handle),
        ("bases", ctypes.c_void_p),
        ("scalars", ctypes.c_void_p),
        ("results", ctypes.c_void_p),
        ("log_scalars_count", ctypes.c_uint),
        ("h2d_copy_finished", Handle),
        ("h2d_copy_finished_callback", HOST_FN),
        ("h2d_copy_finished_callback_data", ctypes.c_void_p),
        ("d2h_copy_finished", Handle),
        ("d2h_copy_finished_callback", HOST_FN),
        ("d2h_copy_finished_callback_data", ctypes.c_void_p),
    ]


class MsmB200Configuration(ctypes.Structure):
    """msm_b200_configuration (include/bellman-cuda-b200.h)."""

    _fields_ = [
        ("mem_pool", Handle),
        ("stream", Handle),
        ("bases", ctypes.c_void_p),
        ("scalars", ctypes.c_void_p),
        ("results", ctypes.c_void_p),
        ("count", ctypes.c_uint),
        ("window_bits", ctypes.c_uint),
    ]


class MsmB200Profile(ctypes.Structure):
    """msm_b200_profile (include/bellman-cuda-b200.h)."""

    STAGES = ("digits", "sort", "zero_counts", "accumulate", "merge_heads", "reduce")
    _fields_ = [
        ("stage_ms", ctypes.c_float * 6),
        ("nonzero_entries", ctypes.c_ulonglong),
        ("nonempty_buckets", ctypes.c_ulonglong),
        ("heads", ctypes.c_ulonglong),
        ("window_bits", ctypes.c_uint),
        ("windows", ctypes.c_uint),
        ("acc_threads", ctypes.c_uint),
        ("launches", ctypes.c_uint),
        ("sort_wait_timeouts", ctypes.c_uint),
        ("affine_levels", ctypes.c_uint),
        ("affine_additions", ctypes.c_ulonglong),
    ]

    @property
    def madds(self) -> int:
        """XYZZ += affine additions of the accumulation."""
        return self.nonzero_entries - self.affine_additions - self.nonempty_buckets - self.heads


class AffinePoint(ctypes.Structure):
    """msm_b200_affine_point (include/bellman-cuda-b200.h): standard-form,
    fully reduced x and y, infinity flag."""

    _fields_ = [("x", ctypes.c_uint32 * 8), ("y", ctypes.c_uint32 * 8), ("infinity", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32 * 3)]

    def as_tuple(self):
        """(infinity, x, y) with x, y as Python integers."""
        x = sum(int(v) << (32 * i) for i, v in enumerate(self.x))
        y = sum(int(v) << (32 * i) for i, v in enumerate(self.y))
        return (bool(self.infinity), x, y)


class RequestTimes(ctypes.Structure):
    """msm_b200_request_times (include/bellman-cuda-b200.h)."""

    _fields_ = [("submit_us", ctypes.c_double), ("start_us", ctypes.c_double), ("done_us", ctypes.c_double), ("group_size", ctypes.c_uint)]


class ServerStats(ctypes.Structure):
    """msm_b200_server_stats (include/bellman-cuda-b200.h)."""

    _fields_ = [("groups", ctypes.c_ulonglong), ("requests", ctypes.c_ulonglong), ("max_inflight_groups", ctypes.c_ulonglong),
                ("arena_bytes", ctypes.c_size_t), ("arena_used", ctypes.c_size_t), ("pending", ctypes.c_size_t)]


def _ptr(x) -> Optional[int]:
    """numpy array -> host address; int -> as is; None -> NULL."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        assert x.flags["C_CONTIGUOUS"]
        return x.ctypes.data
    return int(x)


class BellmanCuda:
    """Thin checked wrapper over one library exporting the bellman-cuda ABI."""

    def __init__(self, path: str = DEFAULT_LIBRARY, extensions: Optional[bool] = None):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run __graft_entry__.build())")
        self.path = path
        self.lib = ctypes.CDLL(path)
        L = self.lib
        vp, sz, u, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint, ctypes.c_int
        sig = {
            "bc_get_device_count": [ctypes.POINTER(i)],
            "bc_get_device": [ctypes.POINTER(i)],
            "bc_set_device": [i],
            "bc_stream_create": [ctypes.POINTER(Handle), ctypes.c_bool],
            "bc_stream_wait_event": [Handle, Handle],
            "bc_stream_synchronize": [Handle],
            "bc_stream_query": [Handle],
            "bc_stream_destroy": [Handle],
            "bc_launch_host_fn": [Handle, HOST_FN, vp],
            "bc_event_create": [ctypes.POINTER(Handle), ctypes.c_bool, ctypes.c_bool],
            "bc_event_record": [Handle, Handle],
            "bc_event_synchronize": [Handle],
            "bc_event_query": [Handle],
            "bc_event_destroy": [Handle],
            "bc_event_elapsed_time": [ctypes.POINTER(ctypes.c_float), Handle, Handle],
            "bc_mem_get_info": [ctypes.POINTER(sz), ctypes.POINTER(sz)],
            "bc_malloc": [ctypes.POINTER(vp), sz],
            "bc_malloc_host": [ctypes.POINTER(vp), sz],
            "bc_free": [vp],
            "bc_free_host": [vp],
            "bc_host_register": [vp, sz],
            "bc_host_unregister": [vp],
            "bc_memcpy": [vp, vp, sz],
            "bc_memcpy_async": [vp, vp, sz, Handle],
            "bc_memset": [vp, i, sz],
            "bc_memset_async": [vp, i, sz, Handle],
            "bc_mem_pool_create": [ctypes.POINTER(Handle), i],
            "bc_mem_pool_destroy": [Handle],
            "bc_malloc_from_pool_async": [ctypes.POINTER(vp), sz, Handle, Handle],
            "bc_free_async": [vp, Handle],
            "ff_set_up": [u, u],
            "msm_set_up": [],
            "msm_execute_async": [MsmConfiguration],
            "msm_tear_down": [],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        has_ext = hasattr(L, "msm_b200_execute_async")
        self.extensions = has_ext if extensions is None else (extensions and has_ext)
        if self.extensions:
            ext = {
                "msm_b200_execute_async": [ctypes.POINTER(MsmB200Configuration)],
                "msm_b200_scratch_bytes": [u, u, ctypes.POINTER(sz)],
                "msm_b200_default_window_bits": [u, ctypes.POINTER(u)],
                "msm_b200_generator_multiples_async": [vp, vp, u, Handle],
                "msm_b200_execute_profiled": [ctypes.POINTER(MsmB200Configuration), ctypes.POINTER(MsmB200Profile)],
                "msm_b200_execute_staged_async": [ctypes.POINTER(MsmB200Configuration), ctypes.POINTER(Handle),
                                                  ctypes.POINTER(ctypes.c_uint)],
                "msm_b200_measure_mul_throughput": [u, ctypes.POINTER(ctypes.c_double)],
                "msm_b200_execute_no_alloc_async": [Handle, vp, vp, vp, u],
                "msm_b200_set_affine_levels": [i],
                "msm_b200_final_sum_async": [vp, vp, Handle],
                "msm_b200_base_table_create": [ctypes.POINTER(vp), vp, u, ctypes.POINTER(u), u, Handle],
                "msm_b200_base_table_bytes": [vp, ctypes.POINTER(sz)],
                "msm_b200_base_table_destroy": [vp],
                "msm_b200_base_table_serialized_bytes": [vp, ctypes.POINTER(sz)],
                "msm_b200_base_table_export": [vp, vp, sz],
                "msm_b200_base_table_import": [ctypes.POINTER(vp), vp, sz, Handle],
                "msm_b200_batch_window_bits": [u, ctypes.POINTER(u)],
                "msm_b200_batch_create": [ctypes.POINTER(vp), vp, ctypes.POINTER(u), u, ctypes.POINTER(u)],
                "msm_b200_batch_execute_async": [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), Handle],
                "msm_b200_batch_info": [vp, ctypes.POINTER(sz), ctypes.POINTER(u), ctypes.POINTER(ctypes.c_ulonglong)],
                "msm_b200_batch_destroy": [vp],
                "msm_b200_server_create": [ctypes.POINTER(vp), vp, sz, u, u],
                "msm_b200_server_submit": [vp, vp, u, vp, ctypes.POINTER(ctypes.c_ulonglong)],
                "msm_b200_server_wait": [vp, ctypes.c_ulonglong, ctypes.POINTER(RequestTimes)],
                "msm_b200_server_get_stats": [vp, ctypes.POINTER(ServerStats)],
                "msm_b200_server_destroy": [vp],
            }
            for name, args in ext.items():
                f = getattr(L, name)
                f.argtypes = args
                f.restype = ctypes.c_int

    # -- helpers -------------------------------------------------------------
    def check(self, code: int, what: str) -> None:
        if code != BC_SUCCESS:
            raise BcError(code, what)

    def call(self, name: str, *args) -> int:
        return getattr(self.lib, name)(*args)

    # -- runtime -------------------------------------------------------------
    def device_count(self) -> int:
        c = ctypes.c_int()
        self.check(self.lib.bc_get_device_count(ctypes.byref(c)), "bc_get_device_count")
        return c.value

    def set_device(self, d: int) -> None:
        self.check(self.lib.bc_set_device(d), "bc_set_device")

    def stream_create(self, blocking_sync: bool = True) -> Handle:
        h = Handle()
        self.check(self.lib.bc_stream_create(ctypes.byref(h), blocking_sync), "bc_stream_create")
        return h

    def stream_synchronize(self, s: Handle) -> None:
        self.check(self.lib.bc_stream_synchronize(s), "bc_stream_synchronize")

    def stream_destroy(self, s: Handle) -> None:
        self.check(self.lib.bc_stream_destroy(s), "bc_stream_destroy")

    def event_create(self, blocking_sync: bool = False, disable_timing: bool = False) -> Handle:
        h = Handle()
        self.check(self.lib.bc_event_create(ctypes.byref(h), blocking_sync, disable_timing), "bc_event_create")
        return h

    def event_record(self, e: Handle, s: Handle) -> None:
        self.check(self.lib.bc_event_record(e, s), "bc_event_record")

    def event_synchronize(self, e: Handle) -> None:
        self.check(self.lib.bc_event_synchronize(e), "bc_event_synchronize")

    def event_query(self, e: Handle) -> int:
        return self.lib.bc_event_query(e)

    def event_destroy(self, e: Handle) -> None:
        self.check(self.lib.bc_event_destroy(e), "bc_event_destroy")

    def elapsed_ms(self, start: Handle, end: Handle) -> float:
        ms = ctypes.c_float()
        self.check(self.lib.bc_event_elapsed_time(ctypes.byref(ms), start, end), "bc_event_elapsed_time")
        return ms.value

    def mem_get_info(self):
        f, t = ctypes.c_size_t(), ctypes.c_size_t()
        self.check(self.lib.bc_mem_get_info(ctypes.byref(f), ctypes.byref(t)), "bc_mem_get_info")
        return f.value, t.value

    def malloc(self, size: int) -> int:
        p = ctypes.c_void_p()
        self.check(self.lib.bc_malloc(ctypes.byref(p), max(1, size)), "bc_malloc")
        return p.value

    def free(self, p: int) -> None:
        self.check(self.lib.bc_free(p), "bc_free")

    def malloc_host(self, size: int) -> int:
        p = ctypes.c_void_p()
        self.check(self.lib.bc_malloc_host(ctypes.byref(p), max(1, size)), "bc_malloc_host")
        return p.value

    def free_host(self, p: int) -> None:
        self.check(self.lib.bc_free_host(p), "bc_free_host")

    def pinned_array(self, shape, dtype=np.uint32):
        """numpy view over fresh page-locked memory; returns (array, pointer)."""
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = self.malloc_host(nbytes)
        buf = (ctypes.c_byte * nbytes).from_address(p)
        return np.frombuffer(buf, dtype=dtype).reshape(shape), p

    def memcpy(self, dst, src, nbytes: int) -> None:
        self.check(self.lib.bc_memcpy(_ptr(dst), _ptr(src), nbytes), "bc_memcpy")

    def memcpy_async(self, dst, src, nbytes: int, s: Handle) -> None:
        self.check(self.lib.bc_memcpy_async(_ptr(dst), _ptr(src), nbytes, s), "bc_memcpy_async")

    def to_device(self, a: np.ndarray) -> int:
        a = np.ascontiguousarray(a)
        p = self.malloc(a.nbytes)
        self.memcpy(p, a, a.nbytes)
        return p

    def from_device(self, p: int, shape, dtype=np.uint32) -> np.ndarray:
        out = np.empty(shape, dtype=dtype)
        self.memcpy(out, p, out.nbytes)
        return out

    def mem_pool_create(self, device: int = 0) -> Handle:
        h = Handle()
        self.check(self.lib.bc_mem_pool_create(ctypes.byref(h), device), "bc_mem_pool_create")
        return h

    def mem_pool_destroy(self, h: Handle) -> None:
        self.check(self.lib.bc_mem_pool_destroy(h), "bc_mem_pool_destroy")

    # -- MSM -----------------------------------------------------------------
    def ff_set_up(self, w_log: int = 25, g_log: int = 14) -> None:
        self.check(self.lib.ff_set_up(w_log, g_log), "ff_set_up")

    def msm_set_up(self) -> None:
        self.check(self.lib.msm_set_up(), "msm_set_up")

    def msm_tear_down(self) -> None:
        self.check(self.lib.msm_tear_down(), "msm_tear_down")

    def msm_execute_async(self, pool: Handle, stream: Handle, bases, scalars, results, log_count: int,
                          h2d_event: Optional[Handle] = None, h2d_callback=None, h2d_data=None,
                          d2h_event: Optional[Handle] = None, d2h_callback=None, d2h_data=None) -> int:
        cfg = MsmConfiguration()
        cfg.mem_pool = pool
        cfg.stream = stream
        cfg.bases = _ptr(bases)
        cfg.scalars = _ptr(scalars)
        cfg.results = _ptr(results)
        cfg.log_scalars_count = log_count
        cfg.h2d_copy_finished = h2d_event or Handle()
        cfg.h2d_copy_finished_callback = h2d_callback or HOST_FN()
        cfg.h2d_copy_finished_callback_data = h2d_data
        cfg.d2h_copy_finished = d2h_event or Handle()
        cfg.d2h_copy_finished_callback = d2h_callback or HOST_FN()
        cfg.d2h_copy_finished_callback_data = d2h_data
        return self.lib.msm_execute_async(cfg)

    def msm(self, pool: Handle, stream: Handle, bases, scalars, results, log_count: int, **kw) -> None:
        self.check(self.msm_execute_async(pool, stream, bases, scalars, results, log_count, **kw), "msm_execute_async")

    # -- extensions ------------------------------------------------------------
    def msm_any(self, pool: Handle, stream: Handle, bases, scalars, results, count: int, window_bits: int = 0) -> int:
        cfg = self._b200_cfg(pool, stream, bases, scalars, results, count, window_bits)
        return self.lib.msm_b200_execute_async(ctypes.byref(cfg))

    def _b200_cfg(self, pool, stream, bases, scalars, results, count, window_bits):
        cfg = MsmB200Configuration()
        cfg.mem_pool = pool
        cfg.stream = stream
        cfg.bases = _ptr(bases)
        cfg.scalars = _ptr(scalars)
        cfg.results = _ptr(results)
        cfg.count = count
        cfg.window_bits = window_bits
        return cfg

    def msm_profiled(self, pool: Handle, stream: Handle, bases, scalars, results, count: int, window_bits: int = 0) -> MsmB200Profile:
        prof = MsmB200Profile()
        cfg = self._b200_cfg(pool, stream, bases, scalars, results, count, window_bits)
        self.check(self.lib.msm_b200_execute_profiled(ctypes.byref(cfg), ctypes.byref(prof)), "msm_b200_execute_profiled")
        return prof

    def set_affine_levels(self, levels: int) -> None:
        """Affine pairing levels of later MSMs, process-wide (negative: by size)."""
        self.check(self.lib.msm_b200_set_affine_levels(levels), "msm_b200_set_affine_levels")

    def msm_staged(self, pool: Handle, stream: Handle, bases, scalars, results, count: int, events, window_bits: int = 0) -> int:
        """Enqueue one MSM recording 7 caller events at its stage boundaries; returns kernels launched."""
        cfg = self._b200_cfg(pool, stream, bases, scalars, results, count, window_bits)
        ev = (Handle * 7)(*events)
        launched = ctypes.c_uint()
        self.check(self.lib.msm_b200_execute_staged_async(ctypes.byref(cfg), ev, ctypes.byref(launched)),
                   "msm_b200_execute_staged_async")
        return launched.value

    def mul_throughput(self, kind: int) -> float:
        v = ctypes.c_double()
        self.check(self.lib.msm_b200_measure_mul_throughput(kind, ctypes.byref(v)), "msm_b200_measure_mul_throughput")
        return v.value

    def generator_multiples(self, k_dev: int, bases_dev: int, count: int, stream: Handle) -> None:
        self.check(self.lib.msm_b200_generator_multiples_async(k_dev, bases_dev, count, stream),
                   "msm_b200_generator_multiples_async")

    def scratch_bytes(self, count: int, window_bits: int = 0) -> int:
        b = ctypes.c_size_t()
        self.check(self.lib.msm_b200_scratch_bytes(count, window_bits, ctypes.byref(b)), "msm_b200_scratch_bytes")
        return b.value

    def msm_no_alloc(self, stream: Handle, bases, scalars, results, count: int) -> int:
        """msm_b200_execute_no_alloc_async: device buffers only, count <= NO_ALLOC_MAX_COUNT; returns the bc_error."""
        return self.lib.msm_b200_execute_no_alloc_async(stream, _ptr(bases), _ptr(scalars), _ptr(results), count)

    def final_sum_async(self, results, point, stream: Handle) -> int:
        """msm_b200_final_sum_async: sum 2^i R_i of 254 Jacobian results (device or
        pinned memory) into one msm_b200_affine_point at `point` (device or pinned
        memory); returns the bc_error."""
        return self.lib.msm_b200_final_sum_async(_ptr(results), _ptr(point), stream)

    # -- batched MSMs over a resident base table -------------------------------
    def base_table_create(self, bases, count: int, stream: Handle, window_bits=None) -> int:
        """Resident table (+ precomputed window multiples) over `count` bases; returns its handle."""
        h = ctypes.c_void_p()
        widths = list(window_bits or [])
        arr = (ctypes.c_uint * max(1, len(widths)))(*widths)
        self.check(self.lib.msm_b200_base_table_create(ctypes.byref(h), _ptr(bases), count, arr if widths else None, len(widths), stream),
                   "msm_b200_base_table_create")
        return h.value

    def base_table_bytes(self, table: int) -> int:
        b = ctypes.c_size_t()
        self.check(self.lib.msm_b200_base_table_bytes(table, ctypes.byref(b)), "msm_b200_base_table_bytes")
        return b.value

    def base_table_destroy(self, table: int) -> None:
        self.check(self.lib.msm_b200_base_table_destroy(table), "msm_b200_base_table_destroy")

    def base_table_export(self, table: int) -> np.ndarray:
        """The table's save format as a uint8 array."""
        n = ctypes.c_size_t()
        self.check(self.lib.msm_b200_base_table_serialized_bytes(table, ctypes.byref(n)), "msm_b200_base_table_serialized_bytes")
        img = np.zeros(n.value, np.uint8)
        self.check(self.lib.msm_b200_base_table_export(table, img.ctypes.data, n.value), "msm_b200_base_table_export")
        return img

    def base_table_import_raw(self, image: np.ndarray, stream: Handle):
        """(bc_error, handle) of msm_b200_base_table_import."""
        h = ctypes.c_void_p()
        image = np.ascontiguousarray(image, dtype=np.uint8)
        rc = self.lib.msm_b200_base_table_import(ctypes.byref(h), image.ctypes.data, image.nbytes, stream)
        return rc, h.value

    def batch_window_bits(self, count: int) -> int:
        c = ctypes.c_uint()
        self.check(self.lib.msm_b200_batch_window_bits(count, ctypes.byref(c)), "msm_b200_batch_window_bits")
        return c.value

    def batch_create_raw(self, table: int, counts, window_bits=None):
        """(bc_error, handle) of msm_b200_batch_create."""
        h = ctypes.c_void_p()
        cnt = (ctypes.c_uint * len(counts))(*[int(c) for c in counts])
        wb = (ctypes.c_uint * len(counts))(*[int(c) for c in window_bits]) if window_bits is not None else None
        rc = self.lib.msm_b200_batch_create(ctypes.byref(h), table, cnt, len(counts), wb)
        return rc, h.value

    def batch_create(self, table: int, counts, window_bits=None) -> int:
        rc, h = self.batch_create_raw(table, counts, window_bits)
        self.check(rc, "msm_b200_batch_create")
        return h

    def batch_execute(self, batch: int, scalars, results, stream: Handle) -> None:
        sp = (ctypes.c_void_p * len(scalars))(*[_ptr(x) for x in scalars])
        rp = (ctypes.c_void_p * len(results))(*[_ptr(x) for x in results])
        self.check(self.lib.msm_b200_batch_execute_async(batch, sp, rp, stream), "msm_b200_batch_execute_async")

    def batch_info(self, batch: int):
        """(scratch bytes, kernels per execution, (window, point) entries)."""
        b, k, e = ctypes.c_size_t(), ctypes.c_uint(), ctypes.c_ulonglong()
        self.check(self.lib.msm_b200_batch_info(batch, ctypes.byref(b), ctypes.byref(k), ctypes.byref(e)), "msm_b200_batch_info")
        return b.value, k.value, e.value

    def batch_destroy(self, batch: int) -> None:
        self.check(self.lib.msm_b200_batch_destroy(batch), "msm_b200_batch_destroy")

    # -- request server ----------------------------------------------------------
    def server_create(self, table: int, scratch_budget: int, streams: int = 4, max_group: int = 16) -> int:
        h = ctypes.c_void_p()
        self.check(self.lib.msm_b200_server_create(ctypes.byref(h), table, scratch_budget, streams, max_group), "msm_b200_server_create")
        return h.value

    def server_submit(self, server: int, scalars, count: int, results) -> int:
        t = ctypes.c_ulonglong()
        self.check(self.lib.msm_b200_server_submit(server, _ptr(scalars), count, _ptr(results), ctypes.byref(t)), "msm_b200_server_submit")
        return t.value

    def server_wait(self, server: int, ticket: int):
        """(bc_error, RequestTimes) of one request; blocks until it has finished."""
        times = RequestTimes()
        rc = self.lib.msm_b200_server_wait(server, ticket, ctypes.byref(times))
        return rc, times

    def server_stats(self, server: int) -> ServerStats:
        st = ServerStats()
        self.check(self.lib.msm_b200_server_get_stats(server, ctypes.byref(st)), "msm_b200_server_get_stats")
        return st

    def server_destroy(self, server: int) -> None:
        self.check(self.lib.msm_b200_server_destroy(server), "msm_b200_server_destroy")

    def default_window_bits(self, count: int) -> int:
        c = ctypes.c_uint()
        self.check(self.lib.msm_b200_default_window_bits(count, ctypes.byref(c)), "msm_b200_default_window_bits")
        return c.value
