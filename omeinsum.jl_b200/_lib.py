"""ctypes binding to libomeb200.so (the C ABI declared in include/ome_b200.h).

The library is the product's only compute path: there is no CPU fallback.
Loading fails loudly if the shared library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libomeb200.so")

# status codes (ome_status)
OK, INVALID_ARGUMENT, DIMENSION_MISMATCH, UNSUPPORTED, OUT_OF_MEMORY, TIMEOUT, CUDA_ERROR = range(7)
# dtypes (ome_dtype)
F32, F64, C32, C64, I64, BOOL, TROP_F32, TROP_F64 = range(8)
# precision modes (ome_prec)
PREC_AUTO, PREC_FP32, PREC_BF16X3, PREC_BF16X6 = range(4)

EXPORTS = [
    "ome_version", "ome_launch_count", "ome_device_status", "ome_selftest_wait_timeout",
    "ome_kernel_timing", "ome_kernel_times", "ome_last_error", "ome_ctx_create", "ome_ctx_destroy", "ome_ctx_workspace_bytes",
    "ome_einsum", "ome_loop_einsum", "ome_einsum_grad", "ome_plan_create", "ome_plan_destroy", "ome_plan_peak_bytes",
    "ome_plan_execute", "ome_plan_gradient", "ome_plan_slice_count", "ome_plan_partial_info",
    "ome_plan_execute_slices", "ome_plan_finish", "ome_reduce_noalloc", "ome_batch_create", "ome_batch_run",
    "ome_batch_info", "ome_batch_destroy", "ome_batch_graph_create", "ome_graph_launch", "ome_graph_destroy",
    "ome_server_create", "ome_server_submit", "ome_server_poll", "ome_server_stats", "ome_server_clock", "ome_server_destroy",
    "ome_treesa", "ome_greedy", "ome_slice_greedy",
]

JOB_COMPLETED, JOB_FAILED, JOB_REJECTED_MEMORY, JOB_REJECTED_WORK = range(4)


class DimensionMismatch(Exception):
    """Julia ``DimensionMismatch`` (src/interfaces.jl:87,100)."""


class ArgumentError(ValueError):
    """Julia ``ArgumentError`` (src/interfaces.jl:78-83)."""


class OMEError(RuntimeError):
    """Any other failure reported by the library (unsupported, CUDA error, ...)."""


class Tensor(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("ndim", C.c_int32),
        ("dims", C.POINTER(C.c_int64)),
        ("strides", C.POINTER(C.c_int64)),
        ("labels", C.POINTER(C.c_int32)),
    ]


class ServerJob(C.Structure):
    """ome_server_job"""
    _fields_ = [("id", C.c_int64), ("outcome", C.c_int32), ("status", C.c_int32), ("arrival_s", C.c_double),
                ("admitted_s", C.c_double), ("done_s", C.c_double)]


class ServingStats(C.Structure):
    """ome_serving_stats"""
    _fields_ = [(k, C.c_int64) for k in ("submitted", "completed", "failed", "rejected_memory", "rejected_work",
                                         "queued", "running")] + \
               [(k, C.c_double) for k in ("p50_ms", "p90_ms", "p99_ms", "jobs_per_s", "makespan_s")]


_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load libomeb200.so (once)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python omeinsum.jl_b200/build.py` "
                "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        i32p = C.POINTER(C.c_int32)
        i64p = C.POINTER(C.c_int64)
        lib.ome_version.restype = C.c_int
        lib.ome_launch_count.restype = C.c_ulonglong
        lib.ome_last_error.restype = C.c_char_p
        lib.ome_device_status.argtypes = [P]
        lib.ome_selftest_wait_timeout.argtypes = [P, C.c_uint64]
        lib.ome_kernel_timing.argtypes = [C.c_int]
        lib.ome_kernel_times.argtypes = [C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_char_p),
                                         C.POINTER(C.c_int32)]
        lib.ome_ctx_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(P)]
        lib.ome_ctx_destroy.argtypes = [P]
        lib.ome_ctx_workspace_bytes.argtypes = [P, C.POINTER(C.c_size_t)]
        lib.ome_einsum.argtypes = [P, P, C.c_int, C.c_int32, C.POINTER(Tensor), C.POINTER(Tensor), P, P, C.c_int32]
        lib.ome_loop_einsum.argtypes = [P, P, C.c_int, C.c_int32, C.POINTER(Tensor), C.POINTER(Tensor), P, P]
        lib.ome_einsum_grad.argtypes = [P, P, C.c_int, C.c_int32, C.POINTER(Tensor), C.POINTER(Tensor), C.c_int32,
                                        C.POINTER(Tensor), C.c_int32]
        lib.ome_plan_create.argtypes = [P, C.c_int, C.c_int32, i32p, i32p, C.c_int32, i32p, i32p, i32p, i32p,
                                        C.c_int32, i32p, i64p, C.c_int32, i32p, C.c_int32, C.POINTER(P)]
        lib.ome_plan_destroy.argtypes = [P]
        lib.ome_plan_peak_bytes.argtypes = [P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        lib.ome_plan_execute.argtypes = [P, P, P, C.POINTER(P), P, P, P]
        lib.ome_plan_gradient.argtypes = [P, P, P, C.POINTER(P), P, P, C.POINTER(P)]
        lib.ome_plan_slice_count.argtypes = [P, i64p]
        lib.ome_plan_partial_info.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
        lib.ome_plan_execute_slices.argtypes = [P, P, P, C.POINTER(P), C.c_int64, C.c_int64, P]
        lib.ome_plan_finish.argtypes = [P, P, P, P, P, P, P]
        lib.ome_batch_create.argtypes = [P, P, C.c_int, C.c_int32, C.POINTER(Tensor), C.POINTER(Tensor),
                                         C.POINTER(Tensor), C.c_int32, C.POINTER(P)]
        lib.ome_batch_run.argtypes = [P, P, P, P, P]
        lib.ome_batch_info.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(C.c_float)]
        lib.ome_batch_destroy.argtypes = [P]
        lib.ome_batch_graph_create.argtypes = [P, P, C.c_int32, C.POINTER(P), C.POINTER(P), C.POINTER(P),
                                               C.POINTER(P)]
        lib.ome_graph_launch.argtypes = [P, P]
        lib.ome_graph_destroy.argtypes = [P]
        lib.ome_server_create.argtypes = [C.c_int, C.c_int32, C.c_size_t, C.c_double, C.POINTER(P)]
        lib.ome_server_submit.argtypes = [P, P, C.c_int32, C.POINTER(P), P, C.POINTER(P), C.c_double, P,
                                          C.POINTER(C.c_int64)]
        lib.ome_server_poll.argtypes = [P, C.c_int32, C.POINTER(ServerJob), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int32)]
        lib.ome_server_stats.argtypes = [P, C.POINTER(ServingStats)]
        lib.ome_server_clock.argtypes = [P, C.POINTER(C.c_double)]
        lib.ome_server_destroy.argtypes = [P]
        lib.ome_reduce_noalloc.argtypes = [P, C.c_int, C.POINTER(Tensor), C.POINTER(Tensor), P, P]
        dp = C.POINTER(C.c_double)
        lib.ome_treesa.argtypes = [C.c_int32, i32p, i32p, C.c_int32, i32p, C.c_int32, dp, i32p, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32,
                                   C.c_int32, C.c_uint64, i32p, dp]
        lib.ome_slice_greedy.argtypes = [C.c_int32, i32p, i32p, C.c_int32, i32p, C.c_int32, dp, i32p, C.c_double,
                                         C.c_int32, i32p, i32p, i32p]
        lib.ome_greedy.argtypes = [C.c_int32, i32p, i32p, C.c_int32, i32p, C.c_int32, dp, C.c_double, C.c_double,
                                   C.c_int32, C.c_uint64, i32p, dp]
        for f in EXPORTS:
            if f not in ("ome_version", "ome_last_error", "ome_launch_count"):
                getattr(lib, f).restype = C.c_int
        _lib = lib
        return lib


def check(rc: int) -> None:
    """Raise the Python counterpart of a non-zero ome_status."""
    if rc == OK:
        return
    msg = load().ome_last_error().decode(errors="replace")
    if rc == INVALID_ARGUMENT:
        raise ArgumentError(msg)
    if rc == DIMENSION_MISMATCH:
        raise DimensionMismatch(msg)
    if rc == OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise OMEError(f"[status {rc}] {msg}")


def device_status(stream=None) -> None:
    """Synchronise and raise OMEError if a bounded device-side wait gave up."""
    check(load().ome_device_status(stream))


class Context:
    """One library context (device + workspace) per CUDA device."""

    def __init__(self, device: int, workspace_bytes: int):
        self.device = device
        self.workspace_bytes = int(workspace_bytes)
        h = C.c_void_p()
        check(load().ome_ctx_create(device, self.workspace_bytes, C.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            load().ome_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts: dict[int, Context] = {}


def release_workspaces() -> None:
    """Destroy the per-device contexts (their workspaces); they are re-created on demand."""
    import torch

    for d, c in list(_contexts.items()):
        torch.cuda.synchronize(d)
        c.close()
        del _contexts[d]
DEFAULT_WORKSPACE = 256 << 20


def context(device: int, min_workspace: int = 0) -> Context:
    """The context of `device`, grown (re-created) if its workspace is smaller
    than `min_workspace` bytes."""
    import torch

    c = _contexts.get(device)
    need = max(min_workspace, DEFAULT_WORKSPACE)
    if c is None or c.workspace_bytes < min_workspace:
        if c is not None:
            torch.cuda.synchronize(device)
            c.close()
        c = Context(device, need if c is None else max(need, c.workspace_bytes * 2, min_workspace))
        _contexts[device] = c
    return c
