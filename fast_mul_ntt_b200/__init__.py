"""B200-native (sm_100a) 3-prime NTT big-integer multiplication.

Python front end of the C ABI in include/fast_mul.h, loaded from the in-tree build
fast_mul_ntt_b200/lib/libfastmul_b200.so.  The API mirrors the reference's two entry points
(HJimmyK/fast_mul_ntt src/fast_mul.h:39,45):

    abs_mul64(in1, in2) -> out      # len(out) == len(in1) + len(in2)
    abs_sqr64(in1)      -> out      # len(out) == 2 * len(in1)

over little-endian numpy uint64 limb arrays, plus device-pointer forms for torch tensors.
There is no CPU fallback: every product runs the CUDA kernels, and a missing library or
GPU raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfastmul_b200.so")

FMN_OK = 0
_ERRNAMES = {1: "FMN_ERR_ARG", 2: "FMN_ERR_CUDA", 3: "FMN_ERR_NOMEM", 4: "FMN_ERR_DEVICE",
             5: "FMN_ERR_TOO_LARGE"}

# Every symbol include/fast_mul.h declares (checked by the tests).
EXPORTS = ["abs_mul64", "abs_sqr64", "fmn_init", "fmn_shutdown", "fmn_last_error", "fmn_mul", "fmn_sqr",
           "fmn_mul_device", "fmn_sqr_device", "fmn_sync", "fmn_workspace_size", "fmn_mul_device_ws",
           "fmn_ws_status", "fmn_ntt_len", "fmn_kernel_kind_name", "fmn_profile_enable", "fmn_profile_take",
           "fmn_launches_per_product", "fmn_bench_modmul", "fmn_mul_device_noalloc", "fmn_mul_batch_device",
           "fmn_batch_graph_create", "fmn_batch_graph_launch", "fmn_batch_graph_sync", "fmn_batch_graph_destroy",
           "fmn_operand_create", "fmn_operand_destroy", "fmn_operand_len", "fmn_mul_operand_device",
           "fmn_operand_workspace_size", "fmn_mul_operand_ws", "fmn_server_create", "fmn_server_submit",
           "fmn_server_wait", "fmn_server_take", "fmn_server_get_stats", "fmn_server_replay", "fmn_server_destroy",
           "fmn_get_plan", "fmn_set_plan", "fmn_autotune", "fmn_load_plans", "fmn_load_default_plans",
           "fmn_set_engine", "fmn_get_engine", "fmn_engine_for", "fmn_pieces_for",
           "fmn_force_pieces", "fmn_bench_bfly32", "fmn_get_plan_engine", "fmn_set_plan_engine",
           "fmn_test_fail_allocs", "fmn_test_carry_timeout", "fmn_server_cancel", "fmn_server_pause",
           "fmn_wrap_for", "fmn_twist_for", "fmn_batch_twist_for", "fmn_force_wrap"]

ENGINE_AUTO, ENGINE_64, ENGINE_32 = 0, 1, 2

FMN_OP_MUL, FMN_OP_SQR, FMN_OP_MUL_OPERAND = 0, 1, 2


class FmnRequest(ctypes.Structure):
    """fmn_request of include/fast_mul.h."""
    _fields_ = [("op", ctypes.c_int), ("in1", ctypes.c_void_p), ("len1", ctypes.c_uint64),
                ("in2", ctypes.c_void_p), ("len2", ctypes.c_uint64), ("operand", ctypes.c_void_p),
                ("out", ctypes.c_void_p), ("check", ctypes.c_void_p), ("tag", ctypes.c_uint64)]


class FmnServerStats(ctypes.Structure):
    """fmn_server_stats of include/fast_mul.h."""
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("mismatches", ctypes.c_uint64),
                ("device_errors", ctypes.c_uint64), ("peak_bytes", ctypes.c_size_t), ("cancelled", ctypes.c_uint64),
                ("launch_ms", ctypes.c_double), ("alloc_ms", ctypes.c_double),
                ("max_launch_ms", ctypes.c_double), ("max_alloc_ms", ctypes.c_double)]


class FmnJob(ctypes.Structure):
    """fmn_job of include/fast_mul.h (device pointers)."""
    _fields_ = [("in1", ctypes.c_void_p), ("len1", ctypes.c_uint64), ("in2", ctypes.c_void_p),
                ("len2", ctypes.c_uint64), ("out", ctypes.c_void_p)]
KERNEL_KINDS = 6

_u64 = ctypes.c_uint64
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p
_lib = None


class FastMulError(RuntimeError):
    """A status code other than FMN_OK from the library."""

    def __init__(self, code, msg):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


def load_library(path=None):
    """Load (once) and return the ctypes handle of the CUDA library."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"CUDA library not built: {p} (run python -m fast_mul_ntt_b200.build)")
    lib = ctypes.CDLL(p)
    lib.abs_mul64.argtypes = [_u64p, _u64, _u64p, _u64, _u64p]
    lib.abs_mul64.restype = None
    lib.abs_sqr64.argtypes = [_u64p, _u64, _u64p]
    lib.abs_sqr64.restype = None
    lib.fmn_init.argtypes = [ctypes.c_int]
    lib.fmn_init.restype = ctypes.c_int
    lib.fmn_shutdown.argtypes = []
    lib.fmn_shutdown.restype = None
    lib.fmn_last_error.argtypes = []
    lib.fmn_last_error.restype = ctypes.c_char_p
    lib.fmn_mul.argtypes = [_u64p, _u64, _u64p, _u64, _u64p]
    lib.fmn_mul.restype = ctypes.c_int
    lib.fmn_sqr.argtypes = [_u64p, _u64, _u64p]
    lib.fmn_sqr.restype = ctypes.c_int
    lib.fmn_mul_device.argtypes = [_vp, _u64, _vp, _u64, _vp, _vp]
    lib.fmn_mul_device.restype = ctypes.c_int
    lib.fmn_sqr_device.argtypes = [_vp, _u64, _vp, _vp]
    lib.fmn_sqr_device.restype = ctypes.c_int
    lib.fmn_sync.argtypes = [_vp]
    lib.fmn_sync.restype = ctypes.c_int
    lib.fmn_workspace_size.argtypes = [_u64, _u64, ctypes.c_int]
    lib.fmn_workspace_size.restype = ctypes.c_size_t
    lib.fmn_mul_device_ws.argtypes = [_vp, _u64, _vp, _u64, _vp, _vp, ctypes.c_size_t, _vp]
    lib.fmn_mul_device_ws.restype = ctypes.c_int
    lib.fmn_ws_status.argtypes = [_vp, _u64, _u64, ctypes.c_int, _vp]
    lib.fmn_ws_status.restype = ctypes.c_int
    lib.fmn_ntt_len.argtypes = [_u64, _u64]
    lib.fmn_ntt_len.restype = _u64
    lib.fmn_kernel_kind_name.argtypes = [ctypes.c_int]
    lib.fmn_kernel_kind_name.restype = ctypes.c_char_p
    lib.fmn_profile_enable.argtypes = [ctypes.c_int]
    lib.fmn_profile_enable.restype = ctypes.c_int
    _dp = ctypes.POINTER(ctypes.c_double)
    lib.fmn_profile_take.argtypes = [_dp, _u64p, _dp, _dp]
    lib.fmn_profile_take.restype = ctypes.c_int
    lib.fmn_launches_per_product.argtypes = [_u64, _u64, ctypes.c_int]
    lib.fmn_launches_per_product.restype = ctypes.c_int
    lib.fmn_bench_modmul.argtypes = [_dp, _dp]
    lib.fmn_bench_modmul.restype = ctypes.c_int
    lib.fmn_bench_bfly32.argtypes = [_dp]
    lib.fmn_bench_bfly32.restype = ctypes.c_int
    lib.fmn_wrap_for.argtypes = [_u64, _u64, ctypes.c_int]
    lib.fmn_wrap_for.restype = _u64
    lib.fmn_twist_for.argtypes = [_u64, _u64, ctypes.c_int]
    lib.fmn_twist_for.restype = _u64
    lib.fmn_batch_twist_for.argtypes = [_u64, _u64, ctypes.c_int]
    lib.fmn_batch_twist_for.restype = _u64
    lib.fmn_force_wrap.argtypes = [ctypes.c_int]
    lib.fmn_force_wrap.restype = ctypes.c_int
    lib.fmn_test_fail_allocs.argtypes = [ctypes.c_int]
    lib.fmn_test_fail_allocs.restype = ctypes.c_int
    lib.fmn_test_carry_timeout.argtypes = [_u64]
    lib.fmn_test_carry_timeout.restype = ctypes.c_int
    lib.fmn_mul_device_noalloc.argtypes = [_vp, _u64, _vp, _u64, _vp, _vp]
    lib.fmn_mul_device_noalloc.restype = ctypes.c_int
    _jp = ctypes.POINTER(FmnJob)
    lib.fmn_mul_batch_device.argtypes = [_jp, ctypes.c_int, _vp]
    lib.fmn_mul_batch_device.restype = ctypes.c_int
    lib.fmn_batch_graph_create.argtypes = [_jp, ctypes.c_int, ctypes.POINTER(_vp)]
    lib.fmn_batch_graph_create.restype = ctypes.c_int
    lib.fmn_batch_graph_launch.argtypes = [_vp, _vp]
    lib.fmn_batch_graph_launch.restype = ctypes.c_int
    lib.fmn_batch_graph_sync.argtypes = [_vp, _vp]
    lib.fmn_batch_graph_sync.restype = ctypes.c_int
    lib.fmn_batch_graph_destroy.argtypes = [_vp]
    lib.fmn_batch_graph_destroy.restype = None
    lib.fmn_operand_create.argtypes = [_vp, _u64, _u64, _vp, ctypes.POINTER(_vp)]
    lib.fmn_operand_create.restype = ctypes.c_int
    lib.fmn_operand_destroy.argtypes = [_vp]
    lib.fmn_operand_destroy.restype = None
    lib.fmn_operand_len.argtypes = [_vp]
    lib.fmn_operand_len.restype = _u64
    lib.fmn_mul_operand_device.argtypes = [_vp, _vp, _u64, _vp, _vp]
    lib.fmn_mul_operand_device.restype = ctypes.c_int
    lib.fmn_operand_workspace_size.argtypes = [_vp, _u64]
    lib.fmn_operand_workspace_size.restype = ctypes.c_size_t
    lib.fmn_mul_operand_ws.argtypes = [_vp, _vp, _u64, _vp, _vp, ctypes.c_size_t, _vp]
    lib.fmn_mul_operand_ws.restype = ctypes.c_int
    lib.fmn_server_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]
    lib.fmn_server_create.restype = ctypes.c_int
    lib.fmn_server_submit.argtypes = [_vp, ctypes.POINTER(FmnRequest)]
    lib.fmn_server_submit.restype = ctypes.c_int
    lib.fmn_server_wait.argtypes = [_vp]
    lib.fmn_server_wait.restype = ctypes.c_int
    lib.fmn_server_take.argtypes = [_vp, _u64p, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.fmn_server_take.restype = ctypes.c_int
    lib.fmn_server_get_stats.argtypes = [_vp, ctypes.POINTER(FmnServerStats)]
    lib.fmn_server_get_stats.restype = ctypes.c_int
    lib.fmn_server_replay.argtypes = [_vp, ctypes.POINTER(FmnRequest), _dp, ctypes.c_int, _dp, _dp]
    lib.fmn_server_replay.restype = ctypes.c_int
    lib.fmn_server_destroy.argtypes = [_vp]
    lib.fmn_server_destroy.restype = None
    lib.fmn_server_cancel.argtypes = [_vp, _u64]
    lib.fmn_server_cancel.restype = ctypes.c_int
    lib.fmn_server_pause.argtypes = [_vp, ctypes.c_int]
    lib.fmn_server_pause.restype = ctypes.c_int
    _ip = ctypes.POINTER(ctypes.c_int)
    lib.fmn_get_plan.argtypes = [ctypes.c_int, _ip, ctypes.c_int]
    lib.fmn_get_plan.restype = ctypes.c_int
    lib.fmn_set_plan.argtypes = [ctypes.c_int, _ip, ctypes.c_int]
    lib.fmn_set_plan.restype = ctypes.c_int
    lib.fmn_autotune.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
    lib.fmn_autotune.restype = ctypes.c_int
    lib.fmn_load_plans.argtypes = [ctypes.c_char_p]
    lib.fmn_load_plans.restype = ctypes.c_int
    lib.fmn_get_plan_engine.argtypes = [ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int]
    lib.fmn_get_plan_engine.restype = ctypes.c_int
    lib.fmn_set_plan_engine.argtypes = [ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int]
    lib.fmn_set_plan_engine.restype = ctypes.c_int
    lib.fmn_load_default_plans.argtypes = []
    lib.fmn_load_default_plans.restype = ctypes.c_int
    lib.fmn_set_engine.argtypes = [ctypes.c_int]
    lib.fmn_set_engine.restype = ctypes.c_int
    lib.fmn_get_engine.argtypes = []
    lib.fmn_get_engine.restype = ctypes.c_int
    lib.fmn_engine_for.argtypes = [_u64, _u64, ctypes.c_int]
    lib.fmn_engine_for.restype = ctypes.c_int
    lib.fmn_pieces_for.argtypes = [_u64, _u64, ctypes.c_int]
    lib.fmn_pieces_for.restype = ctypes.c_int
    lib.fmn_force_pieces.argtypes = [ctypes.c_int]
    lib.fmn_force_pieces.restype = ctypes.c_int
    if path is None:
        _lib = lib
    return lib


def _check(rc):
    if rc != FMN_OK:
        raise FastMulError(rc, _lib.fmn_last_error().decode())


def _limbs(x):
    return np.ascontiguousarray(x, dtype=np.uint64)


def _p(a):
    return a.ctypes.data_as(_u64p)


def init(device=0):
    """Select ``device`` for the calling thread and upload the twiddle tables."""
    _check(load_library().fmn_init(device))


def abs_mul64(in1, in2, out=None):
    """in1 * in2 as a numpy uint64 array of len(in1) + len(in2) limbs (host memory)."""
    lib = load_library()
    a, b = _limbs(in1), _limbs(in2)
    if out is None:
        out = np.empty(len(a) + len(b), dtype=np.uint64)
    if a.size and b.size and a.ctypes.data == b.ctypes.data and len(a) != len(b):
        b = b.copy()
    _check(lib.fmn_mul(_p(a), len(a), _p(b), len(b), _p(out)))
    return out


def abs_sqr64(in1, out=None):
    """in1 * in1 as a numpy uint64 array of 2 * len(in1) limbs (host memory)."""
    lib = load_library()
    a = _limbs(in1)
    if out is None:
        out = np.empty(2 * len(a), dtype=np.uint64)
    _check(lib.fmn_sqr(_p(a), len(a), _p(out)))
    return out


def ntt_len(len1, len2):
    """Transform length of a product (next power of two >= len1 + len2 - 1)."""
    return int(load_library().fmn_ntt_len(len1, len2))


def _stream_ptr(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


_LIMB_DTYPES = None


def _dev_limbs(t, what, need=None):
    """A CUDA tensor of 64-bit limbs, contiguous, with at least ``need`` elements (outputs):
    checked before any launch, since the C ABI takes plain pointers and sizes and a short
    output buffer would be written past its end."""
    global _LIMB_DTYPES
    if _LIMB_DTYPES is None:
        import torch
        _LIMB_DTYPES = frozenset(d for d in (torch.int64, getattr(torch, "uint64", None)) if d is not None)
    if (getattr(t, "is_cuda", False) and t.dtype in _LIMB_DTYPES and t.is_contiguous()
            and (need is None or t.numel() >= need)):
        return t
    if not getattr(t, "is_cuda", False):
        raise ValueError(f"{what}: expected a CUDA tensor")
    if t.element_size() != 8 or t.dtype.is_floating_point or t.dtype.is_complex:
        raise ValueError(f"{what}: expected 64-bit integer limbs, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{what}: expected a contiguous tensor")
    if need is not None and t.numel() < need:
        raise ValueError(f"{what}: holds {t.numel()} limbs, needs {need}")
    return t


def mul_device(a, b, out, stream=None):
    """Device product of int64/uint64 CUDA tensors holding limbs; asynchronous on ``stream``
    (default: torch's current stream).  ``out`` must hold len(a) + len(b) limbs."""
    lib = load_library()
    _dev_limbs(a, "a"), _dev_limbs(b, "b"), _dev_limbs(out, "out", a.numel() + b.numel())
    _check(lib.fmn_mul_device(a.data_ptr(), a.numel(), b.data_ptr(), b.numel(), out.data_ptr(),
                              _stream_ptr(stream)))
    return out


def sqr_device(a, out, stream=None):
    """Device square of a CUDA limb tensor into ``out`` (2 * len(a) limbs)."""
    lib = load_library()
    _dev_limbs(a, "a"), _dev_limbs(out, "out", 2 * a.numel())
    _check(lib.fmn_sqr_device(a.data_ptr(), a.numel(), out.data_ptr(), _stream_ptr(stream)))
    return out


def sync(stream=None):
    """Wait for ``stream`` and raise if a kernel reported an internal error."""
    _check(load_library().fmn_sync(_stream_ptr(stream)))


def workspace_size(len1, len2, sqr=False):
    """Scratch bytes one product needs (for mul_device_ws)."""
    return int(load_library().fmn_workspace_size(len1, len2, 1 if sqr else 0))


def mul_device_ws(a, b, out, ws, stream=None):
    """Device product with caller-provided scratch ``ws`` (a CUDA tensor of at least
    workspace_size bytes, 256-byte aligned)."""
    lib = load_library()
    _dev_limbs(a, "a"), _dev_limbs(b, "b"), _dev_limbs(out, "out", a.numel() + b.numel())
    _check(lib.fmn_mul_device_ws(a.data_ptr(), a.numel(), b.data_ptr(), b.numel(), out.data_ptr(),
                                 ws.data_ptr(), ws.numel() * ws.element_size(), _stream_ptr(stream)))
    return out


def ws_status(ws, stream=None):
    """Raise if the product that used workspace ``ws`` reported a device-side error."""
    _check(load_library().fmn_ws_status(ws.data_ptr(), 0, 0, 0, _stream_ptr(stream)))


def mul_device_noalloc(a, b, out, stream=None):
    """Device product that allocates no memory (fixed ~3 MB scratch array; len(a) + len(b)
    <= 65537).  For callers that cannot allocate device memory while they run; waits for
    ``stream``.  Calls overlapping on the GPU share the array and race."""
    lib = load_library()
    _dev_limbs(a, "a"), _dev_limbs(b, "b"), _dev_limbs(out, "out", a.numel() + b.numel())
    _check(lib.fmn_mul_device_noalloc(a.data_ptr(), a.numel(), b.data_ptr(), b.numel(), out.data_ptr(),
                                      _stream_ptr(stream)))
    return out


def profile_enable(on=True):
    """Record CUDA events around every kernel launch of this thread."""
    _check(load_library().fmn_profile_enable(1 if on else 0))


def profile_take():
    """Per kernel kind: {name: {"ms", "launches", "bytes", "modmuls"}} since the last call."""
    lib = load_library()
    k = KERNEL_KINDS
    ms, bts, mm = (ctypes.c_double * k)(), (ctypes.c_double * k)(), (ctypes.c_double * k)()
    ln = (ctypes.c_uint64 * k)()
    _check(lib.fmn_profile_take(ms, ln, bts, mm))
    return {lib.fmn_kernel_kind_name(i).decode(): {"ms": ms[i], "launches": int(ln[i]), "bytes": bts[i],
                                                    "modmuls": mm[i]} for i in range(k)}


def launches_per_product(len1, len2, sqr=False):
    return int(load_library().fmn_launches_per_product(len1, len2, 1 if sqr else 0))


def bench_modmul():
    """(modmuls/s, butterflies/s) peaks of the Montgomery arithmetic on the current device."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(load_library().fmn_bench_modmul(ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def bench_bfly32():
    """Butterflies/s peak of the 32-bit engine's arithmetic on the current device."""
    a = ctypes.c_double()
    _check(load_library().fmn_bench_bfly32(ctypes.byref(a)))
    return a.value


def _job_array(jobs):
    """[(a, b, out), ...] of CUDA tensors -> ctypes array of FmnJob (a is b: square)."""
    arr = (FmnJob * len(jobs))()
    for i, (a, b, out) in enumerate(jobs):
        _dev_limbs(a, f"jobs[{i}] a"), _dev_limbs(b, f"jobs[{i}] b")
        _dev_limbs(out, f"jobs[{i}] out", a.numel() + (a.numel() if a is b else b.numel()))
        arr[i].in1, arr[i].len1 = a.data_ptr(), a.numel()
        arr[i].in2, arr[i].len2 = b.data_ptr(), b.numel()
        arr[i].out = out.data_ptr()
    return arr


class BatchJobs:
    """A job list for mul_batch_device checked and marshalled once, for a batch that is
    launched again and again on the same tensors (the tensors must outlive it)."""

    def __init__(self, jobs):
        self._jobs = jobs
        self.arr = _job_array(jobs)
        self.n = len(jobs)


def mul_batch_device(jobs, stream=None):
    """All products of ``jobs`` ([(a, b, out)], CUDA limb tensors; ``a is b`` squares; or a
    BatchJobs) in batched launches, asynchronously on ``stream``."""
    lib = load_library()
    if isinstance(jobs, BatchJobs):
        arr, n = jobs.arr, jobs.n
    else:
        arr, n = _job_array(jobs), len(jobs)
    _check(lib.fmn_mul_batch_device(arr, n, _stream_ptr(stream)))


class BatchGraph:
    """A batch captured once in a CUDA graph; ``launch()`` recomputes every product from the
    current contents of the same input tensors into the same outputs."""

    def __init__(self, jobs):
        lib = load_library()
        self._jobs = jobs            # keep the tensors alive
        arr = _job_array(jobs)
        h = ctypes.c_void_p()
        _check(lib.fmn_batch_graph_create(arr, len(jobs), ctypes.byref(h)))
        self.handle = h

    def launch(self, stream=None):
        _check(load_library().fmn_batch_graph_launch(self.handle, _stream_ptr(stream)))

    def sync(self, stream=None):
        _check(load_library().fmn_batch_graph_sync(self.handle, _stream_ptr(stream)))

    def close(self):
        if self.handle:
            load_library().fmn_batch_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Operand:
    """A resident operand: its forward transform stays in device memory, so products with it
    transform only the partner (``mul``).  ``limbs`` (a CUDA tensor) must outlive it."""

    def __init__(self, limbs, max_partner_len, stream=None):
        lib = load_library()
        self.limbs = _dev_limbs(limbs, "limbs")
        h = ctypes.c_void_p()
        _check(lib.fmn_operand_create(limbs.data_ptr(), limbs.numel(), max_partner_len, _stream_ptr(stream),
                                      ctypes.byref(h)))
        self.handle = h
        self.len = limbs.numel()

    def mul(self, b, out, stream=None):
        _dev_limbs(b, "b"), _dev_limbs(out, "out", self.len + b.numel())
        _check(load_library().fmn_mul_operand_device(self.handle, b.data_ptr(), b.numel(), out.data_ptr(),
                                                      _stream_ptr(stream)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            load_library().fmn_operand_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The product server (continuous batching with an HBM budget); ``batching=False`` gives
    the plain per-call path on one stream."""

    def __init__(self, device=0, hbm_budget=120 << 30, max_batch=512, batching=True):
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.fmn_server_create(device, hbm_budget, max_batch, 1 if batching else 0, ctypes.byref(h)))
        self.handle = h

    def submit(self, req):
        _check(load_library().fmn_server_submit(self.handle, ctypes.byref(req)))

    def wait(self):
        _check(load_library().fmn_server_wait(self.handle))

    def cancel(self, tag):
        """Withdraw the requests with this tag that still wait for admission; False if none did."""
        return load_library().fmn_server_cancel(self.handle, tag) == FMN_OK

    def pause(self, paused=True):
        """Hold (or resume) admission; running batches finish."""
        _check(load_library().fmn_server_pause(self.handle, 1 if paused else 0))

    def take(self, max_n=1 << 16):
        tags = (ctypes.c_uint64 * max_n)()
        lat = (ctypes.c_double * max_n)()
        n = ctypes.c_int()
        _check(load_library().fmn_server_take(self.handle, tags, lat, max_n, ctypes.byref(n)))
        return [(int(tags[i]), lat[i]) for i in range(n.value)]

    def stats(self):
        st = FmnServerStats()
        _check(load_library().fmn_server_get_stats(self.handle, ctypes.byref(st)))
        return {k: (float if t is ctypes.c_double else int)(getattr(st, k)) for k, t in FmnServerStats._fields_}

    def replay(self, requests, arrivals):
        """Open-loop replay of a request array at the given arrival times (seconds); returns
        (latencies in ms per request, wall seconds)."""
        n = len(requests)
        arr = (FmnRequest * n)(*requests)
        at = (ctypes.c_double * n)(*arrivals)
        lat = (ctypes.c_double * n)()
        wall = ctypes.c_double()
        _check(load_library().fmn_server_replay(self.handle, arr, at, n, lat, ctypes.byref(wall)))
        return list(lat), wall.value

    def close(self):
        if getattr(self, "handle", None):
            load_library().fmn_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PLAN_DIR = os.path.join(HERE, "tune")


def get_plan(log_n, engine=ENGINE_64):
    """Pass bits of the plan in effect for 2^log_n points of an engine (64-bit by default)."""
    bits = (ctypes.c_int * 4)()
    p = load_library().fmn_get_plan_engine(engine, log_n, bits, 4)
    if p < 0:
        raise FastMulError(-p, "bad length")
    return [bits[i] for i in range(p)]


def set_plan(log_n, bits=None, engine=ENGINE_64):
    """Replace the plan of 2^log_n points of an engine (None restores the default)."""
    bits = list(bits or [])
    arr = (ctypes.c_int * max(1, len(bits)))(*bits)
    _check(load_library().fmn_set_plan_engine(engine, log_n, arr, len(bits)))


def set_engine(engine):
    """Process-wide residue engine for single products: ENGINE_AUTO (default), ENGINE_64 (the
    reference's 62-bit primes) or ENGINE_32 (32-bit digits, products up to 2^25 limbs)."""
    _check(load_library().fmn_set_engine(engine))


def get_engine():
    return load_library().fmn_get_engine()


def engine_for(len1, len2, sqr=False):
    """The engine (ENGINE_64 or ENGINE_32) a product of these lengths runs on."""
    return load_library().fmn_engine_for(len1, len2, 1 if sqr else 0)


def pieces_for(len1, len2, sqr=False):
    """Pieces a product is split into on the 32-bit engine (1: one whole transform)."""
    return load_library().fmn_pieces_for(len1, len2, 1 if sqr else 0)


def force_pieces(pieces):
    """Tests and tuning: split products into this many pieces where possible (0: cost model)."""
    _check(load_library().fmn_force_pieces(pieces))


def wrap_for(len1, len2, sqr=False):
    """Coefficients that wrap around the transform length of a wrapped product (0: not wrapped)."""
    return int(load_library().fmn_wrap_for(len1, len2, 1 if sqr else 0))


def twist_for(len1, len2, sqr=False):
    """Twisted length M of a wrapped product computed modulo X^M - c (0: not twisted)."""
    return int(load_library().fmn_twist_for(len1, len2, 1 if sqr else 0))


def batch_twist_for(len1, len2, sqr=False):
    """Twisted length M of a product run twisted inside a batch (0: whole)."""
    return int(load_library().fmn_batch_twist_for(len1, len2, 1 if sqr else 0))


def force_wrap(mode=1):
    """Tests: wrap every product that allows it -- 1 with the low product, 2 twisted; 0 or
    False restores the cost model."""
    _check(load_library().fmn_force_wrap(int(mode)))


def autotune(n_lo=10, n_hi=27, save_path=None):
    """Time every valid plan for 2^n_lo .. 2^n_hi points on the current GPU and keep the
    fastest; optionally write a plan file."""
    _check(load_library().fmn_autotune(n_lo, n_hi, save_path.encode() if save_path else None))
