"""Python binding of libpolymult_b200.so (include/polymult_b200.h) through ctypes.

Mirrors the reference's plugin interface for this path, the three entry points the FHERMA
harness binds (fherma.toml:7-10; fherma.h:45-48):

    state = fherma_init(N, W, L, q_limbs)      # solve.cu:1392-1478
    c     = fherma_run(state, a, b)            # solve.cu:1480-1498
    fherma_free(state)                         # solve.cu:1530-1534

with the same meaning (q, a, b, c as L little-endian u32 limbs per coefficient; a, b, c of
shape (N, L)) and the same error behaviour (RuntimeError on an invalid point or a size
mismatch).  `Multiplier` is the object form, and adds the device-resident batch call.

There is no fallback: if the CUDA library is missing or no B200 is present, these calls raise.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# POLYMULT_LIB names another build of the same library (a variant under measurement)
LIB_PATH = os.environ.get("POLYMULT_LIB") or os.path.join(HERE, "lib", "libpolymult_b200.so")
HEADER = os.path.join(HERE, "..", "include", "polymult_b200.h")

PM_OK, PM_ERR_INVALID, PM_ERR_CUDA, PM_ERR_DEVICE, PM_ERR_UNSUPPORTED, PM_ERR_INTERNAL = range(6)
PM_DEVICE_CRT_BOUND, PM_DEVICE_FOLD, PM_DEVICE_WAIT = 1, 2, 4  # device status word bits
GEMM_FORMS = {"auto": 0, "plain": 1, "tensor": 2, "mixed": 3}
GEMM_NAMES = {v: k for k, v in GEMM_FORMS.items()}
STAGES = ("dec_a", "cols_a", "rows_a", "dec_b", "cols_b", "rows_fused", "cols_inv", "crt")


class PolymultError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("polymult error %d: %s" % (code, message))
        self.code = code


class PmInfo(ctypes.Structure):
    _fields_ = [("N", ctypes.c_uint32), ("W", ctypes.c_uint32), ("L", ctypes.c_uint32),
                ("K", ctypes.c_int32), ("logN", ctypes.c_int32), ("w1", ctypes.c_int32),
                ("w2", ctypes.c_int32), ("gemm_form", ctypes.c_int32), ("device", ctypes.c_int32),
                ("delta", ctypes.c_uint64), ("table_bytes", ctypes.c_uint64),
                ("scratch_bytes", ctypes.c_uint64), ("launches_per_multiply", ctypes.c_int32),
                ("group", ctypes.c_int32)]


class PmPipelineInfo(ctypes.Structure):
    _fields_ = [("in_chunks", ctypes.c_int32), ("out_chunks", ctypes.c_int32), ("in_body", ctypes.c_int32),
                ("out_body", ctypes.c_int32), ("tuned_ms", ctypes.c_double)]


class PmBatchClass(ctypes.Structure):
    _fields_ = [("N", ctypes.c_uint32), ("W", ctypes.c_uint32), ("L", ctypes.c_uint32),
                ("q", ctypes.c_void_p), ("count", ctypes.c_uint32), ("d_a", ctypes.c_void_p),
                ("d_b", ctypes.c_void_p), ("d_c", ctypes.c_void_p), ("w1", ctypes.c_int32)]


class PmBatchInfo(ctypes.Structure):
    _fields_ = [("classes", ctypes.c_uint32), ("streams", ctypes.c_uint32),
                ("kernel_launches", ctypes.c_int32), ("graph_nodes", ctypes.c_uint64),
                ("scratch_bytes", ctypes.c_uint64)]


class PmBatchClassInfo(ctypes.Structure):
    _fields_ = [("K", ctypes.c_int32), ("w1", ctypes.c_int32), ("w2", ctypes.c_int32),
                ("gemm_form", ctypes.c_int32), ("tuned_ms", ctypes.c_double),
                ("col_tma", ctypes.c_int32), ("crt_tm", ctypes.c_int32), ("launch_groups", ctypes.c_uint32)]


BATCH_TUNE, BATCH_NO_GRAPH = 1, 2
PIPELINE_PINNED = 1


class PmServeStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("mean_batch", ctypes.c_double),
                ("peak_inflight", ctypes.c_uint32), ("max_inflight", ctypes.c_uint32), ("seconds", ctypes.c_double)]

_lib: Optional[ctypes.CDLL] = None


def declared_symbols(header: str = HEADER):
    """Function names declared in include/polymult_b200.h."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pm_[a-z_]+)\s*\(", text)))


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the library (once); raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("libpolymult_b200.so not built (run polymult-challenge_b200/build.py): %s" % path)
    lib = ctypes.CDLL(path)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    vp = ctypes.c_void_p
    lib.pm_init.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, vp, ctypes.c_int, ctypes.c_int,
                            ctypes.POINTER(vp)]
    lib.pm_init.restype = ctypes.c_int
    lib.pm_run.argtypes = [vp, vp, vp, vp]
    lib.pm_run.restype = ctypes.c_int
    lib.pm_run_device.argtypes = [vp, vp, vp, vp, ctypes.c_uint32, vp]
    lib.pm_run_device.restype = ctypes.c_int
    lib.pm_time_stages.argtypes = [vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_int, vp,
                                   ctypes.POINTER(ctypes.c_float)]
    lib.pm_time_stages.restype = ctypes.c_int
    lib.pm_run_device_static.argtypes = [vp, vp, vp, vp, vp]
    lib.pm_run_device_static.restype = ctypes.c_int
    lib.pm_sync.argtypes = [vp]
    lib.pm_sync.restype = ctypes.c_int
    lib.pm_free.argtypes = [vp]
    lib.pm_free.restype = None
    lib.pm_get_info.argtypes = [vp, ctypes.POINTER(PmInfo)]
    lib.pm_get_info.restype = ctypes.c_int
    lib.pm_last_error.argtypes = []
    lib.pm_last_error.restype = ctypes.c_char_p
    lib.pm_plan_selfcheck.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, vp,
                                      ctypes.POINTER(ctypes.c_int32)]
    lib.pm_plan_selfcheck.restype = ctypes.c_int
    lib.pm_selftest_host_pool.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_uint64)]
    lib.pm_selftest_host_pool.restype = ctypes.c_int
    lib.pm_tune_pipeline.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(PmPipelineInfo)]
    lib.pm_tune_pipeline.restype = ctypes.c_int
    lib.pm_set_pipeline.argtypes = [vp, ctypes.c_int, ctypes.c_int32, ctypes.c_int32]
    lib.pm_set_pipeline.restype = ctypes.c_int
    lib.pm_get_pipeline.argtypes = [vp, ctypes.c_int, ctypes.POINTER(PmPipelineInfo)]
    lib.pm_get_pipeline.restype = ctypes.c_int
    lib.pm_batch_init.argtypes = [ctypes.POINTER(PmBatchClass), ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.POINTER(vp)]
    lib.pm_batch_init.restype = ctypes.c_int
    lib.pm_batch_run.argtypes = [vp, vp]
    lib.pm_batch_run.restype = ctypes.c_int
    lib.pm_batch_sync.argtypes = [vp]
    lib.pm_batch_sync.restype = ctypes.c_int
    lib.pm_batch_get_info.argtypes = [vp, ctypes.POINTER(PmBatchInfo)]
    lib.pm_batch_get_info.restype = ctypes.c_int
    lib.pm_batch_get_class.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(PmBatchClassInfo)]
    lib.pm_batch_get_class.restype = ctypes.c_int
    lib.pm_batch_free.argtypes = [vp]
    lib.pm_batch_free.restype = None
    lib.pm_server_init.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, vp, vp, ctypes.c_uint32,
                                   ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(vp)]
    lib.pm_server_init.restype = ctypes.c_int
    lib.pm_server_run.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.POINTER(PmServeStats), vp]
    lib.pm_server_run.restype = ctypes.c_int
    lib.pm_server_host_alloc.argtypes = [vp, ctypes.c_size_t, ctypes.POINTER(vp)]
    lib.pm_server_host_alloc.restype = ctypes.c_int
    lib.pm_server_host_free.argtypes = [vp, vp]
    lib.pm_server_host_free.restype = ctypes.c_int
    lib.pm_server_free.argtypes = [vp]
    lib.pm_server_free.restype = None
    lib.pm_digest.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint32, vp, vp]
    lib.pm_digest.restype = ctypes.c_int
    lib.pm_digest_host.argtypes = [vp, ctypes.c_uint64]
    lib.pm_digest_host.restype = ctypes.c_uint64
    lib.pm_test_fail_scratch_allocs.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.pm_test_fail_scratch_allocs.restype = None
    lib.pm_test_set_status.argtypes = [vp, ctypes.c_uint32]
    lib.pm_test_set_status.restype = ctypes.c_int
    lib.pm_selftest_wait.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32)]
    lib.pm_selftest_wait.restype = ctypes.c_int
    lib.pm_butterfly_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.pm_butterfly_peak.restype = ctypes.c_int
    del u32p
    _lib = lib
    return lib


def _check(code: int):
    if code != PM_OK:
        raise PolymultError(code, load().pm_last_error().decode(errors="replace"))


def _u32(arr, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(arr, dtype=np.uint32)
    if shape is not None and a.shape != shape:
        raise RuntimeError("operand size does not match N x L: got %s, want %s" % (a.shape, shape))
    return a


def host_pool_selftest(pools: int, runs: int, workers: int = 7, vary: bool = False, park: bool = False,
                       split: bool = False) -> int:
    """Stress test of the host staging pool (pm_selftest_host_pool); returns the failures."""
    f = ctypes.c_uint64()
    flags = (1 if vary else 0) | (2 if park else 0) | (4 if split else 0)
    _check(load().pm_selftest_host_pool(pools, runs, workers, flags, ctypes.byref(f)))
    return f.value


def digest_device(d_ptr: int, words: int, count: int = 1, stream: int = 0) -> np.ndarray:
    """pm_digest: 64-bit digests of `count` device arrays of `words` u32 words (contiguous)."""
    out = np.zeros(count, dtype=np.uint64)
    _check(load().pm_digest(d_ptr, words, count, stream or None, out.ctypes.data))
    return out


def digest_host(words) -> int:
    """pm_digest_host: the same digest of a host array."""
    a = np.ascontiguousarray(words, dtype=np.uint32).reshape(-1)
    return int(load().pm_digest_host(a.ctypes.data, a.size))


def wait_selftest(limit_clocks: int, device: int = 0) -> int:
    """The tensor-core kernels' bounded mbarrier waits made to run out (pm_selftest_wait);
    returns the kernel's status word (PM_DEVICE_WAIT expected, bit 8 never)."""
    st = ctypes.c_uint32(0)
    _check(load().pm_selftest_wait(device, limit_clocks, ctypes.byref(st)))
    return st.value


def butterfly_peak(device: int = 0) -> dict:
    """The NTT butterfly's rate with operands in registers (pm_butterfly_peak)."""
    a, b = ctypes.c_double(0), ctypes.c_double(0)
    _check(load().pm_butterfly_peak(device, ctypes.byref(a), ctypes.byref(b)))
    return {"bfly_per_s": a.value, "bfly_per_clk_sm": b.value}


def plan_selfcheck(N: int, W: int, q_limbs) -> int:
    """Host-only plan build + self-checks; returns the number of RNS primes."""
    L = (W + 31) // 32
    q = _u32(q_limbs)
    k = ctypes.c_int32(0)
    _check(load().pm_plan_selfcheck(N, W, L, q.ctypes.data, ctypes.byref(k)))
    return k.value


class Multiplier:
    """c = a*b mod (X^N+1, q) on one B200."""

    def __init__(self, N: int, W: int, q_limbs, gemm: str = "auto", device: int = 0):
        lib = load()
        self.N, self.W = int(N), int(W)
        self.L = (self.W + 31) // 32
        q = _u32(q_limbs)
        if q.size != self.L:
            raise RuntimeError("q must have L limbs")
        h = ctypes.c_void_p()
        _check(lib.pm_init(self.N, self.W, self.L, q.ctypes.data, GEMM_FORMS[gemm], device, ctypes.byref(h)))
        self._h = h

    def info(self) -> dict:
        inf = PmInfo()
        _check(load().pm_get_info(self._h, ctypes.byref(inf)))
        d = {f: getattr(inf, f) for f, _ in PmInfo._fields_}
        d["gemm"] = GEMM_NAMES.get(d["gemm_form"], "?")
        return d

    def multiply(self, a, b, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Host operands (N, L) u32 -> host result, through the chunked PCIe pipeline."""
        shape = (self.N, self.L)
        a, b = _u32(a, shape), _u32(b, shape)
        c = out if out is not None else np.empty(shape, dtype=np.uint32)
        _check(load().pm_run(self._h, a.ctypes.data, b.ctypes.data, c.ctypes.data))
        return c

    def multiply_device(self, a_ptr: int, b_ptr: int, c_ptr: int, count: int = 1, stream: int = 0):
        """Device-resident operands [count][N][L]; asynchronous on `stream` (cudaStream_t as int)."""
        _check(load().pm_run_device(self._h, a_ptr, b_ptr, c_ptr, count, stream or None))

    def multiply_device_static(self, a_ptr: int, b_ptr: int, c_ptr: int, stream: int = 0):
        """One device-resident multiply that allocates nothing (pm_run_device_static)."""
        _check(load().pm_run_device_static(self._h, a_ptr, b_ptr, c_ptr, stream or None))

    def time_stages(self, a_ptr: int, b_ptr: int, c_ptr: int, count: int = 1, reps: int = 3, stream: int = 0):
        """Mean per-kernel durations (ms) in launch order, keyed by STAGES."""
        ms = (ctypes.c_float * len(STAGES))()
        _check(load().pm_time_stages(self._h, a_ptr, b_ptr, c_ptr, count, reps, stream or None, ms))
        return dict(zip(STAGES, [float(x) for x in ms]))

    def sync(self):
        _check(load().pm_sync(self._h))

    def tune_pipeline(self, reps: int = 5, pinned: bool = False) -> dict:
        """Chooses the host pipeline's chunk schedule by measurement (pm_tune_pipeline): for calls
        on pageable buffers, or with pinned=True for calls whose a, b and c are page-locked."""
        inf = PmPipelineInfo()
        _check(load().pm_tune_pipeline(self._h, reps, PIPELINE_PINNED if pinned else 0, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in PmPipelineInfo._fields_}

    def set_pipeline(self, in_body: int, out_body: int, pinned: bool = False):
        """Sets the chunk schedule of one kind of call without measuring (pm_set_pipeline)."""
        _check(load().pm_set_pipeline(self._h, PIPELINE_PINNED if pinned else 0, in_body, out_body))

    def pipeline(self, pinned: bool = False) -> dict:
        inf = PmPipelineInfo()
        _check(load().pm_get_pipeline(self._h, PIPELINE_PINNED if pinned else 0, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in PmPipelineInfo._fields_}

    def close(self):
        if getattr(self, "_h", None):
            load().pm_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Multiplications of uneven points in one CUDA-graph launch (pm_batch_*).

    classes: sequence of (N, W, q_limbs, count, a_ptr, b_ptr, c_ptr[, w1]) -- device operands
    [count][N][L] each, w1 an explicit 4-step split (default -1: logN/2, or tuned).
    tune=True lets the autotuner choose split and GEMM form per class.
    """

    def __init__(self, classes, gemm: str = "auto", tune: bool = False, graph: bool = True, device: int = 0):
        lib = load()
        n = len(classes)
        arr = (PmBatchClass * n)()
        self._q = []
        for i, cls in enumerate(classes):
            N, W, q_limbs, count, a, b, c = cls[:7]
            w1 = int(cls[7]) if len(cls) > 7 else -1
            L = (int(W) + 31) // 32
            q = _u32(q_limbs)
            if q.size != L:
                raise RuntimeError("q must have L limbs")
            self._q.append(q)
            arr[i] = PmBatchClass(int(N), int(W), L, q.ctypes.data, int(count), a or None, b or None, c or None,
                                  w1)
        flags = (BATCH_TUNE if tune else 0) | (0 if graph else BATCH_NO_GRAPH)
        h = ctypes.c_void_p()
        _check(lib.pm_batch_init(arr, n, GEMM_FORMS[gemm], flags, device, ctypes.byref(h)))
        self._h = h

    def run(self, stream: int = 0):
        _check(load().pm_batch_run(self._h, stream or None))

    def sync(self):
        _check(load().pm_batch_sync(self._h))

    def info(self) -> dict:
        inf = PmBatchInfo()
        _check(load().pm_batch_get_info(self._h, ctypes.byref(inf)))
        return {f: getattr(inf, f) for f, _ in PmBatchInfo._fields_}

    def class_info(self, i: int) -> dict:
        inf = PmBatchClassInfo()
        _check(load().pm_batch_get_class(self._h, i, ctypes.byref(inf)))
        d = {f: getattr(inf, f) for f, _ in PmBatchClassInfo._fields_}
        d["gemm"] = GEMM_NAMES.get(d["gemm_form"], "?")
        return d

    def close(self):
        if getattr(self, "_h", None):
            load().pm_batch_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop with continuous batching over resident operands (pm_server_*).

    resident: (R, N, L) u32 host array of the fixed operands, kept on the device in NTT form.
    """

    def __init__(self, N: int, W: int, q_limbs, resident, hbm_budget: int = 150 * 10**9, max_batch: int = 8,
                 streams: int = 4, gemm: str = "auto", device: int = 0):
        lib = load()
        self.N, self.W = int(N), int(W)
        self.L = (self.W + 31) // 32
        q = _u32(q_limbs)
        res = np.ascontiguousarray(resident, dtype=np.uint32)
        if res.ndim != 3 or res.shape[1:] != (self.N, self.L):
            raise RuntimeError("resident operands must have shape (R, N, L)")
        h = ctypes.c_void_p()
        _check(lib.pm_server_init(self.N, self.W, self.L, q.ctypes.data, res.ctypes.data, res.shape[0],
                                  int(hbm_budget), max_batch, streams, GEMM_FORMS[gemm], device, ctypes.byref(h)))
        self._h = h
        self.nresident = res.shape[0]

    def pinned(self, count: int) -> np.ndarray:
        """(count, N, L) u32 array in pinned host memory owned by the server."""
        nbytes = count * self.N * self.L * 4
        p = ctypes.c_void_p()
        _check(load().pm_server_host_alloc(self._h, nbytes, ctypes.byref(p)))
        buf = (ctypes.c_uint32 * (count * self.N * self.L)).from_address(p.value)
        return np.ctypeslib.as_array(buf).reshape(count, self.N, self.L)

    def run(self, t_arrive, sel, a_bufs, c_bufs, digests: bool = False):
        """Plays the request stream; a_bufs[i] / c_bufs[i] are (N, L) u32 host arrays.
        Returns (latency seconds per request, stats dict), plus each request's result digest
        (pm_digest, computed on the device) with digests=True."""
        n = len(t_arrive)
        t = np.ascontiguousarray(t_arrive, dtype=np.float64)
        sv = np.ascontiguousarray(sel, dtype=np.uint32)
        ap = (ctypes.c_void_p * n)(*[x.ctypes.data for x in a_bufs])
        cp = (ctypes.c_void_p * n)(*[x.ctypes.data for x in c_bufs])
        lat = np.zeros(n, dtype=np.float64)
        dig = np.zeros(n, dtype=np.uint64) if digests else None
        st = PmServeStats()
        _check(load().pm_server_run(self._h, n, t.ctypes.data, sv.ctypes.data, ap, cp, lat.ctypes.data,
                                    ctypes.byref(st), dig.ctypes.data if digests else None))
        stats = {f: getattr(st, f) for f, _ in PmServeStats._fields_}
        return (lat, stats, dig) if digests else (lat, stats)

    def close(self):
        if getattr(self, "_h", None):
            load().pm_server_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -- the reference's three entry points -------------------------------------------------

def fherma_init(N: int, W: int, L: int, q_limbs, gemm: str = "auto") -> Multiplier:
    if L != (W + 31) // 32:
        raise RuntimeError("inconsistent W / L")
    try:
        return Multiplier(N, W, q_limbs, gemm=gemm)
    except PolymultError as e:
        raise RuntimeError(str(e)) from e


def fherma_run(state: Multiplier, a, b) -> np.ndarray:
    try:
        return state.multiply(a, b)
    except PolymultError as e:
        raise RuntimeError(str(e)) from e


def fherma_free(state: Optional[Multiplier]) -> None:
    if state is not None:
        state.close()
