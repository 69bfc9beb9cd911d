"""Loader of libofgpu.so and the per-device engine context.

The product path has no CPU fallback: if the library or a GPU is missing,
every pricing call raises `GpuUnavailable`.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import _abi as A
from .core import PricingError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libofgpu.so")

# Every symbol include/of_gpu.h declares.
EXPORTED = [
    "of_abi_version", "of_ctx_create", "of_ctx_destroy", "of_status_str", "of_ctx_last_error", "of_ctx_set_stream",
    "of_ctx_get_stream", "of_device_sm_count", "of_mc_run", "of_mc_strip", "of_strip_plan_create",
    "of_strip_plan_launch", "of_strip_plan_results", "of_strip_plan_destroy", "of_mc_price_book",
    "of_book_plan_create", "of_book_plan_launch", "of_book_plan_results", "of_book_plan_info",
    "of_book_plan_destroy", "of_mc_european_pathwise_aad", "of_heston_price_delta_aad", "of_mc_greek_estimators",
    "of_lsm_price", "of_xoshiro_jump", "of_heston_price_adjoint", "of_mc_european_gpu", "of_mc_strip_noalloc",
    "of_measure_device_peaks", "of_lsm_bermudan", "of_mc_european_qmc", "of_autotune_strip", "of_autotune_book",
    "of_test_bounded_wait", "of_book_price_to_stderr", "of_book_plan_greeks", "of_mc_price_book_greeks",
    "of_book_price_to_stderr_greeks", "of_lsm_barrier",
]


class GpuUnavailable(RuntimeError):
    """The CUDA library or a GPU is missing; the engine has no CPU path."""


class OfGpuError(RuntimeError):
    """A device-side failure (CUDA error, allocation failure, timeout)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(message)


_lib = None
_lock = threading.Lock()


def _declare(L):
    P = C.POINTER
    vp = C.c_void_p
    L.of_abi_version.restype = C.c_int
    L.of_ctx_create.argtypes = [C.c_int, P(vp)]
    L.of_ctx_destroy.argtypes = [vp]
    L.of_ctx_destroy.restype = None
    L.of_status_str.restype = C.c_char_p
    L.of_status_str.argtypes = [C.c_int]
    L.of_ctx_last_error.restype = C.c_char_p
    L.of_ctx_last_error.argtypes = [vp]
    L.of_ctx_set_stream.argtypes = [vp, vp]
    L.of_ctx_get_stream.argtypes = [vp, P(vp)]
    L.of_device_sm_count.argtypes = [vp]
    L.of_mc_run.argtypes = [vp, P(A.OfModel), P(A.OfPayoff), P(A.OfMcConfig), P(A.OfMcResult)]
    L.of_mc_strip.argtypes = [vp, P(A.OfModel), C.c_int32, P(C.c_double), C.c_int64, P(A.OfMcConfig),
                              P(A.OfMcResult)]
    L.of_strip_plan_create.argtypes = [vp, P(A.OfModel), C.c_int32, P(C.c_double), C.c_int64, P(A.OfMcConfig),
                                       P(vp)]
    L.of_strip_plan_launch.argtypes = [vp]
    L.of_strip_plan_results.argtypes = [vp, P(A.OfMcResult)]
    L.of_strip_plan_destroy.argtypes = [vp]
    L.of_strip_plan_destroy.restype = None
    L.of_mc_price_book.argtypes = [vp, P(A.OfBookEntry), C.c_int64, P(A.OfBookConfig), P(A.OfMcResult)]
    L.of_book_plan_create.argtypes = [vp, P(A.OfBookEntry), C.c_int64, P(A.OfBookConfig), P(vp)]
    L.of_book_plan_launch.argtypes = [vp]
    L.of_book_plan_results.argtypes = [vp, P(A.OfMcResult)]
    L.of_book_plan_info.argtypes = [vp, P(C.c_int32), P(C.c_int32), P(C.c_int64), P(C.c_double)]
    L.of_book_plan_destroy.argtypes = [vp]
    L.of_book_plan_destroy.restype = None
    for name in ["of_mc_european_pathwise_aad", "of_heston_price_delta_aad", "of_mc_greek_estimators"]:
        getattr(L, name).argtypes = [vp, P(A.OfGreeksParams), P(A.OfGreeksResult)]
        getattr(L, name).restype = C.c_int
    L.of_lsm_price.argtypes = [vp, P(A.OfLsmContract), C.c_int64, P(A.OfLsmConfig), P(A.OfLsmResult)]
    L.of_lsm_price.restype = C.c_int
    L.of_lsm_barrier.argtypes = [vp, P(A.OfLsmBarrierContract), P(A.OfLsmConfig), P(A.OfLsmResult)]
    L.of_lsm_barrier.restype = C.c_int
    L.of_xoshiro_jump.argtypes = [vp, C.c_uint64, P(C.c_uint64), C.c_int64, P(C.c_uint64)]
    L.of_xoshiro_jump.restype = C.c_int
    L.of_heston_price_adjoint.argtypes = [vp, P(A.OfHestonAdjointParams), P(A.OfAdjointResult)]
    L.of_heston_price_adjoint.restype = C.c_int
    L.of_mc_european_gpu.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int64,
                                     C.c_int64, C.c_uint32, C.c_int32, P(C.c_double), P(C.c_double)]
    L.of_mc_european_gpu.restype = C.c_int
    L.of_mc_strip_noalloc.argtypes = [vp, P(A.OfModel), C.c_int32, P(C.c_double), C.c_int64, P(A.OfMcConfig),
                                      P(A.OfMcResult), C.c_char_p, C.c_size_t]
    L.of_mc_strip_noalloc.restype = C.c_int
    L.of_measure_device_peaks.argtypes = [vp, P(A.OfDevicePeaks)]
    L.of_measure_device_peaks.restype = C.c_int
    L.of_lsm_bermudan.argtypes = [vp, P(A.OfBermudanContract), P(A.OfLsmConfig), P(A.OfLsmResult),
                                  P(A.OfBoundaryPoint), C.c_int64, P(C.c_int64)]
    L.of_lsm_bermudan.restype = C.c_int
    L.of_mc_european_qmc.argtypes = [vp, P(A.OfQmcParams), P(A.OfMcResult)]
    L.of_mc_european_qmc.restype = C.c_int
    L.of_autotune_strip.argtypes = [vp, P(A.OfModel), C.c_int32, P(C.c_double), C.c_int64, P(A.OfMcConfig),
                                    P(A.OfTuneCandidate), C.c_int32, C.c_int32, P(C.c_int32)]
    L.of_autotune_strip.restype = C.c_int
    L.of_autotune_book.argtypes = [vp, P(A.OfBookEntry), C.c_int64, P(A.OfBookConfig), P(A.OfTuneCandidate),
                                   C.c_int32, C.c_int32, P(C.c_int32)]
    L.of_autotune_book.restype = C.c_int
    L.of_test_bounded_wait.argtypes = [vp, C.c_int32, C.c_uint32, P(C.c_int32), P(C.c_double)]
    L.of_test_bounded_wait.restype = C.c_int
    L.of_book_price_to_stderr.argtypes = [vp, P(A.OfBookEntry), C.c_int64, P(A.OfBookConfig), P(A.OfStderrTarget),
                                          P(A.OfMcResult), P(C.c_int64), P(A.OfStderrRound), P(C.c_int32)]
    L.of_book_price_to_stderr.restype = C.c_int
    L.of_book_plan_greeks.argtypes = [vp, P(A.OfBookGreeks)]
    L.of_book_plan_greeks.restype = C.c_int
    L.of_mc_price_book_greeks.argtypes = [vp, P(A.OfBookEntry), C.c_int64, P(A.OfBookConfig), P(A.OfMcResult),
                                          P(A.OfBookGreeks)]
    L.of_mc_price_book_greeks.restype = C.c_int
    L.of_book_price_to_stderr_greeks.argtypes = [vp, P(A.OfBookEntry), C.c_int64, P(A.OfBookConfig),
                                                 P(A.OfStderrTarget), P(A.OfMcResult), P(A.OfBookGreeks),
                                                 P(C.c_int64), P(A.OfStderrRound), P(C.c_int32)]
    L.of_book_price_to_stderr_greeks.restype = C.c_int
    for name in ["of_ctx_create", "of_ctx_set_stream", "of_ctx_get_stream", "of_mc_run", "of_mc_strip",
                 "of_strip_plan_create", "of_strip_plan_launch", "of_strip_plan_results", "of_mc_price_book",
                 "of_book_plan_create", "of_book_plan_launch", "of_book_plan_results", "of_book_plan_info"]:
        getattr(L, name).restype = C.c_int


def load():
    """Loads libofgpu.so (building it first when nvcc is available)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                try:
                    from .build import build
                    build()
                except Exception as e:  # pragma: no cover - depends on toolchain
                    raise GpuUnavailable(f"libofgpu.so is missing and could not be built: {e}") from e
            L = C.CDLL(LIB_PATH)
            _declare(L)
            if L.of_abi_version() != 1:
                raise GpuUnavailable("libofgpu.so ABI version mismatch")
            _lib = L
    return _lib


def raise_for(status: int, ctx_handle=None):
    if status == A.OF_OK:
        return
    L = load()
    msg = L.of_ctx_last_error(ctx_handle).decode() if ctx_handle else L.of_status_str(status).decode()
    if status in (A.OF_ERR_INVALID_INPUT, A.OF_ERR_UNSUPPORTED):
        raise PricingError.InvalidInput(msg)
    if status == A.OF_ERR_NUMERICAL:
        raise PricingError.NumericalError(msg)
    if status == A.OF_ERR_CONVERGENCE:
        raise PricingError.ConvergenceFailure(msg)
    raise OfGpuError(status, f"{L.of_status_str(status).decode()}: {msg}")


class Context:
    """One of_ctx (stream + pooled device buffers) on one device."""

    def __init__(self, device: int = 0):
        L = load()
        h = C.c_void_p()
        st = L.of_ctx_create(device, C.byref(h))
        if st != A.OF_OK:
            raise GpuUnavailable(f"of_ctx_create(device={device}) failed: {L.of_status_str(st).decode()}")
        self._L = L
        self.handle = h
        self.device = device
        self.lock = threading.Lock()

    def check(self, status: int):
        raise_for(status, self.handle)

    @property
    def sm_count(self) -> int:
        return self._L.of_device_sm_count(self.handle)

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        self.check(self._L.of_ctx_get_stream(self.handle, C.byref(s)))
        return s.value or 0

    def set_stream(self, ptr: int):
        self.check(self._L.of_ctx_set_stream(self.handle, C.c_void_p(ptr or None)))

    def device_peaks(self) -> dict:
        """MUFU, FP32 FMA and FP64 FMA throughput of this GPU, measured by probe kernels."""
        out = A.OfDevicePeaks()
        with self.lock:
            self.check(self._L.of_measure_device_peaks(self.handle, C.byref(out)))
        return {"sfu_ops_per_s": out.sfu_ops_per_s, "fp32_flops_per_s": out.fp32_flops_per_s,
                "fp64_flops_per_s": out.fp64_flops_per_s, "probe_ms": out.probe_ms}

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self._L.of_ctx_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


_contexts = {}


def context(device: int = 0) -> Context:
    with _lock:
        ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _contexts.setdefault(device, ctx)
            ctx = _contexts[device]
    return ctx
