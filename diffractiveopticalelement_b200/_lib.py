"""ctypes binding of ``libdoe_b200.so`` (the C ABI declared in include/doe_b200.h).

The engine has no CPU implementation: importing the package is cheap, but the
first call that needs the device raises :class:`EngineUnavailable` when the
library is missing or no CUDA device is visible. Nothing here falls back to host
arithmetic.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdoe_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "doe_b200.h")

DOE_OK = 0
DOE_ERR_NOT_POW2 = 1
DOE_ERR_SIZE_MISMATCH = 2
DOE_ERR_BAD_ARG = 3
DOE_ERR_CUDA = 4
DOE_ERR_TIMEOUT = 5
DOE_ERR_UNSUPPORTED = 6
DOE_ERR_NO_DEVICE = 7


class DOEError(Exception):
    """Raised for a non-zero doe_status; ``code`` holds the status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class EngineUnavailable(RuntimeError):
    """The CUDA engine cannot run here (library not built or no GPU)."""


_dp = C.POINTER(C.c_double)
_vp = C.c_void_p

DOE_ALG_GS, DOE_ALG_WGS, DOE_ALG_FOURIER, DOE_ALG_WGS_FOURIER = 0, 1, 2, 3


class DesignDesc(C.Structure):
    """doe_design_desc (include/doe_b200.h)."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("lambda_", C.c_double), ("z", C.c_double), ("algorithm", C.c_int), ("iterations", C.c_int),
                ("feedback", C.c_double), ("escape", C.c_int), ("beta", C.c_double), ("seed", C.c_double),
                ("illumination", _dp), ("target_amp", _dp), ("roi", _dp), ("init_phase", _dp)]


class DesignResult(C.Structure):
    """doe_design_result."""
    _fields_ = [("phase", _dp), ("amplitude", _dp), ("intensity", _dp), ("error", _dp),
                ("efficiency", _dp), ("weights", _dp), ("rmse", C.c_double)]


class DesignDevDesc(C.Structure):
    """doe_design_dev_desc (device-resident FP32 planes)."""
    _fields_ = [("batch", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("lambda_", C.c_double), ("z", C.c_double), ("lambdas", _dp), ("zs", _dp),
                ("algorithm", C.c_int), ("iterations", C.c_int), ("feedback", C.c_double), ("escape", C.c_int),
                ("beta", C.c_double), ("illumination", _vp), ("target_amp", _vp), ("roi", _vp), ("phase", _vp),
                ("amplitude", _vp), ("weights", _vp), ("error", _vp), ("efficiency", _vp), ("rmse", _vp),
                ("rmse_goal", C.c_double), ("screen_irr", _vp), ("iterations_used", _vp)]


class MultiplaneDevDesc(C.Structure):
    """doe_multiplane_dev_desc (device-resident FP32 planes)."""
    _fields_ = [("batch", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("lambda_", C.c_double), ("nplanes", C.c_int), ("z", _dp), ("weight", _dp), ("iterations", C.c_int),
                ("illumination", _vp), ("target_amp", _vp), ("roi", _vp), ("phase", _vp), ("error", _vp),
                ("efficiency", _vp), ("per_plane_error", _vp)]



class PhaseLossDesc(C.Structure):
    """doe_phase_loss_desc (device-resident FP32 planes)."""
    _fields_ = [("batch", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("lambda_", C.c_double), ("z", C.c_double), ("illumination", _vp), ("target_amp", _vp),
                ("roi", _vp), ("phase", _vp), ("grad", _vp), ("loss", _vp)]


_lib = None
_lock = threading.Lock()


def _declare(L):
    i, d, u64 = C.c_int, C.c_double, C.c_ulonglong
    ctxp = C.c_void_p
    sig = {
        "doe_abi_version": (i, []),
        "doe_ctx_create": (i, [i, C.POINTER(C.c_void_p)]),
        "doe_ctx_destroy": (None, [ctxp]),
        "doe_last_error": (C.c_char_p, [ctxp]),
        "doe_ctx_stream": (C.c_void_p, [ctxp]),
        "doe_ctx_synchronize": (i, [ctxp]),
        "doe_host_alloc": (i, [ctxp, C.POINTER(C.c_void_p), u64]),
        "doe_host_free": (i, [ctxp, _vp]),
        "doe_fft2d": (i, [ctxp, _dp, _dp, i, i, i]),
        "doe_asm_transfer": (i, [ctxp, i, i, d, d, d, d, i, i, d, _dp, _dp, _dp]),
        "doe_asm": (i, [ctxp, _dp, _dp, i, i, d, d, d, d, i, i, d]),
        "doe_asm_sweep": (i, [ctxp, _dp, _dp, i, i, d, d, d, _dp, i, i, i, d, _dp, _dp]),
        "doe_focal_plane": (i, [ctxp, _dp, _dp, i, i, d, d, d, d, _dp, _dp, _dp]),
        "doe_fresnel": (i, [ctxp, _dp, _dp, i, i, d, d, d, d, _dp, _dp, _dp]),
        "doe_fresnel_inverse": (i, [ctxp, _dp, _dp, i, i, d, d, d, d, d, d, _dp, _dp]),
        "doe_fft2d_dev": (i, [ctxp, _vp, i, i, i, i]),
        "doe_asm_sweep_dev": (i, [ctxp, _vp, i, i, i, d, d, _dp, _dp, i, i, i, d, _vp]),
        "doe_asm_c64_noalloc": (i, [_vp, _vp, i, i, d, d, d, d, i, i, d, _vp, C.c_char_p, i]),
        "doe_design": (i, [ctxp, C.POINTER(DesignDesc), C.POINTER(DesignResult)]),
        "doe_random_phase": (i, [i, i, d, _dp]),
        "doe_simulate": (i, [ctxp, _dp, _dp, i, i, d, d, d, d, i, i, i, _dp, _dp, _dp]),
        "doe_simulate_sweep": (i, [ctxp, _dp, _dp, i, i, d, d, d, _dp, i, i, i, i, _dp, _dp, _dp]),
        "doe_screen_metrics": (i, [ctxp, _dp, _dp, i, i, d, d, _dp, _dp, _dp, d, d, _dp]),
        "doe_screen_metrics_dev": (i, [ctxp, i, i, i, _vp, _vp, C.c_longlong, _vp, _vp, C.c_longlong, d, d, d, d,
                                       _vp]),
        "doe_design_batch": (i, [ctxp, i, C.POINTER(DesignDesc), C.POINTER(DesignResult)]),
        "doe_design_dev": (i, [ctxp, C.POINTER(DesignDevDesc)]),
        "doe_autotune_design": (i, [ctxp, C.POINTER(DesignDevDesc), i, C.POINTER(C.c_int)]),
        "doe_multiplane_dev": (i, [ctxp, C.POINTER(MultiplaneDevDesc)]),
        "doe_phase_loss_grad": (i, [ctxp, C.POINTER(PhaseLossDesc)]),
        "doe_design_multi_create": (i, [ctxp, C.POINTER(C.c_void_p)]),
        "doe_error_diffusion": (i, [ctxp, i, C.c_longlong, i, i, i, _dp, _dp]),
        "doe_hologram_record": (i, [ctxp, _dp, _dp, _dp, _dp, C.c_longlong, i, i, _dp, _dp, _dp, _dp, _dp]),
        "doe_hologram_reconstruct": (i, [ctxp, _dp, _dp, _dp, _dp, i, i, d, d, d, d, i, i, d] + [_dp] * 6),
        "doe_modal_intensity": (i, [ctxp, i, _dp, _dp, i, i, _dp, d, d, d, d, i, i, d, _dp]),
        "doe_partially_coherent_modes": (i, [ctxp, i, i, d, d, i, d, d, d, _dp, _dp]),
        "doe_screen_metrics_full": (i, [ctxp, _dp, _dp, i, i, d, d, _dp, _dp, _dp, _dp, d, d, i, i, _dp]),
        "doe_ctx_get_tuning": (i, [ctxp, C.c_char_p, C.POINTER(C.c_longlong)]),
        "doe_design_multi_destroy": (None, [_vp]),
        "doe_design_multi_run": (i, [_vp, i, C.POINTER(DesignDevDesc), i]),
        "doe_phase_supervised_grad": (i, [ctxp, C.c_longlong, _vp, _vp, _vp, _vp]),
        "doe_surrogate_create": (i, [ctxp, i, i, i, i, C.c_ulonglong, C.POINTER(C.c_void_p)]),
        "doe_surrogate_destroy": (None, [_vp]),
        "doe_surrogate_param_count": (C.c_longlong, [_vp]),
        "doe_surrogate_params": (i, [_vp, C.POINTER(C.c_float), i]),
        "doe_surrogate_set_params": (i, [_vp, C.POINTER(C.c_float)]),
        "doe_surrogate_forward": (i, [_vp, i, _vp, _vp, _vp]),
        "doe_surrogate_backward": (i, [_vp, _vp]),
        "doe_surrogate_zero_grad": (i, [_vp]),
        "doe_surrogate_grads_dev": (i, [_vp, _vp]),
        "doe_surrogate_set_grads_dev": (i, [_vp, _vp]),
        "doe_surrogate_adam": (i, [_vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]),
        "doe_multiplane": (i, [ctxp, i, i, d, d, d, _dp, i, _dp, _dp, _dp, _dp, i, _dp, _dp, _dp, _dp, _dp]),
        "doe_autotune": (i, [ctxp, i, i, d, d, d, d, C.POINTER(C.c_int)]),
        "doe_ctx_set_tuning": (i, [ctxp, C.c_char_p, C.c_longlong]),
        "doe_ctx_launch_count": (C.c_ulonglong, [ctxp]),
        "doe_ctx_set_profiling": (i, [ctxp, i]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return L


def load_library():
    """Load (not build) the engine library; raise EngineUnavailable if absent."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise EngineUnavailable(
                    f"{LIB_PATH} is missing: build it with "
                    "`python -m diffractiveopticalelement_b200.build` (needs nvcc)")
            _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def declared_functions() -> list[str]:
    """Entry points declared in include/doe_b200.h."""
    import re
    src = open(HEADER).read()
    return re.findall(r"^\s*(?:int|void|long long|const char\s*\*|void\s*\*)\s*(doe_\w+)\s*\(", src, re.M)


class Context:
    """One engine context (CUDA stream + scratch) on one device."""

    def __init__(self, device: int = 0):
        L = load_library()
        h = C.c_void_p()
        rc = L.doe_ctx_create(int(device), C.byref(h))
        if rc == DOE_ERR_NO_DEVICE:
            raise EngineUnavailable("no CUDA device is visible: the engine has no CPU path")
        if rc != DOE_OK:
            raise DOEError(rc, f"doe_ctx_create failed with status {rc}")
        self.h = h
        self.device = device
        self.lib = L

    def check(self, rc: int):
        if rc != DOE_OK:
            msg = self.lib.doe_last_error(self.h)
            msg = msg.decode() if msg else f"status {rc}"
            raise DOEError(rc, msg)

    def synchronize(self):
        self.check(self.lib.doe_ctx_synchronize(self.h))

    @property
    def stream(self) -> int:
        return self.lib.doe_ctx_stream(self.h) or 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.doe_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_ctx: dict[int, Context] = {}


def context(device: int | None = None) -> Context:
    """Shared per-thread-agnostic default context for `device` (default 0)."""
    dev = 0 if device is None else int(device)
    with _lock:
        c = _ctx.get(dev)
    if c is None:
        c = Context(dev)
        with _lock:
            _ctx[dev] = c
    return c


def f64(a) -> np.ndarray:
    """C-contiguous float64 view/copy of a plane."""
    return np.ascontiguousarray(a, dtype=np.float64)


def dp(a):
    return None if a is None else a.ctypes.data_as(_dp)
