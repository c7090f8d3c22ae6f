"""ctypes mirror of include/csd_shore.h and the loader of libcsdshore.so.

The CUDA library is the only implementation of the fit: if it is missing or
cannot be loaded this module raises, it never substitutes another code path.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcsdshore.so"

# enum csd_status / csd_regularization / csd_alpha_mode / csd_precision
OK, ERR_INVALID, ERR_FIT_REFUSED, ERR_NUMERICAL, ERR_CUDA, ERR_TIMEOUT = range(6)
REG_L1, REG_L2, REG_NONNEG = 1, 2, 3
ALPHA_FIXED, ALPHA_RATIO, ALPHA_PATH_BIC, ALPHA_L2_ANCHORED = range(4)
PRECISION_FP64, PRECISION_MIXED, PRECISION_MIXED_KKT, PRECISION_FP64_KKT = 0, 1, 2, 3


class Gtab(C.Structure):
    _fields_ = [
        ("bvals", C.POINTER(C.c_double)),
        ("bvecs", C.POINTER(C.c_double)),
        ("n", C.c_int32),
        ("big_delta", C.c_double),
        ("small_delta", C.c_double),
        ("b0_threshold", C.c_double),
    ]


class Spec(C.Structure):
    _fields_ = [
        ("radial_order", C.c_int32),
        ("zeta", C.c_double),
        ("regularization", C.c_int32),
        ("alpha_mode", C.c_int32),
        ("alpha", C.c_double),
        ("alpha_ratio", C.c_double),
        ("path_n_alphas", C.c_int32),
        ("path_eps", C.c_double),
        ("slack", C.c_double),
        ("max_iter", C.c_int32),
        ("tol", C.c_double),
        ("non_negative", C.c_int32),
        ("lambda_n", C.c_double),
        ("lambda_l", C.c_double),
        ("nonneg_max_iter", C.c_int32),
        ("nonneg_tol", C.c_double),
        ("nonneg_epsilon", C.c_double),
        ("diagnostics", C.c_int32),
        ("allow_single_shell", C.c_int32),
        ("precision", C.c_int32),
    ]


class FitResult(C.Structure):
    _fields_ = [
        ("coefficients", C.c_void_p),
        ("r2", C.c_void_p),
        ("residual_l2", C.c_void_p),
        ("iterations", C.c_void_p),
        ("regularization_kind", C.c_void_p),
        ("alpha", C.c_void_p),
        ("bic", C.c_void_p),
        ("rss_l2", C.c_void_p),
        ("coef64", C.c_void_p),
        ("converged", C.c_void_p),
        ("n_coeffs", C.c_int32),
        ("n_voxels", C.c_int64),
        ("has_alpha_distribution", C.c_int32),
        ("alpha_distribution", C.c_double * 3),
        ("representative_alpha", C.c_double),
        ("big_delta_seconds", C.c_double),
        ("small_delta_seconds", C.c_double),
        ("tau_seconds", C.c_double),
        ("delta_source", C.c_int32),
        ("n_shells", C.c_int32),
        ("dwi_shells", C.c_double * 32),
        ("lmax", C.c_int32),
        ("n_constraint_dirs", C.c_int32),
        ("total_iterations", C.c_uint64),
        ("warnings", C.c_char * 2048),
    ]


class Timing(C.Structure):
    _fields_ = [
        ("ms_setup", C.c_float),
        ("ms_rhs", C.c_float),
        ("ms_solve", C.c_float),
        ("ms_epilogue", C.c_float),
        ("ms_total", C.c_float),
        ("launches", C.c_int32),
        ("ms_solve_kernel", C.c_float),
        ("tensor_flops", C.c_double),
        ("ms_mixed_kernel", C.c_float),
        ("int8_tensor_ops", C.c_double),
        ("fp64_rerun_voxels", C.c_uint64),
        ("fista_warps", C.c_int32),
        ("fista_tune_ms12", C.c_float),
        ("fista_tune_ms16", C.c_float),
        ("fista_parked", C.c_int64),
        ("ms_kkt_iterate", C.c_float),
        ("ms_kkt_polish", C.c_float),
        ("ms_kkt_fallback", C.c_float),
        ("kkt_fallback_voxels", C.c_int64),
        ("kkt_uncertified", C.c_int64),
        ("kkt_rounds", C.c_uint64),
        ("tf32_tensor_flops", C.c_double),
        ("kkt_max", C.c_double),
        ("ms_host_gather", C.c_float),
        ("ms_host_copy_out", C.c_float),
        ("kkt_iterations", C.c_int32),
        ("kkt_tune_ms", C.c_float * 4),
        ("kkt_overflow", C.c_int64),
    ]


# csd_set_option options
OPT_FISTA_SHAPE = 1
OPT_FISTA_SCHEDULE = 2
OPT_KKT_ITERATIONS = 3
OPT_TENSOR_WAIT_NS = 4
OPT_KKT_ROUNDS = 5
OPT_ICLS = 6


# Every symbol include/csd_shore.h declares, for load checks.
EXPORTS = (
    "csd_version",
    "csd_abi_version",
    "csd_default_spec",
    "csd_shore_n_coeffs",
    "csd_create",
    "csd_destroy",
    "csd_shore_fit_volume",
    "csd_shore_fit_volume_device",
    "csd_shore_design_matrix",
    "csd_last_timing",
    "csd_set_option",
    "csd_shore_fista_batch_noalloc",
    "csd_shore_predict",
    "csd_shore_odf_sh",
    "csd_shore_microstructure",
    "csd_shore_fit_batch_device",
    "csd_shore_fit_adjoint_device",
    "csd_apply_rows_device",
    "csd_shore_odf_matrix",
    "csd_shore_rtop_device",
    "csd_shore_rtop_adjoint_device",
    "csd_geodesic_sphere",
    "csd_shore_odf_peaks",
    "csd_shore_fit_graddev_device",
)

_lib = None
_lock = threading.Lock()


def _declare(lib: C.CDLL) -> C.CDLL:
    lib.csd_version.restype = C.c_char_p
    lib.csd_version.argtypes = []
    lib.csd_abi_version.restype = C.c_int
    lib.csd_abi_version.argtypes = []
    lib.csd_default_spec.restype = None
    lib.csd_default_spec.argtypes = [C.POINTER(Spec)]
    lib.csd_shore_n_coeffs.restype = C.c_int
    lib.csd_shore_n_coeffs.argtypes = [C.c_int32]
    lib.csd_create.restype = C.c_int
    lib.csd_create.argtypes = [C.POINTER(C.c_void_p), C.c_int32, C.c_char_p, C.c_size_t]
    lib.csd_destroy.restype = None
    lib.csd_destroy.argtypes = [C.c_void_p]
    fit_args = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                C.POINTER(Gtab), C.POINTER(Spec), C.POINTER(FitResult)]
    lib.csd_shore_fit_volume.restype = C.c_int
    lib.csd_shore_fit_volume.argtypes = fit_args + [C.c_char_p, C.c_size_t]
    lib.csd_shore_fit_volume_device.restype = C.c_int
    lib.csd_shore_fit_volume_device.argtypes = fit_args + [C.c_void_p, C.c_char_p, C.c_size_t]
    lib.csd_shore_design_matrix.restype = C.c_int
    lib.csd_shore_design_matrix.argtypes = [C.c_void_p, C.POINTER(Gtab), C.c_int32, C.c_double,
                                            C.c_void_p, C.c_char_p, C.c_size_t]
    lib.csd_last_timing.restype = C.c_int
    lib.csd_last_timing.argtypes = [C.c_void_p, C.POINTER(Timing)]
    lib.csd_set_option.restype = C.c_int
    lib.csd_set_option.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
    lib.csd_shore_fista_batch_noalloc.restype = C.c_int
    lib.csd_shore_fista_batch_noalloc.argtypes = [C.POINTER(Gtab), C.POINTER(Spec), C.c_void_p, C.c_int64,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    vol = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.c_double]
    lib.csd_shore_predict.restype = C.c_int
    lib.csd_shore_predict.argtypes = vol + [C.POINTER(Gtab), C.c_void_p, C.c_char_p, C.c_size_t]
    lib.csd_shore_odf_sh.restype = C.c_int
    lib.csd_shore_odf_sh.argtypes = vol + [C.c_int32, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    lib.csd_shore_microstructure.restype = C.c_int
    lib.csd_shore_microstructure.argtypes = vol + [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_float] + \
        [C.c_void_p] * 6 + [C.c_char_p, C.c_size_t]
    tail = [C.c_void_p, C.c_char_p, C.c_size_t]  # stream, err, err_len
    lib.csd_shore_fit_batch_device.restype = C.c_int
    lib.csd_shore_fit_batch_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(Gtab), C.POINTER(Spec),
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + tail
    lib.csd_shore_fit_adjoint_device.restype = C.c_int
    lib.csd_shore_fit_adjoint_device.argtypes = [C.c_void_p, C.POINTER(Gtab), C.POINTER(Spec), C.c_void_p,
                                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p] + tail
    lib.csd_apply_rows_device.restype = C.c_int
    lib.csd_apply_rows_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64,
                                          C.c_void_p] + tail
    lib.csd_shore_odf_matrix.restype = C.c_int
    lib.csd_shore_odf_matrix.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_void_p, C.c_int32, C.c_void_p,
                                         C.c_char_p, C.c_size_t]
    lib.csd_shore_rtop_device.restype = C.c_int
    lib.csd_shore_rtop_device.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_void_p, C.c_int64,
                                          C.c_void_p] + tail
    lib.csd_shore_rtop_adjoint_device.restype = C.c_int
    lib.csd_shore_rtop_adjoint_device.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_void_p, C.c_int64,
                                                  C.c_void_p, C.c_void_p] + tail
    lib.csd_shore_odf_peaks.restype = C.c_int
    lib.csd_shore_odf_peaks.argtypes = vol + [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double] + \
        [C.c_void_p] * 4 + [C.c_char_p, C.c_size_t]
    lib.csd_shore_fit_graddev_device.restype = C.c_int
    lib.csd_shore_fit_graddev_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(Gtab),
                                                 C.POINTER(Spec)] + [C.c_void_p] * 8 + tail
    lib.csd_geodesic_sphere.restype = C.c_int
    lib.csd_geodesic_sphere.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_int32]
    return lib


def load() -> C.CDLL:
    """Load libcsdshore.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH.name} is not built; run `python -m cs_dmri_b200.build` "
                    "(the fit has no implementation other than the CUDA library)")
            _lib = _declare(C.CDLL(str(LIB_PATH)))
    return _lib


class CsdError(ValueError):
    """Raised for a non-zero status; ValueError like the reference's map_err
    (python/src/lib.rs:33-35)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def check(code: int, err) -> None:
    if code != OK:
        raise CsdError(code, err.value.decode("utf-8", "replace"))


_handles: dict[int, C.c_void_p] = {}


def handle(device: int = 0) -> C.c_void_p:
    """Process-wide handle of `device` (created on first use)."""
    lib = load()
    with _lock:
        h = _handles.get(device)
        if h is None:
            h = C.c_void_p()
            err = C.create_string_buffer(1024)
            check(lib.csd_create(C.byref(h), device, err, len(err)), err)
            _handles[device] = h
    return h


def reset_handle(device: int = 0) -> None:
    """Destroy the process-wide handle of `device`: the next call creates a
    new one and pays the per-table set-up, the autotuning and the buffer
    allocations again (a cold start)."""
    lib = load()
    with _lock:
        h = _handles.pop(device, None)
    if h is not None and h.value:
        lib.csd_destroy(h)


def default_spec() -> Spec:
    s = Spec()
    load().csd_default_spec(C.byref(s))
    return s


def set_option(option: int, value: int, device: int = 0) -> None:
    """Set a tuning option of the device's shared handle (csd_set_option)."""
    if load().csd_set_option(handle(device), int(option), int(value)) != OK:
        raise ValueError(f"invalid option {option} or value {value}")


def last_timing(device: int = 0) -> Timing:
    t = Timing()
    load().csd_last_timing(handle(device), C.byref(t))
    return t


class PrivateHandle:
    """A handle of its own (device memory, streams, set-up cache) for a user
    that must not share scratch buffers with other calls, such as a captured
    CUDA graph whose kernels keep pointing at them; released with the object."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.h = C.c_void_p()
        err = C.create_string_buffer(1024)
        check(self.lib.csd_create(C.byref(self.h), device, err, len(err)), err)

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.csd_destroy(self.h)
            self.h = C.c_void_p()
