"""Functional layer: ``shore_fit`` with the keyword interface of the
reference's compiled binding ``_cs_dmri.shore_fit`` (python/src/models.rs:70-198),
running on libcsdshore.so.

Volumes are float32 ``(X, Y, Z, N)`` C-contiguous, masks bool ``(X, Y, Z)``,
gradient tables ``bvals (N,)`` + ``bvecs (N, 3)`` float64.  The result is a
dict with ``coefficients (X, Y, Z, K) float32``, ``warnings``, ``sidecar``
(the coefficient JSON sidecar, src/io/coeffs.rs:28-49), ``alpha_distribution``
and, with ``diagnostics=True``, the maps ``rmse, r2, residual_l2, iterations,
regularization_kind`` plus ``alpha, bic, rss_l2`` where the solver has them.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi

TORTOISE_DEFAULT_GMAX = 80e-3  # src/qspace.rs:262

_REGS = {"l1": _abi.REG_L1, "l2": _abi.REG_L2, "nonneg": _abi.REG_NONNEG}
_PRECISIONS = {"fp64": _abi.PRECISION_FP64, "mixed": _abi.PRECISION_MIXED,
               "mixed-kkt": _abi.PRECISION_MIXED_KKT, "fp64-kkt": _abi.PRECISION_FP64_KKT}
_MODES = {"fixed": _abi.ALPHA_FIXED, "alpha-ratio": _abi.ALPHA_RATIO,
          "path-bic": _abi.ALPHA_PATH_BIC, "l2-anchored": _abi.ALPHA_L2_ANCHORED}


def affine_rotation(affine) -> np.ndarray:
    """Column-normalised 3x3 of a NIfTI affine (src/qspace.rs:296-307)."""
    a = np.asarray(affine, dtype=np.float64)
    if a.shape != (4, 4):
        raise ValueError(f"affine must be 4x4, got {a.shape}")
    r = a[:3, :3].copy()
    norms = np.sqrt((r * r).sum(axis=0))
    scale = np.where(norms > 0, 1.0 / np.where(norms > 0, norms, 1.0), 0.0)
    return r * scale[None, :]


def build_spec(*, radial_order=6, zeta=700.0, regularization="l1", alpha_mode="l2-anchored", alpha=1.0,
               alpha_ratio=1e-3, path_n_alphas=20, path_eps=None, slack=0.05, max_iter=1000, tol=1e-6,
               non_negative=False, lambda_n=1e-8, lambda_l=1e-8, nonneg_max_iter=200, nonneg_tol=1e-9,
               nonneg_epsilon=1e-10, diagnostics=False, allow_single_shell=False,
               precision="fp64") -> _abi.Spec:
    """Flat ShoreFitSpec from the binding's keyword arguments, with the
    binding's string checks (python/src/models.rs:112-144)."""
    if regularization not in _REGS:
        raise ValueError(f"regularization must be l1, l2 or nonneg, got {regularization!r}")
    if regularization == "l1" and alpha_mode not in _MODES:
        raise ValueError(f"alpha_mode must be fixed, alpha-ratio, path-bic or l2-anchored, got {alpha_mode!r}")
    s = _abi.Spec()
    s.radial_order = int(radial_order)
    s.zeta = float(zeta)
    s.regularization = _REGS[regularization]
    s.alpha_mode = _MODES.get(alpha_mode, _abi.ALPHA_L2_ANCHORED)
    s.alpha = float(alpha)
    s.alpha_ratio = float(alpha_ratio)
    s.path_n_alphas = int(path_n_alphas)
    s.path_eps = 0.0 if path_eps is None else float(path_eps)
    if path_eps is not None and not (path_eps > 0):
        s.path_eps = float("nan")  # forces the (0, 1) range error, as the reference
    s.slack = float(slack)
    s.max_iter = int(max_iter)
    s.tol = float(tol)
    s.non_negative = int(bool(non_negative))
    s.lambda_n = float(lambda_n)
    s.lambda_l = float(lambda_l)
    s.nonneg_max_iter = int(nonneg_max_iter)
    s.nonneg_tol = float(nonneg_tol)
    s.nonneg_epsilon = float(nonneg_epsilon)
    s.diagnostics = int(bool(diagnostics))
    s.allow_single_shell = int(bool(allow_single_shell))
    if precision not in _PRECISIONS:
        raise ValueError(f"precision must be fp64, mixed, mixed-kkt or fp64-kkt, got {precision!r}")
    s.precision = _PRECISIONS[precision]
    return s


def build_gtab(bvals, bvecs, b0_threshold=50.0, big_delta=None, small_delta=None):
    bvals = np.ascontiguousarray(np.asarray(bvals, dtype=np.float64).ravel())
    bvecs = np.ascontiguousarray(np.asarray(bvecs, dtype=np.float64))
    if bvecs.ndim != 2 or bvecs.shape[1] != 3:
        raise ValueError(f"bvecs must have shape (N, 3), got {bvecs.shape}")
    if len(bvals) != len(bvecs):
        raise ValueError(f"bvals ({len(bvals)}) and bvecs ({len(bvecs)}) must have the same length")
    g = _abi.Gtab()
    g.bvals = bvals.ctypes.data_as(C.POINTER(C.c_double))
    g.bvecs = bvecs.ctypes.data_as(C.POINTER(C.c_double))
    g.n = len(bvals)
    g.big_delta = math.nan if big_delta is None or small_delta is None else float(big_delta)
    g.small_delta = math.nan if big_delta is None or small_delta is None else float(small_delta)
    g.b0_threshold = float(b0_threshold)
    return g, (bvals, bvecs)  # keep the arrays alive with the struct


def _alpha_strategy_json(kw: dict) -> dict:
    mode = kw.get("alpha_mode", "l2-anchored")
    if mode == "fixed":
        return {"kind": "fixed", "alpha": float(kw.get("alpha", 1.0))}
    if mode == "alpha-ratio":
        return {"kind": "alpha-max-ratio", "ratio": float(kw.get("alpha_ratio", 1e-3))}
    eps = kw.get("path_eps")
    if mode == "path-bic":
        return {"kind": "path-bic", "path": {"n": int(kw.get("path_n_alphas", 20)),
                                             "eps": 1e-3 if eps is None else float(eps)}}
    return {"kind": "path-l2-anchored",
            "path": {"n": int(kw.get("path_n_alphas", 20)), "eps": 1e-4 if eps is None else float(eps)},
            "slack": float(kw.get("slack", 0.05))}


def sidecar(res: _abi.FitResult, kw: dict, bvec_frame: str) -> dict:
    """SidecarMetadata (src/io/coeffs.rs:28-49) as the binding returns it."""
    reg = kw.get("regularization", "l1")
    if reg == "l2":
        solver = {"kind": "tikhonov", "lambda_n": float(kw.get("lambda_n", 1e-8)),
                  "lambda_l": float(kw.get("lambda_l", 1e-8))}
    elif reg == "nonneg":
        solver = {"kind": "shore_icls", "lmax": int(res.lmax), "n_constraint_dirs": int(res.n_constraint_dirs),
                  "max_iter": int(kw.get("nonneg_max_iter", 200)), "tol": float(kw.get("nonneg_tol", 1e-9)),
                  "epsilon": float(kw.get("nonneg_epsilon", 1e-10))}
    else:
        if kw.get("alpha_mode", "l2-anchored") == "fixed":
            chosen = {"scope": "global", "alpha": float(kw.get("alpha", 1.0))}
        elif res.has_alpha_distribution:
            med, p10, p90 = (float(v) for v in res.alpha_distribution)
            chosen = {"scope": "per-voxel", "median": med, "p10": p10, "p90": p90}
        else:
            chosen = {"scope": "global", "alpha": float(res.representative_alpha)}
        solver = {"kind": "fista", "alpha_strategy": _alpha_strategy_json(kw), "chosen_alpha": chosen,
                  "non_negative": bool(kw.get("non_negative", False)), "max_iter": int(kw.get("max_iter", 1000)),
                  "tol": float(kw.get("tol", 1e-6))}
    return {
        "basis": {"name": "shore", "radial_order": int(kw.get("radial_order", 6)),
                  "zeta": float(kw.get("zeta", 700.0))},
        "big_delta_seconds": float(res.big_delta_seconds),
        "small_delta_seconds": float(res.small_delta_seconds),
        "tau_seconds": float(res.tau_seconds),
        "delta_source": "user_supplied" if res.delta_source == 0 else "estimated_tortoise",
        "gmax_tesla_per_meter": TORTOISE_DEFAULT_GMAX,
        "solver": solver,
        "n_coefficients": int(res.n_coeffs),
        "bvec_frame": bvec_frame,
        "dwi_shells": [float(res.dwi_shells[i]) for i in range(res.n_shells)],
    }


_SPEC_KEYS = ("radial_order", "zeta", "regularization", "alpha_mode", "alpha", "alpha_ratio", "path_n_alphas",
              "path_eps", "slack", "max_iter", "tol", "non_negative", "lambda_n", "lambda_l", "nonneg_max_iter",
              "nonneg_tol", "nonneg_epsilon", "diagnostics", "allow_single_shell", "precision")


def shore_fit(data, bvals, bvecs, mask, *, big_delta=None, small_delta=None, b0_threshold=50.0,
              bvec_frame="image-axis", radial_order=6, zeta=700.0, regularization="l1",
              alpha_mode="l2-anchored", alpha=1.0, alpha_ratio=1e-3, path_n_alphas=20, path_eps=None,
              slack=0.05, max_iter=1000, tol=1e-6, non_negative=False, lambda_n=1e-8, lambda_l=1e-8,
              nonneg_max_iter=200, nonneg_tol=1e-9, nonneg_epsilon=1e-10, diagnostics=False,
              allow_single_shell=False, n_threads=None, device: int = 0, return_coef64: bool = False,
              coefficients_out=None, precision: str = "fp64") -> dict:
    """SHORE fit of every masked voxel on the GPU (``_cs_dmri.shore_fit``).

    ``n_threads`` is accepted for signature compatibility and ignored: the fit
    runs on CUDA device ``device``.  ``return_coef64=True`` adds ``coef64``
    (V, K) float64 and ``converged`` (V,) for the masked voxels in x-y-z order.
    ``coefficients_out`` may supply the (X, Y, Z, K) float32 C-contiguous output
    array (for example in page-locked memory, which makes the copy back
    faster); every element is overwritten.  A page-locked ``data`` volume is
    read in place, masked voxels only.  ``precision="mixed"`` (radial order 6)
    runs the L1 iterations with int8 digit-slice tensor-core Gram products and
    FP64 state; the default ``"fp64"`` is the reference arithmetic.
    ``"mixed-kkt"`` and ``"fp64-kkt"`` (fixed alpha or alpha ratio, radial
    order <= 6) return the KKT-certified LASSO optimum instead of the
    reference's early-stopped iterate: support identification by TF32
    tensor-core (or FP64) FISTA iterations, then an FP64 active-set polish;
    ``converged`` is the certificate.
    """
    if bvec_frame not in ("image-axis", "world-ras"):
        raise ValueError(f"bvec_frame must be 'image-axis' or 'world-ras', got {bvec_frame!r}")
    kw = dict(radial_order=radial_order, zeta=zeta, regularization=regularization, alpha_mode=alpha_mode,
              alpha=alpha, alpha_ratio=alpha_ratio, path_n_alphas=path_n_alphas, path_eps=path_eps, slack=slack,
              max_iter=max_iter, tol=tol, non_negative=non_negative, lambda_n=lambda_n, lambda_l=lambda_l,
              nonneg_max_iter=nonneg_max_iter, nonneg_tol=nonneg_tol, nonneg_epsilon=nonneg_epsilon,
              diagnostics=diagnostics, allow_single_shell=allow_single_shell, precision=precision)
    spec = build_spec(**kw)
    data = np.asarray(data)
    if data.ndim != 4:
        raise ValueError(f"data must be 4-D (X, Y, Z, N), got shape {data.shape}")
    data = np.ascontiguousarray(data, dtype=np.float32)
    g, keep = build_gtab(bvals, bvecs, b0_threshold, big_delta, small_delta)
    if data.shape[3] != g.n:
        raise ValueError(f"data has {data.shape[3]} volumes but the gradient table has {g.n}")
    m = np.asarray(mask)
    if m.shape != data.shape[:3]:
        raise ValueError(f"mask shape {m.shape} does not match data spatial shape {data.shape[:3]}")
    m8 = np.ascontiguousarray(m.astype(bool).view(np.uint8) if m.dtype == bool else (m != 0).astype(np.uint8))
    X, Y, Z = data.shape[:3]
    K = _abi.load().csd_shore_n_coeffs(int(radial_order))
    if coefficients_out is not None:
        coeffs = coefficients_out
        if (coeffs.shape != (X, Y, Z, K) or coeffs.dtype != np.float32 or not coeffs.flags.c_contiguous
                or not coeffs.flags.writeable):
            raise ValueError(f"coefficients_out must be a writable C-contiguous float32 array of shape {(X, Y, Z, K)}")
    else:
        coeffs = np.empty((X, Y, Z, max(K, 0)), dtype=np.float32)  # every element is written
    res = _abi.FitResult()
    res.coefficients = coeffs.ctypes.data
    maps = {}
    if diagnostics:
        maps["r2"] = np.zeros((X, Y, Z), np.float32)
        maps["residual_l2"] = np.zeros((X, Y, Z), np.float32)
        maps["iterations"] = np.zeros((X, Y, Z), np.uint32)
        maps["regularization_kind"] = np.zeros((X, Y, Z), np.uint8)
        if regularization == "l1":
            maps["alpha"] = np.zeros((X, Y, Z), np.float32)
            maps["bic"] = np.zeros((X, Y, Z), np.float32)
            if alpha_mode == "l2-anchored":
                maps["rss_l2"] = np.zeros((X, Y, Z), np.float32)
        for k, a in maps.items():
            setattr(res, k, a.ctypes.data)
    nmask = int(m8.sum())
    c64 = conv = None
    if return_coef64:
        c64 = np.zeros((nmask, K), np.float64)
        conv = np.zeros(nmask, np.uint8)
        res.coef64 = c64.ctypes.data
        res.converged = conv.ctypes.data
    lib = _abi.load()
    h = _abi.handle(device)
    err = C.create_string_buffer(4096)
    code = lib.csd_shore_fit_volume(h, data.ctypes.data, m8.ctypes.data, X, Y, Z, C.byref(g), C.byref(spec),
                                    C.byref(res), err, len(err))
    del keep
    _abi.check(code, err)
    out = {"coefficients": coeffs,
           "warnings": [w for w in res.warnings.decode("utf-8", "replace").split("\n") if w],
           "sidecar": sidecar(res, kw, bvec_frame),
           "alpha_distribution": tuple(float(v) for v in res.alpha_distribution)
           if res.has_alpha_distribution else None}
    if diagnostics:
        n = len(np.asarray(bvals).ravel())
        out["rmse"] = (maps["residual_l2"] / np.float32(math.sqrt(n))).astype(np.float32)
        out.update(maps)
    if return_coef64:
        out["coef64"] = c64
        out["converged"] = conv.astype(bool)
    out["total_iterations"] = int(res.total_iterations)
    out["n_voxels"] = int(res.n_voxels)
    return out


def shore_fit_device(data, mask, bvals, bvecs, *, coefficients=None, stream=None, device: int = 0,
                     big_delta=None, small_delta=None, b0_threshold=50.0, **kw):
    """Fit with ``data`` / ``mask`` already resident on the GPU (torch CUDA
    tensors: float32 (X, Y, Z, N) and bool/uint8 (X, Y, Z)).  Writes into
    ``coefficients`` (float32 (X, Y, Z, K) CUDA tensor; allocated if None) and
    returns it.  Diagnostics maps are not produced by this entry point."""
    import torch

    if not (data.is_cuda and mask.is_cuda):
        raise ValueError("shore_fit_device needs CUDA tensors")
    if data.dtype != torch.float32 or not data.is_contiguous() or data.dim() != 4:
        raise ValueError("data must be a contiguous float32 (X, Y, Z, N) CUDA tensor")
    m8 = mask.to(torch.uint8).contiguous() if mask.dtype != torch.uint8 else mask.contiguous()
    kw = {k: v for k, v in kw.items() if k in _SPEC_KEYS}
    kw["diagnostics"] = False
    spec = build_spec(**kw)
    g, keep = build_gtab(bvals, bvecs, b0_threshold, big_delta, small_delta)
    X, Y, Z, N = data.shape
    if N != g.n:
        raise ValueError(f"data has {N} volumes but the gradient table has {g.n}")
    lib = _abi.load()
    K = lib.csd_shore_n_coeffs(int(kw.get("radial_order", 6)))
    if coefficients is None:
        coefficients = torch.empty((X, Y, Z, K), dtype=torch.float32, device=data.device)
    res = _abi.FitResult()
    res.coefficients = coefficients.data_ptr()
    err = C.create_string_buffer(4096)
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream(data.device).cuda_stream
    code = lib.csd_shore_fit_volume_device(_abi.handle(device), data.data_ptr(), m8.data_ptr(), X, Y, Z,
                                           C.byref(g), C.byref(spec), C.byref(res), C.c_void_p(s), err, len(err))
    del keep
    _abi.check(code, err)
    return coefficients, res


def design_matrix(bvals, bvecs, radial_order=6, zeta=700.0, *, big_delta=None, small_delta=None,
                  b0_threshold=50.0, device: int = 0) -> np.ndarray:
    """SHORE design matrix (N, K) built on the GPU (ShoreBasis::design_matrix)."""
    g, keep = build_gtab(bvals, bvecs, b0_threshold, big_delta, small_delta)
    lib = _abi.load()
    K = lib.csd_shore_n_coeffs(int(radial_order))
    out = np.zeros((g.n, K), np.float64)
    err = C.create_string_buffer(1024)
    code = lib.csd_shore_design_matrix(_abi.handle(device), C.byref(g), int(radial_order), float(zeta),
                                       out.ctypes.data, err, len(err))
    del keep
    _abi.check(code, err)
    return out


# ------------------------------------------------------------ post-fit maps

def _coefficient_volume(coefficients, radial_order):
    c = np.asarray(coefficients)
    if c.ndim != 4:
        raise ValueError(f"coefficients must be 4-D (X, Y, Z, K), got shape {c.shape}")
    K = _abi.load().csd_shore_n_coeffs(int(radial_order))
    if c.shape[3] != K:  # python/src/models.rs:216-222
        raise ValueError(f"coefficients have {c.shape[3]} channels but a radial-order-{radial_order} SHORE basis "
                         f"has {K}")
    return np.ascontiguousarray(c, dtype=np.float32)


def shore_predict(coefficients, radial_order, zeta, bvals, bvecs, *, big_delta=None, small_delta=None,
                  n_threads=None, device: int = 0):
    """Signal of a coefficient volume on a new gradient table, (X, Y, Z, N)
    float32 (``_cs_dmri.shore_predict``, python/src/models.rs:252-278, over
    synthesize_volume, src/synth.rs:15-84).  ``n_threads`` is accepted and
    ignored (the work runs on CUDA device ``device``)."""
    c = _coefficient_volume(coefficients, radial_order)
    g, keep = build_gtab(bvals, bvecs, 50.0, big_delta, small_delta)
    X, Y, Z, _ = c.shape
    out = np.empty((X, Y, Z, g.n), np.float32)
    err = C.create_string_buffer(4096)
    code = _abi.load().csd_shore_predict(_abi.handle(device), c.ctypes.data, X, Y, Z, int(radial_order),
                                         float(zeta), C.byref(g), out.ctypes.data, err, len(err))
    del keep
    _abi.check(code, err)
    return out


def shore_odf_sh(coefficients, radial_order, zeta, lmax, mask=None, *, n_threads=None, device: int = 0):
    """Tournier-ordered ODF SH coefficients, (X, Y, Z, (lmax+1)(lmax+2)/2)
    float32, zeros outside ``mask`` (``_cs_dmri.shore_odf_sh``,
    python/src/models.rs:201-250; projection of src/odf.rs:79-102)."""
    if lmax % 2 != 0 or lmax > radial_order:
        raise ValueError(f"lmax must be even and \u2264 radial_order ({radial_order}), got {lmax}")
    c = _coefficient_volume(coefficients, radial_order)
    X, Y, Z, _ = c.shape
    m8 = None
    if mask is not None:
        m = np.asarray(mask)
        if m.shape != (X, Y, Z):
            raise ValueError("mask does not match the coefficient grid")
        m8 = np.ascontiguousarray(m.astype(bool)).view(np.uint8)
    out = np.empty((X, Y, Z, (lmax + 1) * (lmax + 2) // 2), np.float32)
    err = C.create_string_buffer(4096)
    code = _abi.load().csd_shore_odf_sh(_abi.handle(device), c.ctypes.data, X, Y, Z, int(radial_order), float(zeta),
                                        int(lmax), None if m8 is None else m8.ctypes.data, out.ctypes.data, err,
                                        len(err))
    _abi.check(code, err)
    return out


def shore_odf_peaks(coefficients, radial_order, zeta, mask=None, *, sphere_frequency=6, npeaks=5,
                    relative_peak_threshold=0.5, min_separation_angle=25.0, device: int = 0) -> dict:
    """GFA and ODF peaks of a coefficient volume (the quantities the
    reference's SHORE ODX export computes, src/io/odx_out.rs:1008-1090, with
    its defaults npeaks 5, relative threshold 0.5, separation 25 degrees).

    The ODF is sampled on the hemisphere of a class I geodesic sphere of
    ``sphere_frequency`` (181 directions at 6), amplitudes clipped at 0.
    Returns ``gfa`` (X, Y, Z), ``peak_dirs`` (X, Y, Z, npeaks, 3) unit
    vectors in the fit frame, ``peak_values`` (X, Y, Z, npeaks) ODF
    amplitudes and ``peak_qa`` (X, Y, Z, npeaks) amplitudes above the voxel's
    smallest sampled amplitude; slots past the peaks found are zero, as is
    everything outside ``mask``."""
    c = _coefficient_volume(coefficients, radial_order)
    X, Y, Z, _ = c.shape
    m8 = None
    if mask is not None:
        m = np.asarray(mask)
        if m.shape != (X, Y, Z):
            raise ValueError("mask does not match the coefficient grid")
        m8 = np.ascontiguousarray(m.astype(bool)).view(np.uint8)
    npeaks = int(npeaks)
    out = {"gfa": np.empty((X, Y, Z), np.float32), "peak_dirs": np.empty((X, Y, Z, max(npeaks, 0), 3), np.float32),
           "peak_values": np.empty((X, Y, Z, max(npeaks, 0)), np.float32),
           "peak_qa": np.empty((X, Y, Z, max(npeaks, 0)), np.float32)}
    err = C.create_string_buffer(4096)
    code = _abi.load().csd_shore_odf_peaks(
        _abi.handle(device), c.ctypes.data, X, Y, Z, int(radial_order), float(zeta),
        None if m8 is None else m8.ctypes.data, int(sphere_frequency), npeaks, float(relative_peak_threshold),
        float(min_separation_angle), out["gfa"].ctypes.data, out["peak_dirs"].ctypes.data,
        out["peak_values"].ctypes.data, out["peak_qa"].ctypes.data, err, len(err))
    _abi.check(code, err)
    return out


_MICRO = ("rtop", "rtap", "rtpp", "msd", "qiv", "ng")


def shore_microstructure(coefficients, radial_order, zeta, mask, directions=None, *, units="um",
                         outlier_factor=10.0, n_threads=None, device: int = 0):
    """RTOP, RTAP, RTPP, MSD, QIV and NG maps (zero outside ``mask``; NaN
    where a value is rejected as a fit failure, ``outlier_factor`` x its p99;
    ``outlier_factor=None`` keeps every value).  RTAP / RTPP need
    ``directions`` (X, Y, Z, 3) in the coefficients' frame and are NaN where
    a direction is zero or missing (``_cs_dmri.shore_microstructure``,
    python/src/models.rs:283-341; src/io/microstructure.rs:155-298)."""
    if units not in ("um", "mm"):
        raise ValueError(f"units must be 'um' or 'mm', got {units!r}")
    c = _coefficient_volume(coefficients, radial_order)
    X, Y, Z, _ = c.shape
    m = np.asarray(mask)
    if m.shape != (X, Y, Z):
        raise ValueError("mask does not match the coefficient grid")
    m8 = np.ascontiguousarray(m.astype(bool)).view(np.uint8)
    d = None
    if directions is not None:
        d = np.ascontiguousarray(np.asarray(directions, dtype=np.float32))
        if d.shape != (X, Y, Z, 3):
            raise ValueError(f"directions must have shape {(X, Y, Z, 3)}, got {d.shape}")
    maps = {k: np.empty((X, Y, Z), np.float32) for k in _MICRO}
    err = C.create_string_buffer(4096)
    reject = outlier_factor is not None
    code = _abi.load().csd_shore_microstructure(
        _abi.handle(device), c.ctypes.data, X, Y, Z, int(radial_order), float(zeta), m8.ctypes.data,
        None if d is None else d.ctypes.data, 0 if units == "um" else 1, int(reject),
        float(outlier_factor) if reject else 0.0, *(maps[k].ctypes.data for k in _MICRO), err, len(err))
    _abi.check(code, err)
    return maps
