"""ctypes wrapper of the CPU FP64 oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  It shares the argument structs
of the product's C ABI (include/csd_shore.h) so both are driven identically.
"""

from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_lib = None


def build(force: bool = False) -> Path:
    srcs = [HERE / "shore_oracle.cpp", HERE / "shore_oracle.h", HERE.parent / "include" / "csd_shore.h"]
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True,
                       capture_output=True, text=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        d, i32, p = C.c_double, C.c_int32, C.c_void_p
        sig = {
            "oracle_factorial": (d, [C.c_uint32]),
            "oracle_gamma": (d, [d]),
            "oracle_assoc_legendre": (d, [C.c_uint32, C.c_uint32, d]),
            "oracle_gen_laguerre": (d, [C.c_uint32, d, d]),
            "oracle_hyp2f1": (d, [d, d, d, d]),
            "oracle_qvals": (C.c_int, [p, p, p, p, p]),
            "oracle_shells": (C.c_int, [p, i32, d, d, p, p]),
            "oracle_tortoise_deltas": (None, [p, i32, d, p, p]),
            "oracle_n_coeffs": (C.c_int, [i32]),
            "oracle_shore_indices": (None, [i32, p, p, p]),
            "oracle_kappa": (d, [d, C.c_uint32, C.c_uint32]),
            "oracle_shore_radial": (d, [C.c_uint32, C.c_uint32, d, d]),
            "oracle_brainsuite_sh_block": (None, [C.c_uint32, d, d, p]),
            "oracle_design_matrix": (C.c_int, [p, i32, d, p]),
            "oracle_regularization": (None, [i32, p, p]),
            "oracle_radial_factor": (d, [C.c_uint32, C.c_uint32, d]),
            "oracle_brainsuite_to_tournier": (None, [C.c_uint32, i32, p, p]),
            "oracle_shore_to_tournier": (C.c_int, [i32, d, i32, p]),
            "oracle_odf8_hemisphere": (C.c_int, [p]),
            "oracle_sh2amp_cart": (None, [p, i32, i32, p]),
            "oracle_sigma_max": (d, [p, i32, i32]),
            "oracle_fista_fit": (C.c_int, [p, i32, i32, p, d, i32, d, i32, p, p, p, p, p]),
            "oracle_tikhonov_fit": (C.c_int, [p, i32, i32, p, p, d, d, p, p, p]),
            "oracle_icls_solve": (C.c_int, [p, i32, i32, p, i32, p, i32, d, d, p, p, p, p, p]),
            "oracle_alpha_max": (d, [p, i32, i32, p]),
            "oracle_log_path": (C.c_int, [d, i32, d, p]),
            "oracle_bic": (d, [i32, d, i32]),
            "oracle_shore_fit_volume": (C.c_int, [p, p, C.c_int64, C.c_int64, C.c_int64, p, p, p, i32, p,
                                                  C.c_size_t]),
            "oracle_shore_predict": (C.c_int, [p, C.c_int64, C.c_int64, C.c_int64, i32, d, p, p, p, C.c_size_t]),
            "oracle_shore_odf_sh": (C.c_int, [p, C.c_int64, C.c_int64, C.c_int64, i32, d, i32, p, p, p,
                                              C.c_size_t]),
            "oracle_shore_microstructure": (C.c_int, [p, C.c_int64, C.c_int64, C.c_int64, i32, d, p, p, i32, i32,
                                                      C.c_float, p, p, p, p, p, p, p, C.c_size_t]),
            "oracle_microstructure_voxel": (None, [p, i32, d, p, p]),
            "oracle_micro_alpha_factor": (d, [C.c_uint32, C.c_uint32, d]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


# ------------------------------------------------------------ math / basis

def factorial(n): return lib().oracle_factorial(n)
def gamma(x): return lib().oracle_gamma(x)
def assoc_legendre(l, m, x): return lib().oracle_assoc_legendre(l, m, x)
def gen_laguerre(n, a, x): return lib().oracle_gen_laguerre(n, a, x)
def hyp2f1(a, b, c, z): return lib().oracle_hyp2f1(a, b, c, z)
def kappa(zeta, n, l): return lib().oracle_kappa(zeta, n, l)
def shore_radial(n, l, q, zeta): return lib().oracle_shore_radial(n, l, q, zeta)
def radial_factor(n, l, zeta): return lib().oracle_radial_factor(n, l, zeta)
def n_coeffs(order): return lib().oracle_n_coeffs(order)
def bic(n, rss, k): return lib().oracle_bic(n, rss, k)


def _gtab(bvals, bvecs, big_delta=None, small_delta=None, b0_threshold=50.0):
    from cs_dmri_b200._core import build_gtab
    return build_gtab(bvals, bvecs, b0_threshold, big_delta, small_delta)


def shore_indices(order):
    k = n_coeffs(order)
    n, l, m = (np.zeros(k, np.int32) for _ in range(3))
    lib().oracle_shore_indices(order, _p(n), _p(l), _p(m))
    return np.stack([n, l, m], 1)


def brainsuite_sh_block(l, theta, phi):
    out = np.zeros(2 * l + 1)
    lib().oracle_brainsuite_sh_block(l, theta, phi, _p(out))
    return out


def qvals(bvals, bvecs, big_delta=None, small_delta=None, b0_threshold=50.0):
    g, keep = _gtab(bvals, bvecs, big_delta, small_delta, b0_threshold)
    q = np.zeros(g.n)
    big, small, src = C.c_double(), C.c_double(), C.c_int32()
    lib().oracle_qvals(C.addressof(g), _p(q), C.addressof(big), C.addressof(small), C.addressof(src))
    return q, big.value, small.value, src.value


def shells(bvals, b0_threshold=50.0, tolerance=50.0):
    b = _f64(bvals)
    sb = np.zeros(len(b) + 1)
    of = np.zeros(len(b), np.int32)
    n = lib().oracle_shells(_p(b), len(b), b0_threshold, tolerance, _p(sb), _p(of))
    return sb[:n], of


def tortoise_deltas(bvals, gmax=80e-3):
    b = _f64(bvals)
    big, small = C.c_double(), C.c_double()
    lib().oracle_tortoise_deltas(_p(b), len(b), gmax, C.addressof(big), C.addressof(small))
    return big.value, small.value


def design_matrix(bvals, bvecs, order=6, zeta=700.0, big_delta=None, small_delta=None, b0_threshold=50.0):
    g, keep = _gtab(bvals, bvecs, big_delta, small_delta, b0_threshold)
    out = np.zeros((g.n, n_coeffs(order)))
    lib().oracle_design_matrix(C.addressof(g), order, zeta, _p(out))
    return out


def regularization(order):
    k = n_coeffs(order)
    a, b = np.zeros(k), np.zeros(k)
    lib().oracle_regularization(order, _p(a), _p(b))
    return a, b


def brainsuite_to_tournier(l, k):
    idx, sign = C.c_int32(), C.c_double()
    lib().oracle_brainsuite_to_tournier(l, k, C.addressof(idx), C.addressof(sign))
    return idx.value, sign.value


def shore_to_tournier(order, zeta, lmax):
    nsh = (lmax + 1) * (lmax + 2) // 2
    out = np.zeros((nsh, n_coeffs(order)))
    lib().oracle_shore_to_tournier(order, zeta, lmax, _p(out))
    return out


def odf8_hemisphere():
    out = np.zeros((700, 3))
    n = lib().oracle_odf8_hemisphere(_p(out))
    return out[:n].copy()


def sh2amp_cart(dirs, lmax):
    d = _f64(dirs)
    out = np.zeros((len(d), (lmax + 1) * (lmax + 2) // 2))
    lib().oracle_sh2amp_cart(_p(d), len(d), lmax, _p(out))
    return out


# ----------------------------------------------------------------- solvers

def sigma_max(M):
    M = _f64(M)
    return lib().oracle_sigma_max(_p(M), M.shape[0], M.shape[1])


def fista_fit(M, s, alpha, max_iter=1000, tol=1e-6, non_negative=False, warm=None):
    M, s = _f64(M), _f64(s)
    m, n = M.shape
    c = np.zeros(n)
    it, conv, res = C.c_int32(), C.c_int32(), C.c_double()
    w = None if warm is None else _f64(warm)
    lib().oracle_fista_fit(_p(M), m, n, _p(s), alpha, max_iter, tol, int(non_negative),
                           None if w is None else _p(w), _p(c), C.addressof(it), C.addressof(conv),
                           C.addressof(res))
    return c, it.value, bool(conv.value), res.value


def tikhonov_fit(M, s, n_diag, l_diag, lambda_n, lambda_l):
    M, s, nd, ld = _f64(M), _f64(s), _f64(n_diag), _f64(l_diag)
    m, n = M.shape
    c = np.zeros(n)
    res = C.c_double()
    code = lib().oracle_tikhonov_fit(_p(M), m, n, _p(nd), _p(ld), lambda_n, lambda_l, _p(s), _p(c),
                                     C.addressof(res))
    if code != 0:
        raise ValueError("normal-equations matrix should be PD")
    return c, res.value


def icls_solve(H, Cm, b, max_iter=200, tol=1e-10, epsilon=1e-10):
    H, Cm, b = _f64(H), _f64(np.atleast_2d(Cm)), _f64(b)
    m, n = H.shape
    x = np.zeros(n)
    it, act, conv, inf = (C.c_int32() for _ in range(4))
    code = lib().oracle_icls_solve(_p(H), m, n, _p(Cm), Cm.shape[0], _p(b), max_iter, tol, epsilon, _p(x),
                                   C.addressof(it), C.addressof(act), C.addressof(conv), C.addressof(inf))
    if code != 0:
        raise ValueError("H^T H + eps I must be positive definite")
    return x, dict(iterations=it.value, final_active=act.value, converged=bool(conv.value),
                   infeasible=bool(inf.value))


def alpha_max(M, s):
    M, s = _f64(M), _f64(s)
    return lib().oracle_alpha_max(_p(M), M.shape[0], M.shape[1], _p(s))


def log_path(amax, n, eps):
    out = np.zeros(n)
    if lib().oracle_log_path(amax, n, eps, _p(out)) != 0:
        raise ValueError("log_path needs n >= 2, alpha_max > 0, 0 < eps < 1")
    return out


# ------------------------------------------------------------------ volume

def shore_fit(data, bvals, bvecs, mask, *, n_threads: int = 0, big_delta=None, small_delta=None,
              b0_threshold=50.0, bvec_frame="image-axis", return_coef64=True, **kw) -> dict:
    """Whole-volume oracle fit with the keyword interface of shore_fit."""
    from cs_dmri_b200 import _abi
    from cs_dmri_b200._core import build_spec, sidecar

    spec = build_spec(**kw)
    data = np.ascontiguousarray(data, dtype=np.float32)
    g, keep = _gtab(bvals, bvecs, big_delta, small_delta, b0_threshold)
    m8 = np.ascontiguousarray(np.asarray(mask).astype(bool)).view(np.uint8)
    X, Y, Z = data.shape[:3]
    K = n_coeffs(spec.radial_order) if spec.radial_order >= 0 else 0
    coeffs = np.zeros((X, Y, Z, K), np.float32)
    res = _abi.FitResult()
    res.coefficients = coeffs.ctypes.data
    diag = bool(kw.get("diagnostics", False))
    maps = {}
    if diag:
        maps = {"r2": np.zeros((X, Y, Z), np.float32), "residual_l2": np.zeros((X, Y, Z), np.float32),
                "iterations": np.zeros((X, Y, Z), np.uint32),
                "regularization_kind": np.zeros((X, Y, Z), np.uint8)}
        if kw.get("regularization", "l1") == "l1":
            maps["alpha"] = np.zeros((X, Y, Z), np.float32)
            maps["bic"] = np.zeros((X, Y, Z), np.float32)
            if kw.get("alpha_mode", "l2-anchored") == "l2-anchored":
                maps["rss_l2"] = np.zeros((X, Y, Z), np.float32)
        for k, a in maps.items():
            setattr(res, k, a.ctypes.data)
    nmask = int(m8.sum())
    c64 = np.zeros((nmask, max(K, 0)))
    conv = np.zeros(nmask, np.uint8)
    if return_coef64:
        res.coef64 = c64.ctypes.data
        res.converged = conv.ctypes.data
    err = C.create_string_buffer(4096)
    code = lib().oracle_shore_fit_volume(_p(data), _p(m8), X, Y, Z, C.addressof(g), C.addressof(spec),
                                         C.addressof(res), int(n_threads), err, len(err))
    if code != 0:
        raise ValueError(err.value.decode())
    kwf = dict(kw)
    out = {"coefficients": coeffs,
           "warnings": [w for w in res.warnings.decode().split("\n") if w],
           "sidecar": sidecar(res, kwf, bvec_frame),
           "alpha_distribution": tuple(res.alpha_distribution) if res.has_alpha_distribution else None,
           "total_iterations": int(res.total_iterations), "n_voxels": int(res.n_voxels)}
    if diag:
        out["rmse"] = (maps["residual_l2"] / np.float32(math.sqrt(len(np.ravel(bvals))))).astype(np.float32)
        out.update(maps)
    if return_coef64:
        out["coef64"] = c64
        out["converged"] = conv.astype(bool)
    return out


def cpu_count() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


# ------------------------------------------------ synth / odf / scalars

def _coeff_volume(coefficients, radial_order):
    c = np.ascontiguousarray(np.asarray(coefficients, dtype=np.float32))
    if c.ndim != 4 or c.shape[3] != n_coeffs(radial_order):
        raise ValueError(f"coefficients have {c.shape[-1]} channels but a radial-order-{radial_order} SHORE "
                         f"basis has {n_coeffs(radial_order)}")
    return c


def shore_predict(coefficients, radial_order, zeta, bvals, bvecs, *, big_delta=None, small_delta=None):
    """synthesize_volume (synth.rs:15-84) through the binding's gradient table."""
    c = _coeff_volume(coefficients, radial_order)
    g, keep = _gtab(bvals, bvecs, big_delta, small_delta, 50.0)
    X, Y, Z, _ = c.shape
    out = np.zeros((X, Y, Z, g.n), np.float32)
    err = C.create_string_buffer(1024)
    if lib().oracle_shore_predict(_p(c), X, Y, Z, radial_order, zeta, C.addressof(g), _p(out), err, len(err)):
        raise ValueError(err.value.decode())
    return out


def shore_odf_sh(coefficients, radial_order, zeta, lmax, mask=None):
    """shore_odf_sh (python/src/models.rs:201-250)."""
    c = _coeff_volume(coefficients, radial_order)
    X, Y, Z, _ = c.shape
    nsh = (lmax + 1) * (lmax + 2) // 2
    out = np.zeros((X, Y, Z, nsh), np.float32)
    m = None if mask is None else np.ascontiguousarray(np.asarray(mask, bool)).view(np.uint8)
    err = C.create_string_buffer(1024)
    if lib().oracle_shore_odf_sh(_p(c), X, Y, Z, radial_order, zeta, lmax, None if m is None else _p(m), _p(out),
                                 err, len(err)):
        raise ValueError(err.value.decode())
    return out


def shore_microstructure(coefficients, radial_order, zeta, mask, directions=None, *, units="um",
                         outlier_factor=10.0):
    """shore_microstructure (python/src/models.rs:283-341)."""
    c = _coeff_volume(coefficients, radial_order)
    X, Y, Z, _ = c.shape
    m = np.ascontiguousarray(np.asarray(mask, bool)).view(np.uint8)
    d = None if directions is None else np.ascontiguousarray(np.asarray(directions, np.float32))
    maps = {k: np.zeros((X, Y, Z), np.float32) for k in ("rtop", "rtap", "rtpp", "msd", "qiv", "ng")}
    err = C.create_string_buffer(1024)
    reject = outlier_factor is not None
    code = lib().oracle_shore_microstructure(
        _p(c), X, Y, Z, radial_order, zeta, _p(m), None if d is None else _p(d), 1 if units == "mm" else 0,
        int(reject), float(outlier_factor if reject else 0.0), *(_p(maps[k]) for k in maps), err, len(err))
    if code:
        raise ValueError(err.value.decode())
    return maps


def microstructure_voxel(coefs, radial_order, zeta, direction=None):
    """{rtop, msd, qiv, ng, rtap, rtpp} of one FP64 coefficient vector."""
    c = _f64(coefs)
    out = np.zeros(6)
    dp = None if direction is None else _f64(direction)
    lib().oracle_microstructure_voxel(_p(c), radial_order, zeta, None if dp is None else _p(dp), _p(out))
    return dict(zip(("rtop", "msd", "qiv", "ng", "rtap", "rtpp"), out))


def micro_alpha_factor(n, l, zeta):
    return lib().oracle_micro_alpha_factor(n, l, zeta)


# ------------------------------------------------------ derivatives of the fit
# The reference computes no derivatives.  These restate, in plain FP64 numpy,
# the implicit-function derivatives of the solution maps its solvers define:
# the LASSO fit of src/solver/fista.rs:70-143, which minimises
# (1/(2n)) ||M c - s||^2 + alpha ||c||_1 (c >= 0 when non_negative), and the
# Tikhonov fit of src/solver/tikhonov.rs:26-76, H c = M^T s with
# H = M^T M + lambda_N N + lambda_L L (src/basis/shore.rs:180-195).

def l1_adjoint(M, c, gc):
    """Adjoint of the LASSO solution map at ``c`` for the upstream gradient
    ``gc``: on the support S the optimality condition
    G_SS c_S = M_S^T s - n alpha sign(c_S) gives w_S = G_SS^-1 gc_S,
    grad_s = M w and grad_alpha = -n sign(c_S) . w_S.  Returns
    (grad_s, grad_alpha, w)."""
    M, c, gc = _f64(M), _f64(c), _f64(gc)
    n = M.shape[0]
    S = np.flatnonzero(c != 0.0)
    w = np.zeros_like(c)
    if S.size:
        MS = M[:, S]
        w[S] = np.linalg.solve(MS.T @ MS, gc[S])
    return M @ w, float(-n * (np.sign(c[S]) @ w[S])), w


def l2_adjoint(M, c, gc, n_diag, l_diag, lambda_n, lambda_l):
    """Adjoint of the Tikhonov solution map: w = H^-1 gc, grad_s = M w,
    grad_lambda_N = -w . (N c), grad_lambda_L = -w . (L c).  Returns
    (grad_s, (grad_lambda_N, grad_lambda_L), w)."""
    M, c, gc, nd, ld = _f64(M), _f64(c), _f64(gc), _f64(n_diag), _f64(l_diag)
    H = M.T @ M + np.diag(lambda_n * nd + lambda_l * ld)
    w = np.linalg.solve(H, gc)
    return M @ w, (float(-(w @ (nd * c))), float(-(w @ (ld * c)))), w


def lasso_polish(M, s, alpha, c0, non_negative=False, margin=1e-6):
    """The exact LASSO minimiser from an approximate one: solve the optimality
    condition on the support and signs of ``c0``, then certify it - the signs
    hold on the support and |M_j^T r| / n < alpha (1 - margin) off it
    (M_j^T r / n > -alpha (1 - margin) with non_negative), r = s - M c.
    Returns (c, certified)."""
    M, s, c0 = _f64(M), _f64(s), _f64(c0)
    n = M.shape[0]
    S = np.flatnonzero(c0 != 0.0)
    sg = np.sign(c0[S])
    c = np.zeros_like(c0)
    if S.size:
        MS = M[:, S]
        c[S] = np.linalg.solve(MS.T @ MS, MS.T @ s - n * alpha * sg)
    corr = M.T @ (s - M @ c) / n
    off = np.setdiff1d(np.arange(c0.size), S)
    ok = bool(np.all(np.sign(c[S]) == sg))
    if non_negative:
        ok = ok and bool(np.all(sg > 0)) and bool(np.all(corr[off] < alpha * (1.0 - margin)))
    else:
        ok = ok and bool(np.all(np.abs(corr[off]) < alpha * (1.0 - margin)))
    return c, ok


def lasso_optimum_rows(M, S, alpha, C0, non_negative=False, margin=0.0):
    """Row-wise lasso_polish: the exact minimiser of every voxel (rows of the
    signals S) on the support and signs of its approximate solution C0, and
    whether its KKT conditions certify it.  alpha may be one value per row.
    Returns (C, certified)."""
    S, C0 = _f64(S), _f64(C0)
    a = np.broadcast_to(np.asarray(alpha, np.float64), (S.shape[0],))
    out = np.zeros_like(C0)
    ok = np.zeros(S.shape[0], bool)
    for v in range(S.shape[0]):
        out[v], ok[v] = lasso_polish(M, S[v], float(a[v]), C0[v], non_negative=non_negative, margin=margin)
    return out, ok


def geodesic_sphere(frequency, hemisphere=False):
    """Class I geodesic sphere: each icosahedron face cut into f^2 triangles on
    a flat barycentric grid, the points projected on the unit sphere and the
    shared ones kept once; 10 f^2 + 2 vertices.  Returned sorted
    lexicographically (the product keeps generation order)."""
    ph = (1.0 + math.sqrt(5.0)) / 2.0
    ico = np.array([[-1, ph, 0], [1, ph, 0], [-1, -ph, 0], [1, -ph, 0], [0, -1, ph], [0, 1, ph], [0, -1, -ph],
                    [0, 1, -ph], [ph, 0, -1], [ph, 0, 1], [-ph, 0, -1], [-ph, 0, 1]], dtype=np.float64)
    ico /= np.linalg.norm(ico, axis=1, keepdims=True)
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    pts = {}
    f = int(frequency)
    for a, b, c in faces:
        for i in range(f + 1):
            for j in range(f + 1 - i):
                p = ((f - i - j) * ico[a] + i * ico[b] + j * ico[c]) / f
                p = p / np.linalg.norm(p)
                pts.setdefault(tuple(np.round(p * 1e9).astype(np.int64)), p)
    v = np.array(sorted(pts.values(), key=tuple))
    if hemisphere:
        e = 1e-12
        keep = (v[:, 2] > e) | ((np.abs(v[:, 2]) <= e) & (v[:, 1] > e)) | \
            ((np.abs(v[:, 2]) <= e) & (np.abs(v[:, 1]) <= e) & (v[:, 0] > 0))
        v = v[keep]
    return v


def odf_matrix(dirs, radial_order, zeta):
    """ODF amplitudes per SHORE coefficient on ``dirs``: sh2amp (Tournier, the
    values rounded to float32) times the SHORE-to-Tournier projection at
    lmax = radial_order (src/odf.rs:79-102)."""
    lmax = radial_order - radial_order % 2
    return sh2amp_cart(dirs, lmax) @ shore_to_tournier(radial_order, zeta, lmax)


# ------------------------------------------------------------- ODF peaks, GFA
# The quantities of the SHORE ODX export (src/io/odx_out.rs:1008-1090): the ODF
# sampled on a hemisphere, GFA in the form written at odx_out.rs:1036-1050,
# peaks with a relative threshold and a separation angle.  The reference
# samples DSI Studio's ODF8 hemisphere and finds peaks with odx-rs (source
# absent); this restates a mesh local-maximum finder on the hemisphere of the
# class I geodesic sphere, so directions and GFA are not pinned to the
# reference's sphere.

def geodesic_mesh(frequency):
    """(vertices (n, 3), edges (m, 2), hemisphere index of every vertex) of the
    class I geodesic sphere, vertices in generation order: faces of the
    icosahedron in a fixed order, grid points (i, j) with i + j <= f."""
    ph = (1.0 + math.sqrt(5.0)) / 2.0
    ico = np.array([[-1, ph, 0], [1, ph, 0], [-1, -ph, 0], [1, -ph, 0], [0, -1, ph], [0, 1, ph], [0, -1, -ph],
                    [0, 1, -ph], [ph, 0, -1], [ph, 0, 1], [-ph, 0, -1], [-ph, 0, 1]], dtype=np.float64)
    ico /= np.linalg.norm(ico, axis=1, keepdims=True)
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    f = int(frequency)
    ids, verts, edges = {}, [], set()
    for a, b, c in faces:
        grid = {}
        for i in range(f + 1):
            for j in range(f + 1 - i):
                p = ((f - i - j) * ico[a] + i * ico[b] + j * ico[c]) / f
                p = p / np.linalg.norm(p)
                key = tuple(np.round(p * 1e9).astype(np.int64))
                if key not in ids:
                    ids[key] = len(verts)
                    verts.append(p)
                grid[i, j] = ids[key]
        for i in range(f):
            for j in range(f - i):
                for u, w in ((grid[i, j], grid[i + 1, j]), (grid[i, j], grid[i, j + 1]),
                             (grid[i + 1, j], grid[i, j + 1])):
                    edges.add((min(u, w), max(u, w)))
    v = np.array(verts)
    e = 1e-12
    upper = (v[:, 2] > e) | ((np.abs(v[:, 2]) <= e) & (v[:, 1] > e)) | \
        ((np.abs(v[:, 2]) <= e) & (np.abs(v[:, 1]) <= e) & (v[:, 0] > 0))
    hemi = np.full(len(v), -1)
    hemi[upper] = np.arange(upper.sum())
    for i in np.flatnonzero(~upper):
        j = ids.get(tuple(np.round(-v[i] * 1e9).astype(np.int64)))
        if j is not None:
            hemi[i] = hemi[j]
    return v, np.array(sorted(edges)), hemi


def _is_upper(p, e=1e-12):
    return p[2] > e or (abs(p[2]) <= e and p[1] > e) or (abs(p[2]) <= e and abs(p[1]) <= e and p[0] > 0)


def odf_peaks(coefs, radial_order, zeta, frequency=6, npeaks=5, relative_peak_threshold=0.5,
              min_separation_angle=25.0):
    """GFA, peak directions (npeaks, 3), amplitudes and QA of one voxel's
    coefficients: amplitudes on the hemisphere clipped at 0; GFA =
    sqrt(max(0, n/(n-1) (m2 - m1^2/n) / m2)); local maxima of the mesh (not
    below any neighbour, antipodes folded), in decreasing amplitude, stop below
    the relative threshold x the largest, skip any within the separation
    angle of a kept peak."""
    v, edges, hemi = geodesic_mesh(frequency)
    R = int(hemi.max()) + 1
    dirs = np.zeros((R, 3))
    first = np.full(R, -1)
    for i in range(len(v)):  # the upper vertex of each pair comes first in hemisphere numbering
        if first[hemi[i]] < 0 and _is_upper(v[i]):
            first[hemi[i]] = i
            dirs[hemi[i]] = v[i]
    nbrs = [set() for _ in range(R)]
    for a, b in edges:
        ha, hb = hemi[a], hemi[b]
        if ha >= 0 and hb >= 0 and ha != hb:
            nbrs[ha].add(hb)
            nbrs[hb].add(ha)
    A = odf_matrix(dirs, radial_order, zeta)
    amp = np.maximum(A @ _f64(coefs), 0.0)
    n = float(R)
    m1, m2 = amp.sum(), (amp * amp).sum()
    gfa = math.sqrt(max((n / (n - 1.0)) * (m2 - m1 * m1 / n) / m2, 0.0)) if m2 > 0 and R > 1 else 0.0
    cand = [r for r in range(R) if amp[r] > 0 and all(amp[r] >= amp[q] for q in nbrs[r])]
    cand.sort(key=lambda r: (-amp[r], r))
    cos_sep = math.cos(math.radians(min_separation_angle))
    out_d, out_v = [], []
    for r in cand:
        if len(out_d) == npeaks or amp[r] < relative_peak_threshold * amp[cand[0]]:
            break
        if all(abs(dirs[r] @ d) < cos_sep for d in out_d):
            out_d.append(dirs[r])
            out_v.append(amp[r])
    D = np.zeros((npeaks, 3))
    Vv = np.zeros(npeaks)
    D[:len(out_d)] = out_d
    Vv[:len(out_v)] = out_v
    qa = np.where(Vv > 0, np.maximum(Vv - amp.min(), 0.0), 0.0)
    return gfa, D, Vv, qa, amp


# --------------------------------------------------- per-voxel designs (graddev)

def effective_table(bvals, bvecs, T, b0_threshold=50.0):
    """Effective table of one deviation tensor T (src/graddev.rs:160-185 with
    the identity frame rotation): for a diffusion-weighted sample with a
    non-zero direction g, q = T^T g/|g|, b_eff = b |q|^2, dir = q / |q|;
    other samples keep their b and direction."""
    b = _f64(bvals).copy()
    d = _f64(bvecs).reshape(-1, 3).copy()
    T = _f64(T).reshape(3, 3)
    for i in range(b.size):
        gn = np.linalg.norm(d[i])
        if b[i] > b0_threshold and gn > 1e-12:
            q = T.T @ (d[i] / gn)
            b[i] = b[i] * (q @ q)
            d[i] = q / np.linalg.norm(q)
    return b, d


def graddev_fit(signal, bvals, bvecs, T, keep, alpha, radial_order=8, zeta=700.0, big_delta=None, small_delta=None,
                max_iter=1000, tol=1e-6, non_negative=False):
    """One voxel on its own design: the effective table, the kept samples,
    the design matrix of those rows and the reference FISTA on it.  Returns
    (coefficients, iterations, converged, design)."""
    b, d = effective_table(bvals, bvecs, T)
    k = np.ones(b.size, bool) if keep is None else np.asarray(keep, bool)
    M = design_matrix(b[k], d[k], radial_order, zeta, big_delta=big_delta, small_delta=small_delta)
    c, it, conv, _ = fista_fit(M, _f64(signal)[k], alpha, max_iter=max_iter, tol=tol, non_negative=non_negative)
    return c, it, conv, M
