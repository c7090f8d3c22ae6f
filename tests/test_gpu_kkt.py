"""Converged-optimum L1 fits (precision "mixed-kkt": TF32 tensor-core FISTA
iterations for the support, FP64 active-set polish; "fp64-kkt": the same with
FP64 iterations) against the oracle's optimum.

The oracle's optimum of a voxel is the exact solve on the support and signs
of its reference-rule FISTA iterate (oracle.lasso_optimum_rows), kept only
where its KKT conditions certify it: a certified point is the LASSO minimiser
(the objective is convex), so it pins the result independently of how the
GPU found its support.  Both sides solve the same FP64 linear system on the
same support; a coordinate whose |M_j^T r| / n sits within about 1e-9 of
alpha may be taken or left (either is certified), which moves the solution by
~1e-8 relative.  The bound stated for these modes is per-voxel relative L2
<= 1e-6 against the certified optimum (the specification's 1e-5 with room
to spare), and every certified voxel's KKT residual (the form of the
reference's tests/common/mod.rs:127-153) is at most 1e-8.
"""

from contextlib import contextmanager

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@contextmanager
def kkt_iterations(k):
    from cs_dmri_b200 import _abi
    _abi.set_option(_abi.OPT_KKT_ITERATIONS, k)
    try:
        yield
    finally:
        _abi.set_option(_abi.OPT_KKT_ITERATIONS, 0)


@pytest.fixture(scope="module")
def ph():
    from cs_dmri_b200.phantom import make_phantom
    p = make_phantom((12, 10, 6), seed=27)
    p.data[0, 0, 0, :] = 0.0               # zero signal: alpha_max = 0, c = 0
    p.data[1, 0, 0, 7] = np.nan            # a NaN sample: zero coefficients, not certified
    return p


def rows(ph):
    n = ph.data.shape[-1]
    return ph.data.reshape(-1, n)[ph.mask.ravel()].astype(np.float64)


def kkt_residuals(M, S, C, alpha, non_negative=False):
    n = M.shape[0]
    g = (C @ M.T - S) @ M / n
    act = (C > 1e-10) if non_negative else (np.abs(C) > 1e-10)
    sg = np.ones_like(C) if non_negative else np.sign(C)
    a = np.where(act, np.abs(g + alpha * sg), 0.0).max(1)
    exc = (-g - alpha) if non_negative else (np.abs(g) - alpha)
    i = np.where(act, 0.0, np.maximum(exc, 0.0)).max(1)
    return np.maximum(a, i)


def optimum(ph, oracle, order=6, **kw):
    """The oracle's certified optimum of every masked voxel (rows, ok)."""
    ref = oracle.shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta,
                           small_delta=ph.small_delta, diagnostics=True, radial_order=order, **kw)
    M = oracle.design_matrix(ph.bvals, ph.bvecs, order, 700.0, big_delta=ph.big_delta, small_delta=ph.small_delta)
    S = rows(ph)
    alpha = voxel_alpha(oracle, M, S, **kw)
    C, ok = oracle.lasso_optimum_rows(M, np.nan_to_num(S), alpha, ref["coef64"],
                                      non_negative=kw.get("non_negative", False))
    ok &= np.all(np.isfinite(S), axis=1)
    return C, ok, M, S


def voxel_alpha(oracle, M, S, **kw):
    """alpha per voxel in FP64: fixed, or alpha_ratio x alpha_max (src/solver/alpha.rs:47-56)."""
    if kw.get("alpha_mode") == "alpha-ratio":
        return np.array([kw["alpha_ratio"] * oracle.alpha_max(M, s) if np.all(np.isfinite(s)) else np.nan
                         for s in S])
    return np.full(len(S), kw["alpha"])


def fit(ph, precision, order=6, **kw):
    from cs_dmri_b200 import _abi, shore_fit
    out = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                    diagnostics=True, return_coef64=True, precision=precision, radial_order=order, **kw)
    return out, _abi.last_timing(0)


def rel(a, b):
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(nb > 0, nb, 1.0)


@pytest.mark.parametrize("precision", ["mixed-kkt", "fp64-kkt"])
@pytest.mark.parametrize("kw", [dict(alpha_mode="fixed", alpha=0.01),
                                dict(alpha_mode="alpha-ratio", alpha_ratio=0.05),
                                dict(alpha_mode="fixed", alpha=0.01, non_negative=True)])
def test_certified_optimum_matches_oracle(ph, oracle, precision, kw):
    want, ok, M, S = optimum(ph, oracle, **kw)
    got, t = fit(ph, precision, **kw)
    conv = got["converged"]
    nan_vox = ~np.all(np.isfinite(S), axis=1)
    assert np.all(got["coef64"][nan_vox] == 0)
    if kw["alpha_mode"] == "fixed":
        # (with alpha-ratio the NaN voxel's alpha_max is not positive: like the
        # FP64 path, it is reported as a zero voxel, converged at 0 iterations)
        assert not conv[nan_vox].any() and t.kkt_uncertified == int(nan_vox.sum())
    assert conv[~nan_vox].all(), int((~conv[~nan_vox]).sum())
    assert t.kkt_fallback_voxels == 0
    both = ok & conv
    assert both.mean() >= 0.98
    r = rel(got["coef64"][both], want[both])
    assert r.max() <= 1e-6, float(r.max())
    alpha = voxel_alpha(oracle, M, S, **kw)
    conv = conv & ~nan_vox
    res = kkt_residuals(M, S[conv], got["coef64"][conv], alpha[conv][:, None],
                        kw.get("non_negative", False))
    assert res.max() <= 1e-8, float(res.max())
    assert 0.0 <= t.kkt_max <= 1e-8
    # the zero-signal voxel: zero coefficients, certified
    assert np.all(got["coef64"][0] == 0) and conv[0]
    it = got["iterations"][ph.mask].astype(int)
    assert np.all(it[conv & ~np.all(S == 0, axis=1)] >= 1)
    if precision == "mixed-kkt":
        assert t.tf32_tensor_flops > 0 and t.ms_kkt_iterate > 0
    else:
        assert t.tf32_tensor_flops == 0


def test_tf32_and_fp64_support_identification_reach_one_optimum(ph):
    kw = dict(alpha_mode="fixed", alpha=0.01)
    a, _ = fit(ph, "mixed-kkt", **kw)
    b, _ = fit(ph, "fp64-kkt", **kw)
    both = a["converged"] & b["converged"]
    assert both.mean() >= 0.99
    assert rel(a["coef64"][both], b["coef64"][both]).max() <= 1e-6


@pytest.mark.parametrize("k", [1, 8])
def test_few_iterations_take_more_rounds_and_reach_the_optimum(ph, oracle, k):
    """With 1 or 8 support-identification iterations the polish starts far
    from the support: it takes more rounds and ends at the same optimum."""
    kw = dict(alpha_mode="fixed", alpha=0.01)
    want, ok, M, S = optimum(ph, oracle, **kw)
    _, t64 = fit(ph, "mixed-kkt", **kw)
    with kkt_iterations(k):
        got, t = fit(ph, "mixed-kkt", **kw)
    assert t.kkt_rounds > t64.kkt_rounds
    conv = got["converged"]
    both = ok & conv
    assert conv.mean() >= 0.99 and both.mean() >= 0.97
    assert rel(got["coef64"][both], want[both]).max() <= 1e-6


def test_fallback_fit_and_last_polish(ph, oracle):
    """With one polish round allowed the first polish leaves most voxels
    uncertified: they run the FP64 FISTA path with the reference stopping rule
    and a last polish from its result, which certifies them at the same
    optimum."""
    from cs_dmri_b200 import _abi
    kw = dict(alpha_mode="fixed", alpha=0.01)
    want, ok, M, S = optimum(ph, oracle, **kw)
    _abi.set_option(_abi.OPT_KKT_ROUNDS, 1)
    try:
        with kkt_iterations(1):
            got, t = fit(ph, "mixed-kkt", **kw)
    finally:
        _abi.set_option(_abi.OPT_KKT_ROUNDS, 48)
    assert t.kkt_fallback_voxels > 0.5 * len(S) and t.ms_kkt_fallback > 0
    conv = got["converged"]
    both = ok & conv
    assert conv.mean() >= 0.99 and both.mean() >= 0.97
    assert rel(got["coef64"][both], want[both]).max() <= 1e-6


@pytest.mark.parametrize("order", [2, 4])
def test_other_radial_orders(oracle, order):
    from cs_dmri_b200.phantom import make_phantom
    ph2 = make_phantom((6, 5, 4), seed=50 + order)
    kw = dict(alpha_mode="fixed", alpha=0.01)
    want, ok, M, S = optimum(ph2, oracle, order=order, **kw)
    got, _ = fit(ph2, "mixed-kkt", order=order, **kw)
    both = ok & got["converged"]
    assert got["converged"].all() and both.mean() >= 0.98
    assert rel(got["coef64"][both], want[both]).max() <= 1e-6


def test_argument_errors(ph):
    from cs_dmri_b200 import shore_fit
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta)
    with pytest.raises(ValueError, match="alpha_mode fixed or alpha-ratio"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, precision="mixed-kkt", alpha_mode="path-bic", **kw)
    with pytest.raises(ValueError, match="radial orders 2, 4 and 6"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, precision="mixed-kkt", alpha_mode="fixed",
                  alpha=0.01, radial_order=8, **kw)
    with pytest.raises(ValueError, match="precision must be"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, precision="tf32", **kw)


def test_autotuned_support_identification(ph):
    """With no fixed count the handle times the whole path on a synthetic
    batch with 16, 24, 32 and 48 TF32 iterations, once per table, and uses
    the fastest; a fixed count gives the same certified optimum."""
    kw = dict(alpha_mode="fixed", alpha=0.01)
    auto, t = fit(ph, "mixed-kkt", **kw)
    times = list(t.kkt_tune_ms)
    assert t.kkt_iterations in (16, 24, 32, 48) and all(x > 0 for x in times)
    assert t.kkt_iterations == (16, 24, 32, 48)[int(np.argmin(times))]
    other = 48 if t.kkt_iterations != 48 else 16
    with kkt_iterations(other):
        fixed, t2 = fit(ph, "mixed-kkt", **kw)
    assert t2.kkt_iterations == other
    both = auto["converged"] & fixed["converged"]
    assert both.mean() >= 0.99
    assert rel(auto["coef64"][both], fixed["coef64"][both]).max() <= 1e-6
