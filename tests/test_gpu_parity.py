"""Parity of the CUDA library with the CPU oracle on identical seeded inputs.

Tolerances.  The FP64 path runs the reference's iteration (fista.rs:70-143)
in Gram form on FP64 tensor cores, so iterates differ from the oracle only by
rounding; the stopping rule ||dx|| < tol ||x|| can then end a voxel's loop
one iteration earlier or later, which moves its coefficients by about
tol * ||x||.  Coefficient parity is therefore stated as relative L2 <= 1e-5
per voxel (the bound the specification sets for the FP64 path), with
iteration counts equal up to that one-step slack.  Tikhonov is a direct solve:
its agreement is bounded by cond(A) * eps, so it is checked at 1e-8 for
lambda = 0.05 and through the reference's normal-equation residual at the
default lambda = 1e-8.
"""

from contextlib import contextmanager

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPT_FISTA_SHAPE, OPT_FISTA_SCHEDULE = 1, 2  # csd_set_option


@contextmanager
def handle_option(option, value, default):
    """A tuning option of the shared device-0 handle for the block's calls."""
    from cs_dmri_b200 import _abi
    _abi.set_option(option, value)
    try:
        yield
    finally:
        _abi.set_option(option, default)


@pytest.fixture(scope="module")
def ph():
    from cs_dmri_b200.phantom import make_phantom
    p = make_phantom((8, 8, 4), seed=7)
    p.data[0, 0, 0, :] = 0.0        # an all-zero voxel (alpha_max == 0 path)
    return p


def both(ph, oracle, mask=None, **kw):
    from cs_dmri_b200 import shore_fit
    mask = ph.mask if mask is None else mask
    common = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, diagnostics=True)
    common.update(kw)
    gpu = shore_fit(ph.data, ph.bvals, ph.bvecs, mask, return_coef64=True, **common)
    ref = oracle.shore_fit(ph.data, ph.bvals, ph.bvecs, mask, **common)
    return gpu, ref


def rel_rows(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def test_design_matrix_matches_oracle(ph, oracle):
    from cs_dmri_b200 import design_matrix
    for order in (2, 4, 6, 8):
        g = design_matrix(ph.bvals, ph.bvecs, order, 700.0, big_delta=ph.big_delta, small_delta=ph.small_delta)
        o = oracle.design_matrix(ph.bvals, ph.bvecs, order, 700.0, big_delta=ph.big_delta,
                                 small_delta=ph.small_delta)
        assert g.shape == o.shape
        assert np.abs(g - o).max() <= 1e-13 * np.abs(o).max()


def test_fixed_alpha_l1_parity(ph, oracle):
    gpu, ref = both(ph, oracle, alpha_mode="fixed", alpha=0.01)
    assert gpu["n_voxels"] == ref["n_voxels"] == ph.n_voxels
    r = rel_rows(gpu["coef64"], ref["coef64"])
    r = r[np.linalg.norm(ref["coef64"], axis=1) > 0]
    assert r.max() <= 1e-5, r.max()
    it_g = gpu["iterations"][ph.mask].astype(int)
    it_o = ref["iterations"][ph.mask].astype(int)
    assert np.abs(it_g - it_o).max() <= 1
    assert np.mean(it_g == it_o) >= 0.9
    assert np.array_equal(gpu["converged"], ref["converged"]) or np.mean(gpu["converged"] == ref["converged"]) > 0.99
    np.testing.assert_allclose(gpu["residual_l2"], ref["residual_l2"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(gpu["r2"], ref["r2"], rtol=1e-5, atol=1e-6)
    assert np.array_equal(gpu["alpha"], ref["alpha"])
    np.testing.assert_allclose(gpu["bic"], ref["bic"], rtol=1e-5, atol=1e-3)
    assert np.array_equal(gpu["regularization_kind"], ref["regularization_kind"])
    # float32 coefficient volume is the rounded FP64 result, zeros outside the mask
    np.testing.assert_allclose(gpu["coefficients"], ref["coefficients"], rtol=1e-4, atol=1e-3)
    assert gpu["sidecar"] == ref["sidecar"]


@pytest.mark.parametrize("lam", [0.05])
def test_tikhonov_parity(ph, oracle, lam):
    gpu, ref = both(ph, oracle, regularization="l2", lambda_n=lam, lambda_l=lam)
    r = rel_rows(gpu["coef64"], ref["coef64"])
    r = r[np.linalg.norm(ref["coef64"], axis=1) > 0]
    assert r.max() <= 1e-8, r.max()
    assert np.all(gpu["iterations"][ph.mask] == 1) and np.all(gpu["regularization_kind"][ph.mask] == 2)
    np.testing.assert_allclose(gpu["residual_l2"], ref["residual_l2"], rtol=1e-7)
    assert gpu["sidecar"] == ref["sidecar"]


def test_tikhonov_default_lambda_normal_equations(ph, oracle):
    """src/solver/tikhonov.rs at lambda = 1e-8: normal-equation residual, as
    tests/optimization_kkt.rs:189-215 checks it (< 1e-9)."""
    gpu, _ = both(ph, oracle, regularization="l2")
    M = oracle.design_matrix(ph.bvals, ph.bvecs, 6, 700.0, big_delta=ph.big_delta, small_delta=ph.small_delta)
    nd, ld = oracle.regularization(6)
    S = ph.data.reshape(-1, ph.data.shape[-1])[ph.mask.ravel()].astype(np.float64)
    for c, s in zip(gpu["coef64"][1:], S[1:]):
        lhs = M.T @ M @ c + 1e-8 * nd * c + 1e-8 * ld * c
        rhs = M.T @ s
        assert np.linalg.norm(lhs - rhs) / np.linalg.norm(rhs) < 1e-9


def test_alpha_ratio_parity(ph, oracle):
    gpu, ref = both(ph, oracle, alpha_mode="alpha-ratio", alpha_ratio=0.05)
    r = rel_rows(gpu["coef64"], ref["coef64"])
    nz = np.linalg.norm(ref["coef64"], axis=1) > 0
    assert r[nz].max() <= 1e-5
    np.testing.assert_allclose(gpu["alpha"], ref["alpha"], rtol=1e-12)
    assert gpu["alpha"][0, 0, 0] == 0.0 and gpu["iterations"][0, 0, 0] == 0
    assert gpu["bic"][0, 0, 0] == 0.0 and np.all(gpu["coefficients"][0, 0, 0] == 0)
    assert gpu["alpha_distribution"] == pytest.approx(ref["alpha_distribution"], rel=1e-12)


@pytest.mark.parametrize("mode", ["path-bic", "l2-anchored"])
def test_path_strategy_parity(ph, oracle, mode):
    gpu, ref = both(ph, oracle, alpha_mode=mode)
    same = np.isclose(gpu["alpha"][ph.mask], ref["alpha"][ph.mask], rtol=1e-9, atol=0)
    assert same.mean() >= 0.98, same.mean()
    r = rel_rows(gpu["coef64"], ref["coef64"])
    nz = np.linalg.norm(ref["coef64"], axis=1) > 0
    assert r[same & nz].max() <= 1e-5
    assert gpu["alpha"][0, 0, 0] == 0.0 and gpu["iterations"][0, 0, 0] == 0
    if mode == "l2-anchored":
        np.testing.assert_allclose(gpu["rss_l2"], ref["rss_l2"], rtol=1e-6)
    assert gpu["alpha_distribution"] == pytest.approx(ref["alpha_distribution"], rel=1e-9)
    assert gpu["sidecar"]["solver"]["alpha_strategy"] == ref["sidecar"]["solver"]["alpha_strategy"]


def test_empty_mask(ph, oracle):
    gpu, ref = both(ph, oracle, mask=np.zeros(ph.mask.shape, bool), alpha_mode="fixed", alpha=0.01)
    assert gpu["n_voxels"] == 0 and np.all(gpu["coefficients"] == 0)


def test_partial_mask_zeros_outside(ph, oracle):
    m = np.zeros(ph.mask.shape, bool)
    m[2:5, 1:7, 1:3] = True
    gpu, ref = both(ph, oracle, mask=m, alpha_mode="fixed", alpha=0.01)
    assert np.all(gpu["coefficients"][~m] == 0) and np.all(gpu["r2"][~m] == 0)
    assert rel_rows(gpu["coef64"], ref["coef64"]).max() <= 1e-5


def test_nan_voxel_matches_reference_semantics(ph, oracle):
    """A NaN sample makes every soft-threshold comparison false, so the
    reference's prox falls through to 0.0 (src/solver/fista.rs:99-107): the
    voxel converges to zero coefficients at iteration 1.  Other voxels are
    unaffected."""
    data = ph.data.copy()
    data[1, 1, 1, 5] = np.nan
    from cs_dmri_b200 import shore_fit
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01,
              diagnostics=True, max_iter=50)
    out = shore_fit(data, ph.bvals, ph.bvecs, ph.mask, **kw)
    ref = oracle.shore_fit(data, ph.bvals, ph.bvecs, ph.mask, **kw)
    bad = np.zeros(ph.mask.shape, bool)
    bad[1, 1, 1] = True
    assert np.all(np.isfinite(out["coefficients"][~bad]))
    assert out["iterations"][1, 1, 1] == ref["iterations"][1, 1, 1] == 1
    assert np.all(out["coefficients"][1, 1, 1] == 0) and np.all(ref["coefficients"][1, 1, 1] == 0)
    np.testing.assert_array_equal(np.isnan(out["residual_l2"]), np.isnan(ref["residual_l2"]))


def test_max_iter_zero_returns_start(ph, oracle):
    from cs_dmri_b200 import shore_fit
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01,
              diagnostics=True, max_iter=0)
    out = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, return_coef64=True, **kw)
    ref = oracle.shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    assert np.all(out["coef64"] == 0) and np.all(ref["coef64"] == 0)
    assert np.all(out["iterations"] == 0) and not out["converged"].any() and not ref["converged"].any()


def test_single_shell_refused_and_allowed(oracle):
    from cs_dmri_b200 import shore_fit
    z = np.linspace(-1, 1, 40)
    r = np.sqrt(1 - z * z)
    phi = 2.399963 * np.arange(40)
    bvecs = np.vstack([[0, 0, 1], [0, 0, 1], np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)])
    bvals = np.concatenate([[0, 0], np.full(40, 1000.0)])
    data = np.broadcast_to(np.exp(-bvals * 8e-4).astype(np.float32), (2, 2, 1, 42)).copy()
    mask = np.ones((2, 2, 1), bool)
    with pytest.raises(ValueError, match="at least 2 b-value shells"):
        shore_fit(data, bvals, bvecs, mask, big_delta=0.04, small_delta=0.01, regularization="l2")
    out = shore_fit(data, bvals, bvecs, mask, big_delta=0.04, small_delta=0.01, regularization="l2",
                    allow_single_shell=True)
    assert any("only the orientation information" in w for w in out["warnings"])
    with pytest.raises(ValueError, match="b=0 threshold"):
        shore_fit(data, np.zeros(42), bvecs, mask, regularization="l2", allow_single_shell=True)


def test_argument_errors(ph):
    from cs_dmri_b200 import shore_fit
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta)
    with pytest.raises(ValueError, match="positive even"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, radial_order=5, **kw)
    with pytest.raises(ValueError, match="path-n-alphas"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, path_n_alphas=1, **kw)
    with pytest.raises(ValueError, match="path-eps"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, path_eps=2.0, **kw)
    with pytest.raises(ValueError, match="alpha-ratio"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, alpha_mode="alpha-ratio", alpha_ratio=1.5, **kw)
    with pytest.raises(ValueError, match="slack"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, slack=-1.0, **kw)
    with pytest.raises(ValueError, match="volumes"):
        shore_fit(ph.data[..., :-1], ph.bvals, ph.bvecs, ph.mask, **kw)


def test_shore_model_interface(ph, oracle):
    from cs_dmri_b200 import GradientTable, ShoreModel
    gt = GradientTable(ph.bvals, ph.bvecs, big_delta=ph.big_delta, small_delta=ph.small_delta)
    fit = ShoreModel(gt, regularization="l2", lambda_n=0.05, lambda_l=0.05).fit(ph.data, ph.mask)
    ref = oracle.shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta,
                           small_delta=ph.small_delta, regularization="l2", lambda_n=0.05, lambda_l=0.05,
                           diagnostics=True)
    assert fit.coefficients.shape == ph.data.shape[:3] + (72,)
    assert fit.frame == "image" and fit.r2 is not None
    np.testing.assert_allclose(fit.r2, ref["r2"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(fit.rmse, ref["rmse"], rtol=1e-6)
    assert fit.sidecar["solver"]["kind"] == "tikhonov" and not fit.single_shell
    sp = fit.sparsity[ph.mask]
    assert sp[0] == 0.0 and sp[1:].min() > 0.9 and "256 voxels" in repr(fit)


@pytest.mark.parametrize("shape", [1, 12, 16])
def test_fista_kernel_variants_match_oracle(ph, oracle, shape):
    """Every FISTA kernel shape (k_fista_fp64; k_fista_v3 with 12 or 16
    warps per CTA) runs the same per-voxel iteration."""
    with handle_option(OPT_FISTA_SHAPE, shape, 0):
        fits = {mode: both(ph, oracle, alpha_mode=mode, alpha=0.01) for mode in ("fixed", "l2-anchored")}
    for mode, (gpu, ref) in fits.items():
        same = np.isclose(gpu["alpha"][ph.mask], ref["alpha"][ph.mask], rtol=1e-9, atol=0)
        assert same.mean() >= 0.98
        r = rel_rows(gpu["coef64"], ref["coef64"])
        nz = np.linalg.norm(ref["coef64"], axis=1) > 0
        assert r[same & nz].max() <= 1e-5, (shape, mode, r[same & nz].max())
        it_g = gpu["iterations"][ph.mask].astype(int)
        it_o = ref["iterations"][ph.mask].astype(int)
        assert np.abs(it_g - it_o)[same].max() <= 1


def test_pinned_input_and_output_buffers_match(ph):
    """A page-locked input volume is read in place (masked rows only) and a
    caller-supplied output is filled completely; both give the same result
    as pageable buffers."""
    import torch
    from cs_dmri_b200 import shore_fit
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, diagnostics=True, return_coef64=True)
    for mode in ("fixed", "l2-anchored"):
        ref = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, alpha_mode=mode, alpha=0.01, **kw)
        pin = torch.empty(ph.data.shape, dtype=torch.float32, pin_memory=True)
        pin.numpy()[...] = ph.data
        out = torch.full(ph.data.shape[:3] + (72,), float("nan"), dtype=torch.float32, pin_memory=True)
        got = shore_fit(pin.numpy(), ph.bvals, ph.bvecs, ph.mask, alpha_mode=mode, alpha=0.01,
                        coefficients_out=out.numpy(), **kw)
        assert got["coefficients"] is out.numpy() or np.shares_memory(got["coefficients"], out.numpy())
        np.testing.assert_array_equal(out.numpy(), ref["coefficients"])
        np.testing.assert_array_equal(got["coef64"], ref["coef64"])
        for k in ("r2", "residual_l2", "iterations", "alpha", "bic"):
            np.testing.assert_array_equal(got[k], ref[k])
    with pytest.raises(ValueError, match="coefficients_out"):
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, coefficients_out=np.zeros((2, 2, 2, 72), np.float32),
                  big_delta=ph.big_delta, small_delta=ph.small_delta)


@pytest.mark.parametrize("order", [2, 4, 8])
def test_other_radial_orders(order, oracle):
    """Radial orders 2, 4 and 8 (K = 8, 29, 145) run the same kernels with other
    tile counts; order 8 reads its Gram tiles through the caches and uses the
    FFMA right-hand-side and residual passes."""
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((5, 4, 3), seed=31 + order)
    for kw in (dict(alpha_mode="fixed", alpha=0.01), dict(alpha_mode="l2-anchored"),
               dict(regularization="l2", lambda_n=0.05, lambda_l=0.05)):
        gpu, ref = both(ph, oracle, radial_order=order, **kw)
        assert gpu["coefficients"].shape[-1] == oracle.n_coeffs(order)
        if kw.get("regularization") == "l2":
            r = rel_rows(gpu["coef64"], ref["coef64"])
            assert r.max() <= 1e-8, (order, r.max())
            continue
        same = np.isclose(gpu["alpha"][ph.mask], ref["alpha"][ph.mask], rtol=1e-9, atol=0)
        assert same.mean() >= 0.95, (order, kw, same.mean())
        r = rel_rows(gpu["coef64"], ref["coef64"])
        nz = np.linalg.norm(ref["coef64"], axis=1) > 0
        assert r[same & nz].max() <= 1e-5, (order, kw, r[same & nz].max())


@contextmanager
def icls_form(form):
    from cs_dmri_b200 import _abi
    _abi.set_option(_abi.OPT_ICLS, {"gram": 0, "basis": 1}[form])
    try:
        yield
    finally:
        _abi.set_option(_abi.OPT_ICLS, 0)


@pytest.mark.parametrize("form", ["gram", "basis"])
@pytest.mark.parametrize("order", [2, 4, 6])
def test_amplitude_icls_parity(order, form, oracle):
    """Goldfarb-Idnani positivity QP (src/solver/icls.rs via shore_icls.rs),
    in both kernel forms: the Gram form (constraint values carried through
    W^T W, the default for radial orders <= 6) and the orthogonal-basis form.
    The minimiser is unique, so coefficients agree with the oracle's to the
    QP's conditioning; every constraint holds to the solver tolerance and the
    objective matches."""
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((6, 5, 4), seed=41 + order)
    kw = dict(regularization="nonneg", radial_order=order)
    with icls_form(form):
        gpu, ref = both(ph, oracle, **kw)
    assert gpu["sidecar"]["solver"] == ref["sidecar"]["solver"]
    assert gpu["sidecar"]["solver"]["n_constraint_dirs"] == 321
    assert np.all(gpu["regularization_kind"][ph.mask] == 3)
    assert gpu["converged"].all() and ref["converged"].all()
    r = rel_rows(gpu["coef64"], ref["coef64"])
    assert np.median(r) <= 1e-8 and r.max() <= 1e-5, (np.median(r), r.max())
    # feasibility on the constraint sphere and equal objective values
    M = oracle.design_matrix(ph.bvals, ph.bvecs, order, 700.0, big_delta=ph.big_delta, small_delta=ph.small_delta)
    lmax = order
    Cm = oracle.sh2amp_cart(oracle.odf8_hemisphere(), lmax) @ oracle.shore_to_tournier(order, 700.0, lmax)
    S = ph.data.reshape(-1, ph.data.shape[-1])[ph.mask.ravel()].astype(np.float64)
    scale = np.abs(Cm @ gpu["coef64"].T).max()
    assert (Cm @ gpu["coef64"].T).min() >= -1e-7 * max(scale, 1.0)
    obj_g = 0.5 * ((gpu["coef64"] @ M.T - S) ** 2).sum(1)
    obj_o = 0.5 * ((ref["coef64"] @ M.T - S) ** 2).sum(1)
    np.testing.assert_allclose(obj_g, obj_o, rtol=1e-9)
    it_g = gpu["iterations"][ph.mask].astype(int)
    it_o = ref["iterations"][ph.mask].astype(int)
    assert np.mean(np.abs(it_g - it_o) <= 1) >= 0.9
    np.testing.assert_allclose(gpu["residual_l2"], ref["residual_l2"], rtol=1e-6)


def test_icls_forms_follow_one_iteration_path():
    """The Gram form and the orthogonal-basis form take the reference's steps
    from the same start, so their minimisers agree to rounding and their
    iteration counts match (a near-tie between two violated constraints may
    be broken the other way by rounding: at most 1 % of voxels)."""
    from cs_dmri_b200 import shore_fit
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((12, 10, 6), seed=44)
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, diagnostics=True, return_coef64=True,
              regularization="nonneg")
    out = {}
    for form in ("gram", "basis"):
        with icls_form(form):
            out[form] = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    g, b = out["gram"], out["basis"]
    assert g["converged"].all() and b["converged"].all()
    r = rel_rows(g["coef64"], b["coef64"])
    assert np.median(r) <= 1e-9 and r.max() <= 1e-6, (np.median(r), r.max())
    same = g["iterations"][ph.mask] == b["iterations"][ph.mask]
    assert same.mean() >= 0.99, same.mean()


def test_long_gradient_table_uses_the_general_rhs(oracle):
    """N = 518 (the table given twice) at radial order 4: beyond the DMMA
    right-hand-side kernel's 288-sample limit, so the general kernel runs;
    the fit must still match the oracle on the same input."""
    from cs_dmri_b200 import shore_fit
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((5, 4, 3), seed=13)
    data = np.concatenate([ph.data, ph.data], axis=-1)
    bvals = np.concatenate([ph.bvals, ph.bvals])
    bvecs = np.concatenate([ph.bvecs, ph.bvecs])
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, radial_order=4, alpha_mode="fixed",
              alpha=0.01, diagnostics=True)
    gpu = shore_fit(data, bvals, bvecs, ph.mask, return_coef64=True, **kw)
    ref = oracle.shore_fit(data, bvals, bvecs, ph.mask, **kw)
    r = rel_rows(gpu["coef64"], ref["coef64"])
    assert r.max() <= 1e-5, r.max()


def test_pipelined_host_fit_matches_the_device_fit():
    """A page-locked volume fitted with fixed alpha and only coefficients
    requested takes the pipelined host path (chunks of the right-hand side
    overlap the iterations, slabs of the coefficient volume are copied back
    chunk by chunk).  Same kernels, same per-voxel arithmetic: the result is
    bit-identical to the device-buffer fit and to the pageable host fit."""
    import torch
    from cs_dmri_b200 import _abi, shore_fit, shore_fit_device
    from cs_dmri_b200.phantom import make_phantom
    rng = np.random.default_rng(2)
    mask = rng.random((48, 48, 48)) < 0.9
    ph = make_phantom((48, 48, 48), mask=mask, seed=5)   # ~99.5 k voxels -> 3 chunks (0.15 / 0.425 / 0.425)
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01)
    pin = torch.empty(ph.data.shape, dtype=torch.float32, pin_memory=True)
    pin.numpy()[...] = ph.data
    out = torch.full(ph.data.shape[:3] + (72,), float("nan"), dtype=torch.float32, pin_memory=True)
    got = shore_fit(pin.numpy(), ph.bvals, ph.bvecs, ph.mask, coefficients_out=out.numpy(), **kw)
    t = _abi.last_timing(0)
    assert t.ms_rhs == 0.0  # the right-hand side ran overlapped (pipelined path)
    pageable = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    dev, _ = shore_fit_device(torch.from_numpy(ph.data).cuda(), torch.from_numpy(ph.mask).cuda(), ph.bvals,
                              ph.bvecs, **kw)
    np.testing.assert_array_equal(out.numpy(), pageable["coefficients"])
    np.testing.assert_array_equal(out.numpy(), dev.cpu().numpy())
    assert got["total_iterations"] == pageable["total_iterations"]
    # a page-locked output is written in place by the scatter kernels; a
    # pageable one gets the slab copies
    out2 = np.full(ph.data.shape[:3] + (72,), np.nan, np.float32)
    shore_fit(pin.numpy(), ph.bvals, ph.bvecs, ph.mask, coefficients_out=out2, **kw)
    assert _abi.last_timing(0).ms_rhs == 0.0
    np.testing.assert_array_equal(out2, pageable["coefficients"])


def test_pageable_buffers_of_small_and_empty_masks():
    """Pageable input and output on the pipelined path when the mask is
    small (one chunk; given as non-0/1 bytes, which the wrapper maps to 0/1)
    or empty: the staging holds the masked rows only, the caller's output is
    filled completely (masked rows from the fit, the others zero), and the
    result equals the device-buffer fit bit for bit."""
    import torch
    from cs_dmri_b200 import shore_fit, shore_fit_device
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((20, 18, 10), seed=8)
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01)
    mask8 = ph.mask.astype(np.uint8) * 7  # any non-zero byte is inside
    out = np.full(ph.data.shape[:3] + (72,), np.nan, np.float32)
    shore_fit(ph.data, ph.bvals, ph.bvecs, mask8, coefficients_out=out, **kw)
    dev, _ = shore_fit_device(torch.from_numpy(ph.data).cuda(), torch.from_numpy(ph.mask).cuda(), ph.bvals,
                              ph.bvecs, **kw)
    np.testing.assert_array_equal(out, dev.cpu().numpy())
    empty = np.zeros(ph.mask.shape, bool)
    out0 = np.full(ph.data.shape[:3] + (72,), np.nan, np.float32)
    shore_fit(ph.data, ph.bvals, ph.bvecs, empty, coefficients_out=out0, **kw)
    assert np.all(out0 == 0.0)


def test_fista_autotuner_choice_changes_nothing():
    """The per-table autotuner picks k_fista_v3's warps per CTA (12 or 16)
    from a timed synthetic batch; both give bit-identical fits."""
    from cs_dmri_b200 import _abi, shore_fit
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((12, 10, 8), seed=23)
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01,
              return_coef64=True)
    auto = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    t = _abi.last_timing(0)
    assert t.fista_warps in (12, 16)
    assert t.fista_tune_ms12 > 0 and t.fista_tune_ms16 > 0
    assert t.fista_warps == (12 if t.fista_tune_ms12 < t.fista_tune_ms16 else 16)
    fits = {}
    for shape in (12, 16):
        with handle_option(OPT_FISTA_SHAPE, shape, 0):
            fits[shape] = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    for f in fits.values():
        np.testing.assert_array_equal(f["coef64"], auto["coef64"])
        np.testing.assert_array_equal(f["coefficients"], auto["coefficients"])


def test_two_pass_fista_schedule_changes_nothing():
    """With at least four voxels per FISTA slot a fit runs in two passes:
    every voxel up to iteration 80, then the unfinished ones resumed from
    their exact state, largest predicted remaining iteration count first.  The
    coefficients, iteration counts and convergence flags are bit-identical to
    a single pass (handle option CSD_OPT_FISTA_SCHEDULE = 0), on the device-buffer path and on the
    pipelined host path (whose larger chunks take the two passes)."""
    import torch
    from cs_dmri_b200 import _abi, shore_fit
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((64, 64, 50), seed=31)  # 204,800 voxels
    V = int(ph.mask.sum())
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01)
    two = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, return_coef64=True, diagnostics=True, **kw)
    parked = _abi.last_timing(0).fista_parked
    assert 0.5 * V < parked <= V
    with handle_option(OPT_FISTA_SCHEDULE, 0, 1):
        one = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, return_coef64=True, diagnostics=True, **kw)
        assert _abi.last_timing(0).fista_parked == 0
    for k in ("coef64", "coefficients", "iterations", "converged"):
        np.testing.assert_array_equal(two[k], one[k])
    assert two["total_iterations"] == one["total_iterations"]
    pin = torch.empty(ph.data.shape, dtype=torch.float32, pin_memory=True)
    pin.numpy()[...] = ph.data
    out = torch.full(ph.data.shape[:3] + (72,), float("nan"), dtype=torch.float32, pin_memory=True)
    got = shore_fit(pin.numpy(), ph.bvals, ph.bvecs, ph.mask, coefficients_out=out.numpy(), **kw)
    t = _abi.last_timing(0)
    assert t.ms_rhs == 0.0 and 0 < t.fista_parked < V  # pipelined; its two larger chunks took two passes
    np.testing.assert_array_equal(out.numpy(), one["coefficients"])
    assert got["total_iterations"] == one["total_iterations"]
