"""Mixed-precision L1 path (int8 digit-slice tensor-core Gram products, FP64
state) against the FP64 oracle and the FP64 GPU path on the same inputs.

Tolerance.  The mixed path forms each Gram product G (x_k - x_{k-1}) to about
2^-32 of max|d| max|G|, so its iterates follow the FP64 iterate path closely;
a voxel whose stopping decision lies within 1 % of tol is re-fitted in FP64.
The bound stated for this path is coefficient relative L2 <= 1e-5 per voxel
(the FP64-path bound) and <= 1e-6 over the whole volume; iteration counts
match the oracle's up to the same one-step slack as the FP64 path.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ph():
    from cs_dmri_b200.phantom import make_phantom
    p = make_phantom((12, 10, 6), seed=21)
    p.data[0, 0, 0, :] = 0.0
    return p


def fit(ph, precision, mask=None, **kw):
    from cs_dmri_b200 import shore_fit
    mask = ph.mask if mask is None else mask
    return shore_fit(ph.data, ph.bvals, ph.bvecs, mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                     diagnostics=True, return_coef64=True, precision=precision, **kw)


def oracle_fit(ph, oracle, mask=None, **kw):
    mask = ph.mask if mask is None else mask
    return oracle.shore_fit(ph.data, ph.bvals, ph.bvecs, mask, big_delta=ph.big_delta,
                            small_delta=ph.small_delta, diagnostics=True, **kw)


def errors(a, b):
    nz = np.linalg.norm(b, axis=1) > 0
    per = np.linalg.norm(a - b, axis=1)[nz] / np.linalg.norm(b, axis=1)[nz]
    glob = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
    return per, glob


@pytest.mark.parametrize("kw", [dict(alpha_mode="fixed", alpha=0.01),
                                dict(alpha_mode="alpha-ratio", alpha_ratio=0.05),
                                dict(alpha_mode="fixed", alpha=0.01, non_negative=True)])
def test_mixed_matches_oracle(ph, oracle, kw):
    mix = fit(ph, "mixed", **kw)
    ref = oracle_fit(ph, oracle, **kw)
    per, glob = errors(mix["coef64"], ref["coef64"])
    assert per.max() <= 1e-5, per.max()
    assert glob <= 1e-6, glob
    it_m = mix["iterations"][ph.mask].astype(int)
    it_o = ref["iterations"][ph.mask].astype(int)
    assert np.mean(it_m == it_o) >= 0.99
    assert np.abs(it_m - it_o).max() <= 1
    np.testing.assert_allclose(mix["r2"], ref["r2"], rtol=0, atol=1e-6)


def test_mixed_matches_fp64_gpu_and_reports_tensor_work(ph):
    from cs_dmri_b200 import _abi
    f64 = fit(ph, "fp64", alpha_mode="fixed", alpha=0.01)
    mix = fit(ph, "mixed", alpha_mode="fixed", alpha=0.01)
    t = _abi.last_timing(0)
    assert t.int8_tensor_ops > 0 and t.ms_mixed_kernel > 0
    # each voxel-iteration is one row of a 36-MMA (128 x 80 x 32) batch
    assert t.int8_tensor_ops >= mix["total_iterations"] * 36 * 2 * 80 * 32 * 0.99
    assert t.fp64_rerun_voxels <= 0.2 * ph.n_voxels
    per, glob = errors(mix["coef64"], f64["coef64"])
    assert per.max() <= 1e-5 and glob <= 1e-6, (per.max(), glob)


@pytest.mark.parametrize("mode", ["path-bic", "l2-anchored"])
def test_mixed_warm_started_paths(ph, oracle, mode):
    """Path strategies warm-start every fit from the previous alpha's answer:
    the mixed kernel forms u_0 = G x_warm - b through the same digit products."""
    mix = fit(ph, "mixed", alpha_mode=mode)
    ref = oracle_fit(ph, oracle, alpha_mode=mode)
    same_alpha = np.isclose(mix["alpha"][ph.mask], ref["alpha"][ph.mask], rtol=1e-12, atol=0)
    assert same_alpha.mean() >= 0.99
    per, _ = errors(mix["coef64"][same_alpha], ref["coef64"][same_alpha])
    assert per.max() <= 1e-5, per.max()


def test_mixed_partial_mask_and_tail_tiles(ph, oracle):
    """A mask whose voxel count is not a multiple of the 128-voxel tile."""
    mask = ph.mask.copy()
    mask.ravel()[::3] = False
    mask.ravel()[5] = True
    mix = fit(ph, "mixed", mask=mask, alpha_mode="fixed", alpha=0.01)
    ref = oracle_fit(ph, oracle, mask=mask, alpha_mode="fixed", alpha=0.01)
    assert mix["n_voxels"] == int(mask.sum())
    assert np.all(mix["coefficients"][~mask] == 0)
    per, _ = errors(mix["coef64"], ref["coef64"])
    assert per.max() <= 1e-5


def test_mixed_nan_voxel_semantics(ph, oracle):
    from cs_dmri_b200 import shore_fit
    data = ph.data.copy()
    data[1, 1, 1, 3] = np.nan
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, diagnostics=True, alpha_mode="fixed",
              alpha=0.01)
    mix = shore_fit(data, ph.bvals, ph.bvecs, ph.mask, precision="mixed", **kw)
    ref = oracle.shore_fit(data, ph.bvals, ph.bvecs, ph.mask, **kw)
    np.testing.assert_array_equal(mix["coefficients"][1, 1, 1], ref["coefficients"][1, 1, 1])
    assert mix["iterations"][1, 1, 1] == ref["iterations"][1, 1, 1]


def test_mixed_precision_arguments(ph):
    with pytest.raises(ValueError, match="radial order 6"):
        fit(ph, "mixed", radial_order=4, alpha_mode="fixed", alpha=0.01)
    with pytest.raises(ValueError, match="precision"):
        fit(ph, "bf16", alpha_mode="fixed", alpha=0.01)
    # L2 has no FISTA iterations: the precision switch leaves it unchanged
    a = fit(ph, "mixed", regularization="l2", lambda_n=0.05, lambda_l=0.05)
    b = fit(ph, "fp64", regularization="l2", lambda_n=0.05, lambda_l=0.05)
    np.testing.assert_array_equal(a["coefficients"], b["coefficients"])


def test_mixed_larger_volume_against_fp64_gpu():
    """4,000 voxels (the 20 x 20 x 10 grid): whole-volume error and tail."""
    from cs_dmri_b200.phantom import make_phantom
    p = make_phantom((20, 20, 10), seed=1)
    f64 = fit(p, "fp64", alpha_mode="fixed", alpha=0.01)
    mix = fit(p, "mixed", alpha_mode="fixed", alpha=0.01)
    per, glob = errors(mix["coef64"], f64["coef64"])
    assert glob <= 1e-6, glob
    assert per.max() <= 1e-5, per.max()
    assert np.percentile(per, 99) <= 1e-6


def test_two_pass_schedule_changes_nothing_in_the_mixed_path():
    """The mixed kernel's two-pass schedule parks a voxel's x, d, u rows and
    guard flag at iteration 80 and resumes them slowest-first: coefficients,
    iteration counts, convergence flags and the voxels re-run in FP64 are
    those of a single pass (handle option CSD_OPT_FISTA_SCHEDULE = 0)."""
    from cs_dmri_b200 import _abi, shore_fit
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((64, 64, 50), seed=31)  # 204,800 voxels: two passes
    V = int(ph.mask.sum())
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01,
              precision="mixed", return_coef64=True, diagnostics=True)
    two = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    t2 = _abi.last_timing(0)
    assert 0.5 * V < t2.fista_parked <= V
    _abi.set_option(_abi.OPT_FISTA_SCHEDULE, 0)
    try:
        one = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
        t1 = _abi.last_timing(0)
    finally:
        _abi.set_option(_abi.OPT_FISTA_SCHEDULE, 1)
    assert t1.fista_parked == 0
    assert t1.fp64_rerun_voxels == t2.fp64_rerun_voxels
    for k in ("coef64", "coefficients", "iterations", "converged"):
        np.testing.assert_array_equal(two[k], one[k])
    assert two["total_iterations"] == one["total_iterations"]


@pytest.mark.parametrize("precision", ["mixed", "mixed-kkt"])
def test_tensor_core_wait_gives_up_and_the_handle_recovers(ph, precision):
    """The tensor-core kernels bound every wait for their products.  With the
    limit set to 1 ns (handle option CSD_OPT_TENSOR_WAIT_NS) the first wait
    gives up: the kernel flags the error, lets the products in flight land,
    frees its tensor memory and returns, and the call reports CSD_ERR_TIMEOUT
    (status 5).  The next fit on the same handle succeeds and equals a fit
    that never timed out."""
    from cs_dmri_b200 import _abi
    kw = dict(alpha_mode="fixed", alpha=0.01)
    before = fit(ph, precision, **kw)
    _abi.set_option(_abi.OPT_TENSOR_WAIT_NS, 1)
    try:
        with pytest.raises(_abi.CsdError) as e:
            fit(ph, precision, **kw)
        assert e.value.code == 5 and "gave up" in str(e.value)
    finally:
        _abi.set_option(_abi.OPT_TENSOR_WAIT_NS, 2_000_000_000)
    after = fit(ph, precision, **kw)
    for k in ("coef64", "coefficients", "iterations", "converged"):
        np.testing.assert_array_equal(before[k], after[k])
