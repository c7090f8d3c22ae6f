"""Per-voxel-design fit on the GPU (csd_shore_fit_graddev_device) against the
oracle: the effective table of each voxel's deviation tensor, its kept
samples, the design of those rows and the reference FISTA (oracle.graddev_fit),
at radial orders 8 (the workload's) and 6.

Tolerances as for the shared-design fit: coefficients within 1e-5 of the
largest coefficient (a stopping decision within rounding of tol can move the
iterate by tol x |x|), iteration counts within 1; the Lipschitz constant
sigma_max(M_v)^2 / n_v (Lanczos on G_v against the oracle's Jacobi
eigensolve) at 1e-12.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def inputs():
    from cs_dmri_b200.graddev import graddev_phantom
    return graddev_phantom(96, seed=7)


@pytest.mark.parametrize("order", [8, 6])
def test_matches_oracle(oracle, inputs, order):
    from cs_dmri_b200.graddev import shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = inputs
    out = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.01, radial_order=order, big_delta=big,
                            small_delta=small)
    c = out["coefficients"].cpu().numpy()
    it = out["iterations"].cpu().numpy()
    lip = out["lipschitz"].cpu().numpy()
    assert np.array_equal(out["n_samples"].cpu().numpy(), keep.sum(1))
    off = 0
    for v in range(0, len(S), 3):
        want, wit, wconv, M = oracle.graddev_fit(S[v], bvals, bvecs, T[v], keep[v], 0.01, radial_order=order,
                                                 big_delta=big, small_delta=small)
        np.testing.assert_allclose(lip[v], oracle.sigma_max(M) ** 2 / M.shape[0], rtol=1e-12)
        np.testing.assert_allclose(c[v], want, rtol=0, atol=1e-5 * np.abs(want).max())
        assert abs(int(it[v]) - wit) <= 1
        off += int(it[v]) != wit
    assert off <= 2


def test_identity_matches_the_shared_design_fit(inputs):
    import torch
    from cs_dmri_b200.autograd import DifferentiableShore
    from cs_dmri_b200.graddev import shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = inputs
    out = shore_fit_graddev(S, bvals, bvecs, None, None, alpha=0.01, radial_order=6, big_delta=big,
                            small_delta=small)
    m = DifferentiableShore(bvals, bvecs, big_delta=big, small_delta=small)
    ref = m.fit(torch.from_numpy(S).cuda(), 0.01).cpu().numpy()
    c = out["coefficients"].cpu().numpy()
    scale = np.abs(ref).max(1, keepdims=True)
    assert np.all(np.abs(c - ref) <= 1e-5 * scale)


def test_per_voxel_alpha_and_edge_cases(inputs):
    import torch
    from cs_dmri_b200.graddev import shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = inputs
    kw = dict(radial_order=6, big_delta=big, small_delta=small)
    a = np.where(np.arange(len(S)) % 2 == 0, 0.01, 0.05)
    both = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=a, **kw)["coefficients"].cpu().numpy()
    one = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.01, **kw)["coefficients"].cpu().numpy()
    five = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.05, **kw)["coefficients"].cpu().numpy()
    np.testing.assert_array_equal(both[0::2], one[0::2])
    np.testing.assert_array_equal(both[1::2], five[1::2])
    none = np.zeros_like(keep)
    out = shore_fit_graddev(S[:4], bvals, bvecs, T[:4], none[:4], alpha=0.01, **kw)
    assert float(out["coefficients"].abs().max()) == 0.0
    assert int(out["iterations"].max()) == 0 and not bool(out["converged"].any())
    with pytest.raises(ValueError, match="radial orders 6 and 8"):
        shore_fit_graddev(S[:4], bvals, bvecs, radial_order=4, big_delta=big, small_delta=small)
    with pytest.raises(ValueError, match="sample_mask"):
        shore_fit_graddev(S[:4], bvals, bvecs, sample_mask=keep[:3], big_delta=big, small_delta=small)
    assert torch.cuda.is_available()


@pytest.mark.parametrize("precision", ["fp64-kkt", "mixed-kkt"])
@pytest.mark.parametrize("order", [8, 6])
def test_certified_optimum_per_voxel_design(oracle, inputs, order, precision):
    """precision "fp64-kkt" / "mixed-kkt" on per-voxel designs: the support
    from 32 FISTA iterations (FP64, or FP32 on the hi plane of G_v), the polish
    on the voxel's own Gram matrix (FP64, or FP64 on hi + lo), the
    certificate.  Against the oracle's optimum of each voxel - the exact solve
    on the support and signs of the oracle's reference-rule fit on the same
    design, kept where its KKT conditions certify it - at per-voxel relative
    L2 <= 1e-6, every voxel certified."""
    from cs_dmri_b200 import _abi
    from cs_dmri_b200.graddev import shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = inputs
    out = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.01, radial_order=order, big_delta=big,
                            small_delta=small, precision=precision)
    t = _abi.last_timing(0)
    c = out["coefficients"].cpu().numpy()
    assert bool(out["converged"].all()) and t.kkt_uncertified == 0 and t.kkt_iterations == 32
    checked = 0
    for v in range(0, len(S), 2):
        c0, _, _, M = oracle.graddev_fit(S[v], bvals, bvecs, T[v], keep[v], 0.01, radial_order=order,
                                         big_delta=big, small_delta=small)
        s_v = np.asarray(S[v], np.float64)[keep[v]]
        want, ok = oracle.lasso_polish(M, s_v, 0.01, c0, margin=0.0)
        if not ok:
            continue
        checked += 1
        assert np.linalg.norm(c[v] - want) <= 1e-6 * max(np.linalg.norm(want), 1e-300), v
    assert checked >= 0.9 * len(range(0, len(S), 2))


@pytest.mark.parametrize("order", [8, 6])
def test_mixed_kkt_per_voxel_design_against_fp64_kkt(inputs, order):
    """precision "mixed-kkt" on per-voxel designs keeps G_v as FP32 planes
    hi + lo and runs the Lanczos estimate and the support iterations in FP32;
    the polish certifies the same optimum as "fp64-kkt" (per-voxel relative
    L2 <= 1e-6, every voxel certified, Lipschitz estimates within 1e-5).
    Precision "mixed" (the int8 path of the shared design) is refused."""
    from cs_dmri_b200.graddev import shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = inputs
    kw = dict(alpha=0.01, radial_order=order, big_delta=big, small_delta=small)
    a = shore_fit_graddev(S, bvals, bvecs, T, keep, precision="fp64-kkt", **kw)
    b = shore_fit_graddev(S, bvals, bvecs, T, keep, precision="mixed-kkt", **kw)
    assert bool(a["converged"].all()) and bool(b["converged"].all())
    ca, cb = a["coefficients"].cpu().numpy(), b["coefficients"].cpu().numpy()
    rel = np.linalg.norm(ca - cb, axis=1) / np.maximum(np.linalg.norm(ca, axis=1), 1e-300)
    assert rel.max() <= 1e-6, rel.max()
    la, lb = a["lipschitz"].cpu().numpy(), b["lipschitz"].cpu().numpy()
    assert np.abs(la - lb).max() <= 1e-5 * la.max()
    with pytest.raises(Exception, match="precision fp64, fp64-kkt or mixed-kkt"):
        shore_fit_graddev(S, bvals, bvecs, T, keep, precision="mixed", **kw)


def test_certified_support_iterations_autotuned():
    """A certified per-voxel-design call of at least four tuning prefixes (24
    voxels per SM each) picks the support-iteration count by timing 16, 24, 32
    and 48 on its own first voxels, once per table, order and mode; a later
    call takes the cached count.  The fit ends at the certified optimum
    whatever the count: the same coefficients (1e-9) as a forced count of 32."""
    import torch

    from cs_dmri_b200 import _abi
    from cs_dmri_b200.graddev import graddev_phantom, shore_fit_graddev
    n = 4 * 24 * torch.cuda.get_device_properties(0).multi_processor_count + 16
    S, bvals, bvecs, T, keep, big, small = graddev_phantom(n, seed=9)
    kw = dict(alpha=0.01, radial_order=6, big_delta=big, small_delta=small, precision="mixed-kkt")
    _abi.set_option(_abi.OPT_KKT_ITERATIONS, 32)
    try:
        forced = shore_fit_graddev(S, bvals, bvecs, T, keep, **kw)
    finally:
        _abi.set_option(_abi.OPT_KKT_ITERATIONS, 0)
    tuned = shore_fit_graddev(S, bvals, bvecs, T, keep, **kw)
    t = _abi.last_timing(0)
    assert t.kkt_iterations in (16, 24, 32, 48) and min(t.kkt_tune_ms) > 0.0
    assert t.kkt_uncertified == 0 and bool(tuned["converged"].all())
    again = shore_fit_graddev(S, bvals, bvecs, T, keep, **kw)
    t2 = _abi.last_timing(0)
    assert t2.kkt_iterations == t.kkt_iterations and list(t2.kkt_tune_ms) == list(t.kkt_tune_ms)
    a, b = forced["coefficients"].cpu().numpy(), tuned["coefficients"].cpu().numpy()
    rel = np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(a, axis=1), 1e-300)
    assert rel.max() <= 1e-9, rel.max()
    assert np.array_equal(b, again["coefficients"].cpu().numpy())
