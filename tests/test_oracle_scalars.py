"""The oracle's SHORE post-fit maps (predict, ODF SH, microstructure scalars)
pinned by the reference's own tests: the unit KATs of
src/scalars/microstructure.rs:318-361 and io/microstructure.rs:620-645, and the
single-tensor ground-truth integration tests of tests/scalars.rs (a Tikhonov
fit of an analytic tensor signal on a dense multi-shell table, scalars within
the reference's ratio tolerances of the closed forms)."""

import math

import numpy as np
import pytest


def dense_multishell():
    """1 b0 + 4 shells (b = 1000..4000) x 64 golden-spiral directions
    (tests/scalars.rs:26-43)."""
    bvals, bvecs = [0.0], [[0.0, 0.0, 0.0]]
    phi = math.pi * (3.0 - math.sqrt(5.0))
    for b in (1000.0, 2000.0, 3000.0, 4000.0):
        for k in range(64):
            t = (k + 0.5) / 64
            z = 1.0 - 2.0 * t
            r = math.sqrt(max(1.0 - z * z, 0.0))
            a = phi * k
            v = np.array([math.cos(a) * r, math.sin(a) * r, z])
            bvals.append(b)
            bvecs.append(list(v / max(np.linalg.norm(v), 1e-12)))
    return np.array(bvals), np.array(bvecs)


BIG, SMALL = 0.0431, 0.0107
TAU = BIG - SMALL / 3.0


def tensor_fit(oracle, evals):
    bvals, bvecs = dense_multishell()
    adc = bvecs ** 2 @ np.asarray(evals)
    s = np.exp(-bvals * adc)
    M = oracle.design_matrix(bvals, bvecs, 6, 700.0, big_delta=BIG, small_delta=SMALL)
    nd, ld = oracle.regularization(6)
    c, _ = oracle.tikhonov_fit(M, s, nd, ld, 1e-6, 1e-6)
    return c


def truth(l1, l2, l3, tau):
    rtpp = 1.0 / (2.0 * math.sqrt(math.pi * l1 * tau))
    rtap = 1.0 / (2.0 * math.sqrt(math.pi * l2 * tau)) / (2.0 * math.sqrt(math.pi * l3 * tau))
    return dict(rtop=rtpp * rtap, rtap=rtap, rtpp=rtpp, msd=2.0 * (l1 + l2 + l3) * tau)


def close(a, b, tol):
    return math.isfinite(a) and abs(a - b) / abs(b) <= tol


def test_ng_zero_for_pure_gaussian(oracle):
    c = np.zeros(oracle.n_coeffs(4))
    c[0] = 1.0
    assert abs(oracle.microstructure_voxel(c, 4, 700.0)["ng"]) <= 1e-12


def test_alpha_factor_n0_l0(oracle):
    want = math.sqrt(2.0 * math.pi * 700.0 ** 1.5 * math.gamma(1.5))
    assert abs(oracle.micro_alpha_factor(0, 0, 700.0) - want) <= 1e-9


def test_rtap_rtpp_nan_without_direction(oracle):
    c = np.ones(oracle.n_coeffs(4))
    v = oracle.microstructure_voxel(c, 4, 700.0, [0.0, 0.0, 0.0])
    assert math.isnan(v["rtap"]) and math.isnan(v["rtpp"])
    v = oracle.microstructure_voxel(c, 4, 700.0, None)
    assert math.isnan(v["rtap"])


def test_isotropic_tensor_rtop_msd(oracle):
    d = 0.7e-3
    v = oracle.microstructure_voxel(tensor_fit(oracle, [d, d, d]), 6, 700.0)
    t = truth(d, d, d, TAU)
    assert close(v["rtop"], t["rtop"], 0.10), (v["rtop"], t["rtop"])
    assert close(v["msd"], t["msd"], 0.10), (v["msd"], t["msd"])


def test_anisotropic_tensor_rtap_rtpp(oracle):
    l1, l2, l3 = 1.7e-3, 0.3e-3, 0.3e-3
    v = oracle.microstructure_voxel(tensor_fit(oracle, [l1, l2, l3]), 6, 700.0, [1.0, 0.0, 0.0])
    t = truth(l1, l2, l3, TAU)
    assert close(v["rtop"], t["rtop"], 0.15)
    assert close(v["msd"], t["msd"], 0.20)
    assert close(v["rtap"], t["rtap"], 0.30)
    assert close(v["rtpp"], t["rtpp"], 0.20)


@pytest.fixture(scope="module")
def coef_volume():
    from cs_dmri_b200.phantom import make_phantom
    from oracle import oracle as O
    ph = make_phantom((5, 4, 3), seed=4)
    mask = ph.mask.copy()
    mask[0, 0, :] = False
    out = O.shore_fit(ph.data, ph.bvals, ph.bvecs, mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                      regularization="l2", lambda_n=0.05, lambda_l=0.05)
    return ph, mask, out["coefficients"]


def test_predict_is_the_design_product(oracle, coef_volume):
    ph, mask, c = coef_volume
    out = oracle.shore_predict(c, 6, 700.0, ph.bvals, ph.bvecs, big_delta=ph.big_delta,
                               small_delta=ph.small_delta)
    M = oracle.design_matrix(ph.bvals, ph.bvecs, 6, 700.0, big_delta=ph.big_delta, small_delta=ph.small_delta)
    want = (c.astype(np.float64) @ M.T).astype(np.float32)
    np.testing.assert_allclose(out, want, rtol=2e-7, atol=1e-6)
    assert np.all(out[~mask] == 0)  # all-zero coefficient voxels are skipped


def test_odf_sh_is_the_projection(oracle, coef_volume):
    ph, mask, c = coef_volume
    for lmax in (0, 2, 4, 6):
        out = oracle.shore_odf_sh(c, 6, 700.0, lmax, mask)
        P = np.zeros(((lmax + 1) * (lmax + 2) // 2, oracle.n_coeffs(6)))
        oracle.lib().oracle_shore_to_tournier(6, 700.0, lmax, P.ctypes.data)
        want = (c.astype(np.float64) @ P.T).astype(np.float32)
        want[~mask] = 0
        np.testing.assert_allclose(out, want, rtol=2e-7, atol=1e-6)


def test_outlier_rule_and_units(oracle, coef_volume):
    """Rejection = NaN every finite value strictly above factor x nearest-rank
    p99 of the finite values (io/microstructure.rs:222-270, 303-326); um
    scaling multiplies the f32 value by the f32 unit factor."""
    ph, mask, c = coef_volume
    rng = np.random.default_rng(3)
    dirs = rng.normal(size=c.shape[:3] + (3,)).astype(np.float32)
    dirs[1, 1, 1] = 0.0
    raw = oracle.shore_microstructure(c, 6, 700.0, mask, dirs, units="mm", outlier_factor=None)
    um = oracle.shore_microstructure(c, 6, 700.0, mask, dirs, units="um", outlier_factor=None)
    scale = dict(rtop=np.float32(1e-9), rtap=np.float32(1e-6), rtpp=np.float32(1e-3), msd=np.float32(1e6),
                 qiv=np.float32(1e15), ng=np.float32(1.0))
    for k, s in scale.items():
        np.testing.assert_array_equal(um[k][mask], raw[k][mask] * s)
        assert np.all(raw[k][~mask] == 0)
    assert np.isnan(raw["rtap"][1, 1, 1]) and np.isnan(raw["rtpp"][1, 1, 1])
    for factor in (10.0, 1.0001):
        rej = oracle.shore_microstructure(c, 6, 700.0, mask, dirs, units="mm", outlier_factor=factor)
        for k in scale:
            v = raw[k][mask].copy()
            fin = v[np.isfinite(v)]
            if fin.size:
                f = np.sort(fin)
                p99 = f[min(int(math.floor(0.99 * (f.size - 1) + 0.5)), f.size - 1)]
                thr = np.float32(factor) * p99
                v[np.isfinite(v) & (v > thr)] = np.nan
            np.testing.assert_array_equal(rej[k][mask], v)
