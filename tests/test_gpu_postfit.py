"""Post-fit maps on the GPU against the oracle: predicted signal on a new
gradient table (synth.rs), ODF SH projection (odf.rs) and the microstructure
scalars (scalars/microstructure.rs, io/microstructure.rs).

Tolerance.  Every map is an FP64 computation rounded to float32 at the end,
as in the reference; the GPU evaluates the same operations in the same order
but its transcendental functions (pow, atan2, acos, the Lanczos Gamma built on
them) may differ from the host's by an ulp of FP64, which can move a float32
result by one ulp.  Values are compared at 1e-6 relative, NaN patterns and
exact zeros exactly.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vol(oracle):
    from cs_dmri_b200 import shore_fit
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((9, 7, 5), seed=11)
    mask = ph.mask.copy()
    mask[0, :, :] = False
    mask[3, 3, 2] = False
    c = shore_fit(ph.data, ph.bvals, ph.bvecs, mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                  regularization="l2", lambda_n=0.05, lambda_l=0.05)["coefficients"]
    return ph, mask, c


def test_predict_matches_oracle(vol, oracle):
    from cs_dmri_b200 import shore_predict
    from cs_dmri_b200.gradients import GradientTable  # noqa: F401  (API surface)
    ph, mask, c = vol
    rng = np.random.default_rng(5)
    # a new table: the phantom's directions on different shells, with a b0
    bvals = np.concatenate([[0.0], rng.uniform(200, 4000, 40)])
    v = rng.normal(size=(41, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v[0] = 0.0
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta)
    got = shore_predict(c, 6, 700.0, bvals, v, **kw)
    want = oracle.shore_predict(c, 6, 700.0, bvals, v, **kw)
    assert got.shape == want.shape == c.shape[:3] + (41,)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6 * np.abs(want).max())
    assert np.all(got[~mask] == 0)


def test_predict_on_the_fit_table_reproduces_the_fit(vol):
    from cs_dmri_b200 import shore_fit, shore_predict
    ph, mask, _ = vol
    out = shore_fit(ph.data, ph.bvals, ph.bvecs, mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                    regularization="l2", lambda_n=0.05, lambda_l=0.05, diagnostics=True)
    s = shore_predict(out["coefficients"], 6, 700.0, ph.bvals, ph.bvecs, big_delta=ph.big_delta,
                      small_delta=ph.small_delta)
    resid = np.linalg.norm(ph.data[mask] - s[mask], axis=1)
    np.testing.assert_allclose(resid, out["residual_l2"][mask], rtol=1e-4)


@pytest.mark.parametrize("lmax", [0, 2, 4, 6])
def test_odf_sh_matches_oracle(vol, oracle, lmax):
    from cs_dmri_b200 import shore_odf_sh
    ph, mask, c = vol
    for m in (mask, None):
        got = shore_odf_sh(c, 6, 700.0, lmax, m)
        want = oracle.shore_odf_sh(c, 6, 700.0, lmax, m)
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6 * max(np.abs(want).max(), 1e-30))
        if m is not None:
            assert np.all(got[~m] == 0)


@pytest.mark.parametrize("units,factor", [("um", 10.0), ("mm", None), ("mm", 1.0001)])
def test_microstructure_matches_oracle(vol, oracle, units, factor):
    from cs_dmri_b200 import shore_microstructure
    ph, mask, c = vol
    rng = np.random.default_rng(9)
    dirs = rng.normal(size=c.shape[:3] + (3,)).astype(np.float32)
    dirs[1, 1, 1] = 0.0
    dirs[2, 2, 2, 1] = np.nan
    got = shore_microstructure(c, 6, 700.0, mask, dirs, units=units, outlier_factor=factor)
    want = oracle.shore_microstructure(c, 6, 700.0, mask, dirs, units=units, outlier_factor=factor)
    for k in ("rtop", "rtap", "rtpp", "msd", "qiv", "ng"):
        g, w = got[k], want[k]
        np.testing.assert_array_equal(np.isnan(g), np.isnan(w), err_msg=k)
        fin = np.isfinite(w)
        np.testing.assert_allclose(g[fin], w[fin], rtol=1e-6, atol=0, err_msg=k)
        assert np.all(g[~mask] == 0), k
    assert np.isnan(got["rtap"][1, 1, 1]) and np.isnan(got["rtpp"][2, 2, 2])


def test_microstructure_without_directions(vol, oracle):
    from cs_dmri_b200 import shore_microstructure
    ph, mask, c = vol
    got = shore_microstructure(c, 6, 700.0, mask)
    assert np.all(np.isnan(got["rtap"][mask])) and np.all(np.isnan(got["rtpp"][mask]))
    want = oracle.shore_microstructure(c, 6, 700.0, mask)
    np.testing.assert_allclose(got["rtop"][mask], want["rtop"][mask], rtol=1e-6)


def test_postfit_argument_errors(vol):
    from cs_dmri_b200 import shore_microstructure, shore_odf_sh, shore_predict
    ph, mask, c = vol
    with pytest.raises(ValueError, match="lmax must be even"):
        shore_odf_sh(c, 6, 700.0, 5)
    with pytest.raises(ValueError, match="lmax must be even"):
        shore_odf_sh(c, 6, 700.0, 8)
    with pytest.raises(ValueError, match="channels but a radial-order-4"):
        shore_odf_sh(c, 4, 700.0, 4)
    with pytest.raises(ValueError, match="channels"):
        shore_predict(c[..., :50], 6, 700.0, ph.bvals, ph.bvecs)
    with pytest.raises(ValueError, match="units must be"):
        shore_microstructure(c, 6, 700.0, mask, units="nm")
    with pytest.raises(ValueError, match="mask does not match"):
        shore_microstructure(c, 6, 700.0, mask[:-1])


def test_shore_fit_methods(vol, oracle):
    """ShoreFit.odf_sh / predict / microstructure (python/cs_dmri/shore.py:152-205)."""
    from cs_dmri_b200 import ShoreModel, shore_odf_sh
    from cs_dmri_b200.gradients import GradientTable
    ph, mask, _ = vol
    gt = GradientTable(ph.bvals, ph.bvecs, big_delta=ph.big_delta, small_delta=ph.small_delta)
    fit = ShoreModel(gt, regularization="l2", lambda_n=0.05, lambda_l=0.05).fit(ph.data, mask)
    np.testing.assert_array_equal(fit.odf_sh(), shore_odf_sh(fit.coefficients, 6, 700.0, 6, mask))
    s = fit.predict()
    assert s.shape == ph.data.shape and s.min() >= 0
    raw = fit.predict(clip=False)
    np.testing.assert_array_equal(s, np.maximum(raw, 0))
    maps = fit.microstructure()
    want = oracle.shore_microstructure(fit.coefficients, 6, 700.0, mask)
    np.testing.assert_allclose(maps["msd"][mask], want["msd"][mask], rtol=1e-6)
