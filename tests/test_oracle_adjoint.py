"""The oracle's derivatives of the fit, pinned by finite differences.

The reference computes no derivatives, so there is no golden vector: the
oracle's implicit-function adjoints (oracle.l1_adjoint, oracle.l2_adjoint) are
checked against central differences of the solution maps themselves - the
exact LASSO minimiser (the oracle's FISTA run to 1e-13 and polished on its
support, with a KKT certificate) and the Tikhonov solve - and the sphere and
ODF helpers against their defining properties."""

import numpy as np
import pytest

ALPHA = 0.01


@pytest.fixture(scope="module")
def problem(oracle):
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((5, 5, 4), seed=8)
    M = oracle.design_matrix(ph.bvals, ph.bvecs, 6, 700.0, big_delta=ph.big_delta, small_delta=ph.small_delta)
    S = ph.data[ph.mask][:6].astype(np.float64)
    return M, S


def exact_lasso(oracle, M, s, alpha, warm=None, non_negative=False):
    c, _, conv, _ = oracle.fista_fit(M, s, alpha, max_iter=200000, tol=1e-13, non_negative=non_negative, warm=warm)
    assert conv
    cp, ok = oracle.lasso_polish(M, s, alpha, c, non_negative=non_negative)
    assert ok, "KKT certificate failed"
    return cp


@pytest.mark.parametrize("non_negative", [False, True])
def test_l1_adjoint_matches_finite_differences(oracle, problem, non_negative):
    M, S = problem
    rng = np.random.default_rng(1)
    n = M.shape[0]
    for s in S[:4]:
        c = exact_lasso(oracle, M, s, ALPHA, non_negative=non_negative)
        gc = rng.normal(size=c.size)
        gs, ga, w = oracle.l1_adjoint(M, c, gc)
        assert np.all(w[c == 0] == 0)
        # directional derivative along a random signal direction
        ds = rng.normal(size=s.size) * np.abs(s).mean() * 1e-4
        cp = exact_lasso(oracle, M, s + ds, ALPHA, warm=c, non_negative=non_negative)
        cm = exact_lasso(oracle, M, s - ds, ALPHA, warm=c, non_negative=non_negative)
        assert np.array_equal(cp != 0, c != 0) and np.array_equal(cm != 0, c != 0)
        fd = gc @ (cp - cm) / 2.0
        np.testing.assert_allclose(gs @ ds, fd, rtol=1e-6, atol=1e-12 * np.abs(gc).sum() * np.abs(c).max())
        # alpha
        h = ALPHA * 1e-4
        cp = exact_lasso(oracle, M, s, ALPHA + h, warm=c, non_negative=non_negative)
        cm = exact_lasso(oracle, M, s, ALPHA - h, warm=c, non_negative=non_negative)
        np.testing.assert_allclose(ga, gc @ (cp - cm) / (2 * h), rtol=1e-6)
        assert n == M.shape[0]


def test_l2_adjoint_matches_finite_differences(oracle, problem):
    M, S = problem
    nd, ld = oracle.regularization(6)
    lam_n, lam_l = 0.05, 0.02
    rng = np.random.default_rng(2)
    for s in S[:3]:
        c, _ = oracle.tikhonov_fit(M, s, nd, ld, lam_n, lam_l)
        gc = rng.normal(size=c.size)
        gs, (gn, gl), _ = oracle.l2_adjoint(M, c, gc, nd, ld, lam_n, lam_l)
        ds = rng.normal(size=s.size)
        cp, _ = oracle.tikhonov_fit(M, s + ds, nd, ld, lam_n, lam_l)
        cm, _ = oracle.tikhonov_fit(M, s - ds, nd, ld, lam_n, lam_l)
        np.testing.assert_allclose(gs @ ds, gc @ (cp - cm) / 2, rtol=1e-7)
        for which, g in ((0, gn), (1, gl)):
            lam = [lam_n, lam_l]
            h = lam[which] * 1e-3
            lp, lm = list(lam), list(lam)
            lp[which] += h
            lm[which] -= h
            cp, _ = oracle.tikhonov_fit(M, s, nd, ld, *lp)
            cm, _ = oracle.tikhonov_fit(M, s, nd, ld, *lm)
            np.testing.assert_allclose(g, gc @ (cp - cm) / (2 * h), rtol=1e-5)


def test_polish_refuses_a_wrong_support(oracle, problem):
    M, S = problem
    c = exact_lasso(oracle, M, S[0], ALPHA)
    wrong = c.copy()
    k = np.flatnonzero(c)[0]
    wrong[k] = 0.0  # drop one active coefficient: the certificate must fail
    _, ok = oracle.lasso_polish(M, S[0], ALPHA, wrong)
    assert not ok


@pytest.mark.parametrize("f", [1, 2, 3, 6])
def test_geodesic_sphere(oracle, f):
    v = oracle.geodesic_sphere(f)
    assert v.shape == (10 * f * f + 2, 3)
    np.testing.assert_allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-15)
    # antipodally symmetric: every vertex has its opposite
    d = np.linalg.norm(v[:, None, :] + v[None, :, :], axis=2)
    assert d.min(1).max() < 1e-12
    h = oracle.geodesic_sphere(f, hemisphere=True)
    assert len(h) == len(v) // 2


def test_odf_of_an_isotropic_propagator_is_constant(oracle):
    A = oracle.odf_matrix(oracle.geodesic_sphere(6), 6, 700.0)
    l = oracle.shore_indices(6)[:, 1]
    c = np.where(l == 0, np.linspace(1.0, 2.0, l.size), 0.0)  # only l = 0 terms: isotropic
    odf = A @ c
    np.testing.assert_allclose(odf, odf[0], rtol=1e-6)  # SH values are float32-rounded
