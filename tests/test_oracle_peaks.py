"""The oracle's ODF sampling, GFA and peak finder (oracle.odf_peaks) on
analytic tensor signals: a Tikhonov fit (tiny weights) of a single tensor
along u has one peak within the sphere's vertex spacing of u; a 90-degree
crossing of two equal tensors has two peaks near the two axes; an isotropic
signal has GFA ~ 0.  The reference's own finder (odx-rs) is not in the
repository, so these are the pins."""

import math

import numpy as np
import pytest

from tests.test_oracle_scalars import dense_multishell


@pytest.fixture(scope="module")
def design(oracle):
    bvals, bvecs = dense_multishell()
    M = oracle.design_matrix(bvals, bvecs, 6, 700.0, big_delta=0.0431, small_delta=0.0107)
    nd, ld = oracle.regularization(6)
    return bvals, bvecs, M, nd, ld


def tensor_signal(bvals, bvecs, u, lam=(1.7e-3, 0.2e-3)):
    u = np.asarray(u, float) / np.linalg.norm(u)
    return np.exp(-bvals * (lam[1] + (lam[0] - lam[1]) * (bvecs @ u) ** 2))


def angle(a, b):
    return math.degrees(math.acos(min(1.0, abs(float(np.dot(a, b))))))


def test_mesh(oracle):
    for f in (1, 2, 6):
        v, e, h = oracle.geodesic_mesh(f)
        assert len(v) == 10 * f * f + 2 and len(e) == 30 * f * f
        deg = np.bincount(e.ravel(), minlength=len(v))
        assert (deg == 5).sum() == 12 and np.all((deg == 5) | (deg == 6))
        assert h.max() + 1 == len(v) // 2 and np.all(np.bincount(h) == 2)


@pytest.mark.parametrize("u", [(1, 0, 0), (0, 0.6, 0.8), (0.3, -0.4, 0.866)])
def test_single_fibre_peak(oracle, design, u):
    bvals, bvecs, M, nd, ld = design
    c, _ = oracle.tikhonov_fit(M, tensor_signal(bvals, bvecs, u), nd, ld, 1e-6, 1e-6)
    gfa, D, V, qa, amp = oracle.odf_peaks(c, 6, 700.0, npeaks=3)
    assert angle(D[0], np.asarray(u) / np.linalg.norm(u)) < 6.0  # vertex spacing of the frequency-6 sphere
    assert V[0] > 0 and np.all(V[1:] == 0) and gfa > 0.3
    assert qa[0] == pytest.approx(V[0] - amp.min())


def test_crossing_has_two_peaks(oracle, design):
    bvals, bvecs, M, nd, ld = design
    a, b = np.array([1.0, 0, 0]), np.array([0, 1.0, 0])
    s = 0.5 * tensor_signal(bvals, bvecs, a, (2.2e-3, 0.1e-3)) + 0.5 * tensor_signal(bvals, bvecs, b, (2.2e-3, 0.1e-3))
    c, _ = oracle.tikhonov_fit(M, s, nd, ld, 1e-6, 1e-6)
    gfa, D, V, qa, amp = oracle.odf_peaks(c, 6, 700.0, npeaks=3)
    assert V[1] > 0.5 * V[0]
    found = sorted([min(angle(D[i], a), angle(D[i], b)) for i in range(2)])
    assert found[1] < 8.0
    assert angle(D[0], D[1]) > 80.0


def test_isotropic_gfa_zero(oracle, design):
    bvals, bvecs, M, nd, ld = design
    c, _ = oracle.tikhonov_fit(M, np.exp(-bvals * 1e-3), nd, ld, 1e-6, 1e-6)
    gfa, D, V, qa, amp = oracle.odf_peaks(c, 6, 700.0)
    assert gfa < 1e-3
