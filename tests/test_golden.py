"""The oracle against external golden vectors: the reference's eight
scikit-learn LASSO fixtures (tests/optimization_sklearn.rs, same tolerances)
and scikit-learn golds on the real SHORE design (tests/golden/make_golden.py)."""

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def lasso_objective(M, y, b, alpha):  # tests/common/mod.rs:109-115
    r = M @ b - y
    return 0.5 / M.shape[0] * r @ r + alpha * np.abs(b).sum()


def kkt(M, y, b, alpha, positive):  # tests/common/mod.rs:117-189
    g = M.T @ (M @ b - y) / M.shape[0]
    act = np.abs(b) > 1e-10 if not positive else b > 1e-10
    if positive:
        a = np.abs(g[act] + alpha).max(initial=0.0)
        i = np.maximum(-g[~act] - alpha, 0).max(initial=0.0)
    else:
        a = np.abs(g[act] + alpha * np.sign(b[act])).max(initial=0.0)
        i = np.maximum(np.abs(g[~act]) - alpha, 0).max(initial=0.0)
    return a, i


def fixtures():
    z = np.load(GOLDEN / "lasso_fixtures.npz")
    return [(str(n), {k.split("__")[1]: z[k] for k in z.files if k.startswith(f"{n}__")})
            for n in z["__names__"]]


@pytest.mark.parametrize("name,fx", fixtures(), ids=[n for n, _ in fixtures()])
def test_oracle_matches_sklearn_lasso_fixture(oracle, name, fx):
    M, y, alpha, pos = fx["design"], fx["signal"], float(fx["alpha"]), bool(fx["positive"])
    coef, it, conv, _ = oracle.fista_fit(M, y, alpha, 200_000, 1e-12, pos)
    ref = fx["coef"]
    assert np.linalg.norm(coef - ref) / max(1.0, np.linalg.norm(ref)) < 1e-3
    obj = lasso_objective(M, y, coef, alpha)
    assert abs(obj - float(fx["objective"])) / max(1.0, abs(float(fx["objective"]))) < 1e-6
    a, i = kkt(M, y, coef, alpha, pos)
    assert a < 1e-5 and i < 1e-5
    assert abs(oracle.alpha_max(M, y) - float(fx["alpha_max"])) <= 1e-12 * float(fx["alpha_max"])


@pytest.mark.parametrize("alpha", [0.5, 2.0])
def test_oracle_matches_sklearn_on_shore_design(oracle, alpha):
    z = np.load(GOLDEN / "shore_lasso.npz")
    M, S = z["design"], z["signals"]
    for s, ref, obj_ref in zip(S, z[f"coef_a{alpha}"], z[f"obj_a{alpha}"]):
        coef, *_ = oracle.fista_fit(M, s, alpha, 400_000, 1e-13)
        obj = lasso_objective(M, s, coef, alpha)
        # the minimum is pinned by the objective; coefficients to the LASSO tolerance
        assert abs(obj - obj_ref) / abs(obj_ref) < 1e-6
        assert np.linalg.norm(coef - ref) / max(1.0, np.linalg.norm(ref)) < 1e-3
