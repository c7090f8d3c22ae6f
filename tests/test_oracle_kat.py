"""Known-answer tests of the CPU oracle, restating the reference's own unit
tests for the SHORE path (math.rs, qspace.rs, basis/shore.rs, odf.rs,
solver/{fista,tikhonov,icls,alpha}.rs).  These pin the oracle before it is
trusted as the checker of the GPU library."""

import math

import numpy as np
import pytest


def test_factorial_and_gamma(oracle):  # src/math.rs:173-185
    assert oracle.factorial(0) == 1.0
    assert oracle.factorial(5) == 120.0
    assert oracle.factorial(10) == 3628800.0
    for n in range(1, 11):
        assert abs(oracle.gamma(n) - oracle.factorial(n - 1)) < 1e-6
    # Lanczos to ~14 digits against the exact Gamma
    for x in (0.7, 1.5, 3.25, 7.5, 12.0):
        assert abs(oracle.gamma(x) - math.gamma(x)) / math.gamma(x) < 1e-13


def test_legendre_known_values(oracle):  # src/math.rs:187-207
    L = oracle.assoc_legendre
    assert abs(L(0, 0, 0.3) - 1.0) < 1e-12
    assert abs(L(1, 0, 0.3) - 0.3) < 1e-12
    assert abs(L(1, 1, 0.3) + math.sqrt(1 - 0.09)) < 1e-12
    assert abs(L(2, 0, 0.4) - 0.5 * (3 * 0.16 - 1)) < 1e-12
    assert abs(L(2, 2, 0.4) - 3 * (1 - 0.16)) < 1e-12


def test_legendre_matches_scipy(oracle):
    from scipy.special import lpmv
    for l in range(0, 9):
        for m in range(0, l + 1):
            for x in (-0.9, -0.2, 0.0, 0.45, 0.99):
                assert abs(oracle.assoc_legendre(l, m, x) - lpmv(m, l, x)) <= 1e-11 * max(1, abs(lpmv(m, l, x)))


def test_hyp2f1_terminating_series(oracle):  # src/math.rs:209-233
    cases = [(0, 0, 1.0), (-2, 0, 1.0), (-4, 0, 1.0), (-6, 0, 1.0), (-2, 2, 3.650793650793651e-1),
             (-4, 2, 2.274392274392287e-1), (-2, 4, 2.167832167832167e-1)]
    for a, ell, expected in cases:
        assert abs(oracle.hyp2f1(a, ell / 2 + 1.5, ell + 1.5, 2.0) - expected) < 1e-12


def test_laguerre_known_values(oracle):  # src/math.rs:235-246
    assert abs(oracle.gen_laguerre(0, 0.5, 0.7) - 1.0) < 1e-12
    assert abs(oracle.gen_laguerre(1, 0.5, 0.7) - (1.0 + 0.5 - 0.7)) < 1e-12
    x, a = 0.7, 0.5
    assert abs(oracle.gen_laguerre(2, a, x) - ((1 + a) * (2 + a) / 2 - (2 + a) * x + x * x / 2)) < 1e-12
    from scipy.special import eval_genlaguerre
    for n in range(0, 9):
        for x in (0.0, 0.3, 2.5, 9.0):
            ref = eval_genlaguerre(n, 1.5, x)
            assert abs(oracle.gen_laguerre(n, 1.5, x) - ref) <= 1e-10 * max(1, abs(ref))


def test_tortoise_deltas(oracle):  # src/qspace.rs:497-513, 601-615
    gyro, gmax = 267.51532e6, 80e-3
    big, small = oracle.tortoise_deltas([0.0, 3000.0], gmax)
    temp = 3000.0 / gyro / gyro / gmax / gmax / 2.0 * 1e6
    small_ms = temp ** (1 / 3) * 1000.0
    assert abs(small - small_ms * 1e-3) < 1e-15
    assert abs(big - 3 * small_ms * 1e-3) < 1e-15
    assert abs(big / small - 3.0) < 1e-9
    assert 5e-3 < small < 30e-3


def test_qvals_zero_for_b0_and_user_deltas(oracle):  # src/qspace.rs:481-528
    q, big, small, src = oracle.qvals([0.0, 1000.0], [[0, 0, 0], [1, 0, 0]], 0.043, 0.011)
    assert q[0] == 0.0 and q[1] > 0.0 and src == 0
    tau = 0.043 - 0.011 / 3.0
    assert abs(q[1] - math.sqrt(1000.0 / (4 * math.pi * math.pi * tau))) < 1e-12
    q, big, small, src = oracle.qvals([0.0, 3000.0], [[0, 0, 0], [1, 0, 0]])
    assert src == 1


def test_shells(oracle):  # src/qspace.rs:565-599
    b, of = oracle.shells([0.0, 1000.0, 1010.0, 990.0, 0.0, 3000.0, 3000.0], 50.0, 50.0)
    assert len(b) == 3 and b[0] == 0.0
    assert list(np.flatnonzero(of == 0)) == [0, 4]
    assert abs(b[1] - 1000.0) < 10.0 and list(np.flatnonzero(of == 1)) == [1, 2, 3]
    assert abs(b[2] - 3000.0) < 1e-9 and list(np.flatnonzero(of == 2)) == [5, 6]
    b, of = oracle.shells([1000.0, 1000.0, 3000.0], 50.0, 50.0)
    assert len(b) == 2 and abs(b[0] - 1000) < 1e-9 and abs(b[1] - 3000) < 1e-9


def test_coefficient_count(oracle):  # src/basis/shore.rs:210-219
    assert oracle.n_coeffs(6) == 72
    assert oracle.n_coeffs(2) == 8
    assert oracle.n_coeffs(8) == 145
    idx = oracle.shore_indices(6)
    assert tuple(idx[0]) == (0, 0, 0) and tuple(idx[-1]) == (6, 6, 6)


def test_brainsuite_sh_blocks(oracle):  # src/basis/shore.rs:221-236
    v = oracle.brainsuite_sh_block(0, 0.3, 0.7)
    assert abs(v[0] - 1 / math.sqrt(4 * math.pi)) < 1e-12
    v = oracle.brainsuite_sh_block(2, 0.4, 1.1)
    c = math.cos(1.1)
    assert len(v) == 5 and abs(v[2] - math.sqrt(5 / (4 * math.pi)) * 0.5 * (3 * c * c - 1)) < 1e-10


def test_design_matrix_q0_pattern(oracle):  # src/basis/shore.rs:238-273
    raw = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1]], float)
    bvecs = raw / np.maximum(np.linalg.norm(raw, axis=1, keepdims=True), 1e-12)
    bvals = [0, 1000, 1000, 1000, 2000, 2000, 2000]
    M = oracle.design_matrix(bvals, bvecs, order=4, zeta=700.0, big_delta=0.043, small_delta=0.011)
    idx = oracle.shore_indices(4)
    assert M.shape == (7, oracle.n_coeffs(4))
    for col, (_, ell, _) in enumerate(idx):
        if ell > 0:
            assert abs(M[0, col]) < 1e-12
    assert abs(M[0, 0] - oracle.kappa(700.0, 0, 0) / math.sqrt(4 * math.pi)) < 1e-10


def test_design_matrix_matches_scipy_restatement(oracle):
    """Independent scipy evaluation of the BrainSuite SHORE basis."""
    from scipy.special import eval_genlaguerre, lpmv
    from cs_dmri_b200.phantom import gradient_table
    bvals, bvecs = gradient_table(1)
    M = oracle.design_matrix(bvals, bvecs, order=6, zeta=700.0, big_delta=0.043, small_delta=0.011)
    tau = 0.043 - 0.011 / 3
    q = np.where(bvals <= 50, 0, np.sqrt(bvals / (4 * np.pi ** 2 * tau)))
    x, y, z = (bvecs * q[:, None]).T
    r = np.sqrt(x * x + y * y + z * z)
    th = np.arctan2(y, x)
    ph = np.where(r > 0, np.arccos(np.clip(z / np.where(r > 0, r, 1), -1, 1)), 0)
    cols = []
    for n in range(7):
        for l in range(0, n + 1, 2):
            kap = math.sqrt(2 * math.factorial(n - l) / (700.0 ** 1.5 * math.gamma(n + 1.5)))
            u = r * r / 700.0
            rad = kap * eval_genlaguerre(n - l, l + 0.5, u) * np.exp(-u / 2) * u ** (l / 2)
            blk = np.zeros((len(r), 2 * l + 1))
            if l == 0:
                blk[:, 0] = 1 / math.sqrt(4 * math.pi)
            else:
                p = [math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - k) / math.factorial(l + k))
                     * lpmv(k, l, np.cos(ph)) for k in range(l + 1)]
                for k in range(1, l + 1):
                    blk[:, l - k] = math.sqrt(2) * p[k] * np.cos(k * th)
                    blk[:, l + k] = math.sqrt(2) * (1 if (k + 1) % 2 == 0 else -1) * p[k] * np.sin(k * th)
                blk[:, l] = p[0]
            cols.append(rad[:, None] * blk)
    ref = np.hstack(cols)
    assert np.abs(M - ref).max() <= 1e-12 * np.abs(ref).max()


def test_regularization_diagonals(oracle):  # src/basis/shore.rs:180-195
    nd, ld = oracle.regularization(6)
    idx = oracle.shore_indices(6)
    assert np.allclose(nd, (idx[:, 0] * (idx[:, 0] + 1)) ** 2)
    assert np.allclose(ld, (idx[:, 1] * (idx[:, 1] + 1)) ** 2)


def test_radial_factor_matches_scipy(oracle):  # src/odf.rs:158-179
    cases = [(0, 0, 2.766998550654e-2), (2, 0, 3.788868806943e-2), (2, 2, -4.286615722265e-2),
             (4, 0, 4.340694526519e-2), (4, 2, -4.391643925880e-2), (4, 4, 5.400628174864e-2),
             (6, 0, 4.738453459969e-2), (6, 2, -4.722289470498e-2), (6, 4, 4.949860498183e-2),
             (6, 6, -6.322725024349e-2)]
    for n, l, e in cases:
        assert abs(oracle.radial_factor(n, l, 700.0) - e) < 1e-10


def test_brainsuite_to_tournier_index(oracle):  # src/odf.rs:189-203
    for k, idx, sign in [(0, 5, 1.0), (1, 4, 1.0), (2, 3, 1.0), (3, 2, 1.0), (4, 1, -1.0)]:
        assert oracle.brainsuite_to_tournier(2, k) == (idx, sign)


def test_projection_matches_brainsuite_eval(oracle):  # src/odf.rs:205-248
    P = oracle.shore_to_tournier(6, 700.0, 6)
    assert P.shape == (28, 72)
    dirs = [(0.3, 0.7), (1.4, 0.5), (-1.1, 1.2), (2.7, 1.5), (0.0, 0.0)]
    idx = oracle.shore_indices(6)
    for theta, phi in dirs:
        u = np.array([[math.cos(theta) * math.sin(phi), math.sin(theta) * math.sin(phi), math.cos(phi)]])
        yt = oracle.sh2amp_cart(u, 6)[0]  # float32-rounded Tournier SH
        for col, (n, l, m) in enumerate(idx):
            k = m + l
            rhs = oracle.radial_factor(n, l, 700.0) * oracle.brainsuite_sh_block(l, theta, phi)[k]
            assert abs(P[:, col] @ yt - rhs) < 1e-7 * max(1.0, abs(rhs))
    ell0 = [c for c, (_, l, _) in enumerate(idx) if l == 0]
    for c in ell0:
        assert P[0, c] != 0 and np.all(P[1:, c] == 0)


def test_hemisphere_is_321_unit_directions(oracle):
    h = oracle.odf8_hemisphere()
    assert h.shape == (321, 3)
    assert np.allclose(np.linalg.norm(h, axis=1), 1.0)
    # no antipodal pair inside the hemisphere
    d = h @ h.T
    assert d.min() > -1 + 1e-9


def test_fista_recovers_sparse_signal(oracle):  # src/solver/fista.rs:188-216
    m = np.array([1.0, 0.0, 0.5, -0.2, 0.0, 1.0, -0.1, 0.3, -0.3, 0.4, 1.0, 0.0, 0.2, -0.1, 0.0, 1.0,
                  0.5, 0.5, 0.5, 0.5, -0.5, 0.5, -0.5, 0.5, 0.5, -0.5, 0.5, -0.5, 0.1, 0.2, -0.3, 0.4]).reshape(8, 4)
    c = np.array([2.0, 0.0, -1.5, 0.0])
    coef, it, conv, _ = oracle.fista_fit(m, m @ c, 1e-3, 2000, 1e-9)
    assert abs(coef[0] - 2) < 0.05 and abs(coef[1]) < 0.05 and abs(coef[2] + 1.5) < 0.05 and abs(coef[3]) < 0.05


def test_fista_zero_alpha_is_least_squares(oracle):  # src/solver/fista.rs:217-231
    m = np.array([1.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0, -1.0]).reshape(4, 2)
    coef, *_ = oracle.fista_fit(m, m @ np.array([2.0, -3.0]), 0.0, 5000, 1e-12)
    assert abs(coef[0] - 2) < 1e-3 and abs(coef[1] + 3) < 1e-3


def _toy():  # src/solver/alpha.rs:328-343
    m = np.array([1.0, 0.0, 0.5, -0.2, 0.1, 0.0, 1.0, -0.1, 0.3, -0.4, -0.3, 0.4, 1.0, 0.0, 0.2,
                  0.2, -0.1, 0.0, 1.0, 0.5, 0.5, 0.5, 0.5, 0.5, -0.2, -0.5, 0.5, -0.5, 0.5, 0.3,
                  0.5, -0.5, 0.5, -0.5, -0.1, 0.1, 0.2, -0.3, 0.4, 0.0, 0.7, 0.0, 0.1, -0.2, 0.6,
                  -0.4, 0.3, 0.2, -0.1, 0.0]).reshape(10, 5)
    return m, m @ np.array([2.0, 0.0, -1.5, 0.0, 0.0])


def test_alpha_max_zeros_solution(oracle):  # src/solver/alpha.rs:345-371
    m, s = _toy()
    amax = oracle.alpha_max(m, s)
    assert np.all(oracle.fista_fit(m, s, amax, 500, 1e-9)[0] == 0.0)
    assert np.count_nonzero(oracle.fista_fit(m, s, amax * 0.5, 2000, 1e-9)[0]) > 0


def test_log_path_endpoints(oracle):  # src/solver/alpha.rs:373-382
    p = oracle.log_path(10.0, 5, 1e-3)
    assert len(p) == 5 and abs(p[0] - 10) < 1e-12 and abs(p[4] - 1e-2) < 1e-12 and np.all(np.diff(p) < 0)
    with pytest.raises(ValueError):
        oracle.log_path(10.0, 1, 1e-3)


def test_warm_path_matches_cold(oracle):  # src/solver/alpha.rs:384-411
    m, s = _toy()
    amax = oracle.alpha_max(m, s)
    alphas = oracle.log_path(amax, 6, 1e-2)
    warm = None
    for a in alphas:
        w, *_ = oracle.fista_fit(m, s, a, 5000, 1e-10, warm=warm)
        cold, *_ = oracle.fista_fit(m, s, a, 5000, 1e-10)
        assert np.linalg.norm(w - cold) / max(np.linalg.norm(w), np.linalg.norm(cold), 1e-12) < 1e-3
        warm = w


def test_bic_formula(oracle):  # src/solver/alpha.rs:96-103
    assert abs(oracle.bic(100, 4.0, 3) - (100 * math.log(4.0 / 100) + math.log(100) * 3)) < 1e-12
    assert math.isfinite(oracle.bic(10, 0.0, 0))


def test_tikhonov_unregularized(oracle):  # src/solver/tikhonov.rs:85-106
    m = np.array([1.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0, -1.0]).reshape(4, 2)
    c, _ = oracle.tikhonov_fit(m, m @ np.array([2.0, -3.0]), np.zeros(2), np.zeros(2), 1e-12, 0.0)
    assert np.allclose(c, [2.0, -3.0], atol=1e-6)


def _synthetic_gtab(per_shell):  # tests/optimization_kkt.rs:221-235
    bvals, bvecs = [0.0], [[0.0, 0.0, 0.0]]
    for b in (1000.0, 2000.0, 3000.0):
        for i in range(per_shell):
            phi = math.pi * (1 + math.sqrt(5))
            z = 1 - (2 * i + 1) / per_shell
            r = math.sqrt(max(1 - z * z, 0))
            t = phi * i
            bvecs.append([r * math.cos(t), r * math.sin(t), z])
            bvals.append(b)
    return np.array(bvals), np.array(bvecs)


@pytest.mark.parametrize("per_shell,lam,bound", [(60, 1e-2, 1e-10), (80, 1e-8, 1e-9)])
def test_tikhonov_normal_equations_on_shore(oracle, per_shell, lam, bound):  # tests/optimization_kkt.rs:163-215
    bvals, bvecs = _synthetic_gtab(per_shell)
    M = oracle.design_matrix(bvals, bvecs, order=6, zeta=700.0, big_delta=0.04, small_delta=0.012)
    nd, ld = oracle.regularization(6)
    rng = np.random.default_rng(per_shell)
    beta = np.zeros(72)
    beta[rng.choice(72, 6, replace=False)] = rng.uniform(0.5, 2, 6) * rng.choice([-1, 1], 6)
    y = M @ beta + 0.005 * rng.standard_normal(len(bvals))
    c, _ = oracle.tikhonov_fit(M, y, nd, ld, lam, lam)
    lhs = M.T @ M @ c + lam * nd * c + lam * ld * c
    rhs = M.T @ y
    assert np.linalg.norm(lhs - rhs) / np.linalg.norm(rhs) < bound


def _brute_nnls(h, b):  # src/solver/icls.rs:701-737
    n = h.shape[1]
    best = None
    for mask in range(1 << n):
        free = [i for i in range(n) if (mask >> i) & 1]
        x = np.zeros(n)
        if free:
            hf = h[:, free]
            try:
                xf = np.linalg.solve(hf.T @ hf, hf.T @ b)
            except np.linalg.LinAlgError:
                continue
            if np.any(xf < -1e-9):
                continue
            x[free] = xf
        cost = 0.5 * np.sum((h @ x - b) ** 2)
        if best is None or cost < best[1]:
            best = (x, cost)
    return best[0]


def test_icls_cases(oracle):  # src/solver/icls.rs:526-699
    h = np.array([1.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0, -1.0]).reshape(4, 2)
    x, d = oracle.icls_solve(h, np.eye(2), h @ np.array([2.0, 3.0]), epsilon=1e-12)
    assert np.allclose(x, [2, 3], atol=1e-7) and d["final_active"] == 0 and d["converged"]
    x, d = oracle.icls_solve(np.eye(2), np.eye(2), np.array([-1.0, 1.0]), epsilon=1e-12)
    assert np.allclose(x, [0, 1], atol=1e-9) and d["final_active"] == 1 and d["converged"]
    x, d = oracle.icls_solve(np.eye(3), np.eye(3), np.array([1.0, 2.0, -1.0]), epsilon=1e-12)
    assert np.allclose(x, [1, 2, 0], atol=1e-9) and d["final_active"] == 1
    x, _ = oracle.icls_solve(np.array([[1.0]]), np.array([[1.0]]), np.array([-2.0]), epsilon=1e-12)
    assert abs(x[0]) < 1e-10
    x, _ = oracle.icls_solve(np.eye(2), np.array([[1.0, 1.0]]), np.zeros(2), epsilon=1e-12)
    assert np.allclose(x, 0, atol=1e-10)
    x, d = oracle.icls_solve(np.eye(2), np.array([[1.0, 1.0]]), np.array([-2.0, 1.0]), epsilon=1e-12)
    assert np.allclose(x, [-1.5, 1.5], atol=1e-9) and d["converged"] and d["final_active"] == 1
    h = np.array([1.0, 0.5, 0.2, 0.5, 1.0, 0.4, 0.2, 0.4, 1.0, 0.3, 0.3, 0.3]).reshape(4, 3)
    b = np.array([1.0, -0.5, 0.8, 0.2])
    x, d = oracle.icls_solve(h, np.eye(3), b, epsilon=1e-12, tol=1e-12)
    assert np.all(x >= -1e-9) and np.allclose(x, _brute_nnls(h, b), atol=1e-7) and d["converged"]
