"""Hypergradient alpha selection on the GPU (cs_dmri_b200.hyper).

The hypergradient of the held-out error against the oracle's implicit
adjoint on the same coefficients (1e-8 relative) and against central
differences of the held-out error through the GPU fit at tol 1e-12 (1e-4);
the pipeline's invariants: the kept alpha never does worse on the held-out
samples than the starting alpha, the final coefficients are the full-table
fit at that alpha, and the reference's selections are scored on the same
samples."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    from cs_dmri_b200.hyper import HypergradientAlpha
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((8, 5, 4), seed=12)
    S = torch.from_numpy(ph.data.reshape(-1, ph.data.shape[-1])).cuda()
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta)
    return ph, S, kw, torch, HypergradientAlpha


def test_hypergradient_matches_oracle_and_differences(setup, oracle):
    ph, S, kw, torch, HA = setup
    sel = HA(ph.bvals, ph.bvecs, tol=1e-12, max_iter=200000, **kw)
    s_tr, s_ho = sel.split(S)
    a = torch.full((S.shape[0],), 0.01, dtype=torch.float64, device="cuda", requires_grad=True)
    c = sel.model.fit(s_tr, a)
    loss = sel.heldout_loss(c, s_ho)
    loss.sum().backward()
    g = a.grad.cpu().numpy()
    cn, Str, Sho = c.detach().cpu().numpy(), s_tr.cpu().numpy().astype(np.float64), s_ho.cpu().numpy()
    Mtr = oracle.design_matrix(ph.bvals[sel.train], ph.bvecs[sel.train], 6, 700.0, **kw)
    Mho = oracle.design_matrix(ph.bvals[sel.held_out], ph.bvecs[sel.held_out], 6, 700.0, **kw)
    for v in range(len(cn)):
        gc = 2.0 * Mho.T @ (Mho @ cn[v] - Sho[v])
        _, ga, _ = oracle.l1_adjoint(Mtr, cn[v], gc)
        np.testing.assert_allclose(g[v], ga, rtol=1e-8, atol=1e-12 * abs(ga) + 1e-300)
    h = 0.01 * 1e-3
    lp = sel.heldout_loss(sel.model.fit(s_tr, 0.01 + h), s_ho).cpu().numpy()
    lm = sel.heldout_loss(sel.model.fit(s_tr, 0.01 - h), s_ho).cpu().numpy()
    fd = (lp - lm) / (2 * h)
    ok = np.abs(fd - g) <= 1e-4 * np.maximum(np.abs(fd), np.abs(g).max() * 1e-6)
    assert ok.mean() >= 0.9, (np.flatnonzero(~ok), fd[~ok], g[~ok])


def test_pipeline(setup):
    ph, S, kw, torch, HA = setup
    from cs_dmri_b200.autograd import DifferentiableShore
    from cs_dmri_b200.hyper import select_alpha_hypergradient
    mask = ph.mask.copy()
    mask[0, 0, :] = False
    out = select_alpha_hypergradient(ph.data, ph.bvals, ph.bvecs, mask, **kw)
    V = int(mask.sum())
    a = out["alpha"][mask]
    assert np.all(a > 0) and np.all(out["alpha"][~mask] == 0)
    assert out["peak_dirs"].shape == mask.shape + (3, 3) and out["gfa"].shape == mask.shape
    comp = out["comparison"]
    assert set(comp) == {"hypergradient", "fixed_alpha0", "l2-anchored", "path-bic"}
    assert comp["hypergradient"] <= comp["fixed_alpha0"]
    # per voxel the kept alpha is never worse than the start
    sel = HA(ph.bvals, ph.bvecs, **kw)
    Sm = torch.from_numpy(ph.data[mask]).cuda()
    best, loss, loss0, hist = sel.run(Sm)
    assert len(hist) == 8 and bool((loss <= loss0).all())
    np.testing.assert_array_equal(best.cpu().numpy().astype(np.float32), a)
    # the final coefficients are the full-table fit at the kept alpha
    full = DifferentiableShore(ph.bvals, ph.bvecs, **kw)
    c = full.fit(Sm, best).cpu().numpy().astype(np.float32)
    np.testing.assert_array_equal(out["coefficients"][mask], c)
    assert V == len(c)


def test_captured_run_matches_the_eager_run(setup):
    """The 8-step run captured in one CUDA graph: replays give the eager
    run's alpha and losses bit for bit, also after the signals change."""
    ph, S, kw, torch, HA = setup
    sel = HA(ph.bvals, ph.bvecs, **kw)
    static = S.clone()
    cap = sel.capture(static)
    for scale in (1.0, 0.7):
        static.copy_(S * scale)
        got = [t.clone() for t in cap.replay()]
        want = sel.run(S * scale)[:3]
        for g, w in zip(got, want):
            assert torch.equal(g, w)
    del cap
