"""Differentiable fit on the GPU (cs_dmri_b200.autograd) against the oracle.

* the batch fit is the volume fit: bit-identical FP64 coefficients;
* the adjoint kernels against the oracle's implicit-function adjoints on the
  same coefficients (relative 1e-9: both solve the same well-conditioned
  support system in FP64, in different summation orders);
* on 200 seeded voxels (the differentiable-fit workload's check), gradients
  against central differences through the GPU fit itself run to tol 1e-12:
  on a fixed support the L1 solution is affine in the signal, so the
  difference quotient is exact up to the fit tolerance (relative 1e-6);
* RTOP / ODF / prediction maps and their adjoints against the oracle.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALPHA = 0.01


@pytest.fixture(scope="module")
def ctx(oracle):
    import torch
    from cs_dmri_b200.autograd import DifferentiableShore
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((10, 5, 4), seed=21)  # 200 voxels
    S = ph.data.reshape(-1, ph.data.shape[-1])
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta)
    M = oracle.design_matrix(ph.bvals, ph.bvecs, 6, 700.0, **kw)
    St = torch.from_numpy(S).cuda()
    return dict(ph=ph, S=S, St=St, kw=kw, M=M, torch=torch, DS=DifferentiableShore)


def model(ctx, **kw):
    ph = ctx["ph"]
    return ctx["DS"](ph.bvals, ph.bvecs, **ctx["kw"], **kw)


def test_batch_fit_is_the_volume_fit(ctx):
    from cs_dmri_b200 import shore_fit
    ph, S = ctx["ph"], ctx["S"]
    vol = S.reshape(len(S), 1, 1, -1)
    mask = np.ones(vol.shape[:3], bool)
    for reg, extra in (("l1", dict(alpha_mode="fixed", alpha=ALPHA)), ("l2", dict(lambda_n=0.05, lambda_l=0.02))):
        want = shore_fit(vol, ph.bvals, ph.bvecs, mask, regularization=reg, return_coef64=True, **ctx["kw"],
                         **extra)["coef64"]
        m = model(ctx, regularization=reg)
        got = m.fit(ctx["St"], ALPHA) if reg == "l1" else m.fit(ctx["St"], lambda_n=0.05, lambda_l=0.02)
        np.testing.assert_array_equal(got.cpu().numpy(), want)


def test_per_voxel_alpha_and_warm_start(ctx, oracle):
    torch = ctx["torch"]
    m = model(ctx)
    St = ctx["St"]
    a = np.where(np.arange(len(St)) % 2 == 0, 0.01, 0.05)
    c = m.fit(St, torch.tensor(a, dtype=torch.float64, device="cuda")).cpu().numpy()
    c1 = m.fit(St, 0.01).cpu().numpy()
    c5 = m.fit(St, 0.05).cpu().numpy()
    np.testing.assert_array_equal(c[0::2], c1[0::2])
    np.testing.assert_array_equal(c[1::2], c5[1::2])
    # a warm start follows the oracle's warm-started iterations
    warm = torch.from_numpy(c5).cuda()
    cw = m.fit(St, 0.01, warm=warm).cpu().numpy()
    for v in range(0, len(St), 25):
        want, _, _, _ = oracle.fista_fit(ctx["M"], ctx["S"][v].astype(np.float64), 0.01, warm=c5[v])
        np.testing.assert_allclose(cw[v], want, rtol=0, atol=1e-5 * np.abs(want).max())


def test_l1_adjoint_matches_oracle(ctx, oracle):
    torch = ctx["torch"]
    m = model(ctx)
    c = m.fit(ctx["St"], ALPHA)
    rng = np.random.default_rng(4)
    gc = rng.normal(size=c.shape)
    gs, gh = m.signal_gradient(c, torch.from_numpy(gc).cuda())
    gs, gh, cn = gs.cpu().numpy(), gh.cpu().numpy(), c.cpu().numpy()
    for v in range(len(cn)):
        ws, wa, w = oracle.l1_adjoint(ctx["M"], cn[v], gc[v])
        np.testing.assert_allclose(gs[v], ws, rtol=0, atol=1e-9 * np.abs(ws).max() + 1e-300)
        np.testing.assert_allclose(gh[v, 0], wa, rtol=1e-9, atol=1e-300)
        assert gh[v, 1] == 0.0


def test_l2_adjoint_matches_oracle(ctx, oracle):
    torch = ctx["torch"]
    m = model(ctx, regularization="l2")
    c = m.fit(ctx["St"], lambda_n=0.05, lambda_l=0.02)
    rng = np.random.default_rng(5)
    gc = rng.normal(size=c.shape)
    gs, gh = m.signal_gradient(c, torch.from_numpy(gc).cuda(), lambda_n=0.05, lambda_l=0.02)
    gs, gh, cn = gs.cpu().numpy(), gh.cpu().numpy(), c.cpu().numpy()
    nd, ld = oracle.regularization(6)
    for v in range(0, len(cn), 7):
        ws, (wn, wl), _ = oracle.l2_adjoint(ctx["M"], cn[v], gc[v], nd, ld, 0.05, 0.02)
        np.testing.assert_allclose(gs[v], ws, rtol=0, atol=1e-9 * np.abs(ws).max())
        np.testing.assert_allclose(gh[v], [wn, wl], rtol=1e-9)


def test_l1_gradients_match_finite_differences(ctx, oracle):
    """200 voxels.  (1) The GPU fit at tol 1e-12 against the exact minimiser
    (the oracle's polish on the fit's support, KKT-certified).  (2) Signal and
    alpha gradients against central differences of the exact solution map -
    on a certified support it is affine in the signal and in alpha, so the
    difference quotient is exact to rounding.  (3) Against central
    differences through the GPU fit itself, with steps large enough that the
    fit tolerance stays far below the change."""
    torch = ctx["torch"]
    m = model(ctx, tol=1e-12, max_iter=200000)
    S, St, M = ctx["S"], ctx["St"], ctx["M"]
    S64 = S.astype(np.float64)
    c = m.fit(St, ALPHA).cpu().numpy()
    exact, ok = zip(*(oracle.lasso_polish(M, S64[v], ALPHA, c[v]) for v in range(len(S))))
    exact, ok = np.array(exact), np.array(ok)
    assert ok.mean() >= 0.95
    err = np.abs(c - exact).max(1) / np.abs(exact).max(1)
    assert np.all(err[ok] < 1e-6), err.max()
    rng = np.random.default_rng(6)
    gc = rng.normal(size=c.shape)
    gs, gh = m.signal_gradient(torch.from_numpy(c).cuda(), torch.from_numpy(gc).cuda())
    gs, gh = gs.cpu().numpy(), gh.cpu().numpy()
    d = rng.normal(size=S.shape) * 1e-3 * np.abs(S).mean()
    h = ALPHA * 1e-3
    checked = 0
    for v in np.flatnonzero(ok):
        cp, okp = oracle.lasso_polish(M, S64[v] + d[v], ALPHA, exact[v])
        cm, okm = oracle.lasso_polish(M, S64[v] - d[v], ALPHA, exact[v])
        ap, oka = oracle.lasso_polish(M, S64[v], ALPHA + h, exact[v])
        am, okb = oracle.lasso_polish(M, S64[v], ALPHA - h, exact[v])
        if not (okp and okm and oka and okb):
            continue
        checked += 1
        fd = gc[v] @ (cp - cm) / 2
        np.testing.assert_allclose(gs[v] @ d[v], fd, rtol=1e-6, atol=1e-9 * np.abs(gc[v]) @ np.abs(cp - cm))
        fa = gc[v] @ (ap - am) / (2 * h)
        np.testing.assert_allclose(gh[v, 0], fa, rtol=1e-6, atol=1e-9 * np.abs(gc[v]) @ np.abs(ap - am) / h)
    assert checked >= 0.9 * len(S)
    # through the GPU fit: float32 perturbed signals, exact differences in f64
    d32 = (rng.normal(size=S.shape) * 2e-2 * np.abs(S).mean()).astype(np.float32)
    Sp, Sm = (S + d32).astype(np.float32), (S - d32).astype(np.float32)
    cp = m.fit(torch.from_numpy(Sp).cuda(), ALPHA).cpu().numpy()
    cm = m.fit(torch.from_numpy(Sm).cuda(), ALPHA).cpu().numpy()
    same = ok & np.all((cp != 0) == (c != 0), axis=1) & np.all((cm != 0) == (c != 0), axis=1)
    assert same.mean() >= 0.5
    lhs = np.einsum("vn,vn->v", gs, Sp.astype(np.float64) - Sm.astype(np.float64))
    rhs = np.einsum("vk,vk->v", gc, cp - cm)
    scale = np.einsum("vk,vk->v", np.abs(gc), np.abs(cp - cm))
    assert np.all(np.abs(lhs - rhs)[same] <= 1e-4 * scale[same])


def test_l2_lambda_gradient_through_autograd(ctx):
    torch = ctx["torch"]
    m = model(ctx, regularization="l2")
    St = ctx["St"]
    ln = torch.tensor(0.05, dtype=torch.float64, device="cuda", requires_grad=True)
    ll = torch.tensor(0.02, dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.from_numpy(np.random.default_rng(7).normal(size=(len(St), m.K))).cuda()
    (m.fit(St, lambda_n=ln, lambda_l=ll) * w).sum().backward()
    for lam, g, which in ((0.05, ln.grad, "n"), (0.02, ll.grad, "l")):
        h = lam * 1e-3
        f = {}
        for sgn in (1, -1):
            kw = dict(lambda_n=0.05, lambda_l=0.02)
            kw["lambda_" + which] = lam + sgn * h
            f[sgn] = float((m.fit(St, **kw) * w).sum())
        np.testing.assert_allclose(float(g), (f[1] - f[-1]) / (2 * h), rtol=1e-5)


def test_rtop_odf_predict_and_their_adjoints(ctx, oracle):
    torch = ctx["torch"]
    from cs_dmri_b200.autograd import geodesic_sphere
    m = model(ctx)
    c = m.fit(ctx["St"], ALPHA)
    cn = c.cpu().numpy()
    rt = m.rtop(c).cpu().numpy()
    want = np.array([oracle.microstructure_voxel(cn[v], 6, 700.0)["rtop"] for v in range(len(cn))])
    np.testing.assert_allclose(rt, want, rtol=1e-12)
    # RTOP adjoint against central differences of the oracle's RTOP
    cr = c.clone().requires_grad_(True)
    g = np.random.default_rng(8).normal(size=len(cn))
    (m.rtop(cr) * torch.from_numpy(g).cuda()).sum().backward()
    grad = cr.grad.cpu().numpy()
    for v in range(0, len(cn), 20):
        def central(k, h):
            cp, cm = cn[v].copy(), cn[v].copy()
            cp[k] += h
            cm[k] -= h
            return (oracle.microstructure_voxel(cp, 6, 700.0)["rtop"] -
                    oracle.microstructure_voxel(cm, 6, 700.0)["rtop"]) / (2 * h)
        fd = np.zeros(m.K)
        for k in range(m.K):  # Richardson-extrapolated central differences
            h = 1e-4 * np.abs(cn[v]).max()
            fd[k] = (4 * central(k, h / 2) - central(k, h)) / 3
        np.testing.assert_allclose(grad[v], g[v] * fd, rtol=1e-5, atol=1e-7 * np.abs(g[v] * fd).max())
    # ODF on the 362-vertex sphere and its adjoint
    dirs = geodesic_sphere(6)
    A = oracle.odf_matrix(dirs, 6, 700.0)
    co = c.clone().requires_grad_(True)
    odf = m.odf(co)
    np.testing.assert_allclose(odf.detach().cpu().numpy(), cn @ A.T, rtol=1e-12, atol=1e-12 * np.abs(cn @ A.T).max())
    go = np.random.default_rng(9).normal(size=odf.shape)
    (odf * torch.from_numpy(go).cuda()).sum().backward()
    np.testing.assert_allclose(co.grad.cpu().numpy(), go @ A, rtol=1e-12, atol=1e-12 * np.abs(go @ A).max())
    # prediction on a held-out table
    ph = ctx["ph"]
    sel = np.arange(0, len(ph.bvals), 10)
    P = oracle.design_matrix(ph.bvals[sel], ph.bvecs[sel], 6, 700.0, **ctx["kw"])
    pred = m.predict(c, ph.bvals[sel], ph.bvecs[sel]).cpu().numpy()
    np.testing.assert_allclose(pred, cn @ P.T, rtol=1e-12, atol=1e-12 * np.abs(cn @ P.T).max())


def test_end_to_end_backward(ctx, oracle):
    """signals -> fit -> (RTOP, ODF) -> scalar loss, backward through every
    kernel, against the oracle's adjoint chain."""
    torch = ctx["torch"]
    from cs_dmri_b200.autograd import geodesic_sphere
    m = model(ctx)
    St = ctx["St"].clone().requires_grad_(True)
    alpha = torch.tensor(ALPHA, dtype=torch.float64, device="cuda", requires_grad=True)
    c = m.fit(St, alpha)
    loss = m.rtop(c).sum() + 1e-3 * m.odf(c).square().sum()
    loss.backward()
    cn = c.detach().cpu().numpy()
    A = oracle.odf_matrix(geodesic_sphere(6), 6, 700.0)
    cr = c.detach().clone().requires_grad_(True)
    m.rtop(cr).sum().backward()
    gc = cr.grad.cpu().numpy() + 2e-3 * (cn @ A.T) @ A
    gs_want = np.zeros_like(ctx["S"], dtype=np.float64)
    ga_want = 0.0
    for v in range(len(cn)):
        gs_want[v], ga, _ = oracle.l1_adjoint(ctx["M"], cn[v], gc[v])
        ga_want += ga
    got = St.grad.cpu().numpy()
    assert St.grad.dtype == torch.float32
    np.testing.assert_allclose(got, gs_want, rtol=1e-5, atol=1e-6 * np.abs(gs_want).max())
    np.testing.assert_allclose(float(alpha.grad), ga_want, rtol=1e-8)


def test_previous_iteration_schedule_changes_nothing(ctx):
    """Repeated L1 fits of one batch take the voxels up slowest first (the
    previous fit's iteration counts); coefficients stay bit-identical to the
    fits in voxel order, at a fixed alpha and across alpha and warm-start
    changes."""
    torch = ctx["torch"]
    St = ctx["St"]
    ref, sch = model(ctx, schedule="index"), model(ctx)
    assert sch.schedule == "previous"
    warm = None
    for a in (0.01, 0.01, 0.03, 0.01):
        want = ref.fit(St, a, warm=warm).cpu().numpy()
        got = sch.fit(St, a, warm=warm).cpu().numpy()
        np.testing.assert_array_equal(got, want)
        warm = torch.from_numpy(want).cuda()
    it = sch._iters.cpu().numpy()
    assert it.min() >= 1 and it.max() > it.min()  # counts recorded for the next fit's order
    half = sch.fit(St[:100], 0.01).cpu().numpy()  # another batch size: voxel order again
    np.testing.assert_array_equal(half, ref.fit(St[:100], 0.01).cpu().numpy())
    with pytest.raises(ValueError, match="schedule"):
        model(ctx, schedule="fastest")


def test_calls_on_one_handle_run_in_call_order():
    """The batch fit returns with its work queued on the caller's stream; a
    call that then switches the handle's gradient table on the handle's own
    stream (here the design matrix of another table) must not reach the
    shared set-up before the queued fit has used it.  100,000 voxels, so the
    fit runs the two-pass schedule and its second pass starts late."""
    import torch
    from cs_dmri_b200 import design_matrix
    from cs_dmri_b200.autograd import DifferentiableShore
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((50, 50, 40), seed=12)
    S = torch.from_numpy(ph.data.reshape(-1, ph.data.shape[-1])).cuda()
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta)
    a = torch.full((S.shape[0],), 0.01, dtype=torch.float64, device="cuda")
    ref = DifferentiableShore(ph.bvals, ph.bvecs, **kw).fit(S, a)
    torch.cuda.synchronize()
    other = np.arange(0, len(ph.bvals), 2)
    for _ in range(2):
        c = DifferentiableShore(ph.bvals, ph.bvecs, **kw).fit(S, a)  # queued, not waited for
        design_matrix(ph.bvals[other], ph.bvecs[other], **kw)       # another table on the same handle
        assert torch.equal(c, ref)


def test_zero_support_and_errors(ctx):
    torch = ctx["torch"]
    m = model(ctx)
    St = ctx["St"][:16]
    c = m.fit(St, 1e9)  # alpha above alpha_max: every coefficient 0
    assert float(c.abs().max()) == 0.0
    gs, gh = m.signal_gradient(c, torch.ones_like(c))
    assert float(gs.abs().max()) == 0.0 and float(gh.abs().max()) == 0.0
    with pytest.raises(ValueError, match="l1 or l2"):
        model(ctx, regularization="nonneg")
    with pytest.raises(ValueError, match="float32"):
        m.fit(St.double(), ALPHA)
    with pytest.raises(ValueError, match="one value per voxel"):
        m.fit(St, torch.full((3,), 0.01, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError, match="needs alpha"):
        m.fit(St)


@pytest.mark.parametrize("reg", ["l1", "l2"])
def test_radial_order_8_adjoint_matches_oracle(ctx, oracle, reg):
    """K = 145: the adjoint kernels' five-register rows and the cached-matrix
    apply (the 259 x 145 design does not fit in shared memory)."""
    torch = ctx["torch"]
    ph = ctx["ph"]
    m = model(ctx, regularization=reg, radial_order=8)
    St = ctx["St"][:48]
    c = m.fit(St, 0.01) if reg == "l1" else m.fit(St, lambda_n=0.05, lambda_l=0.02)
    gc = np.random.default_rng(11).normal(size=c.shape)
    kw = dict(alpha=0.01) if reg == "l1" else dict(lambda_n=0.05, lambda_l=0.02)
    gs, gh = m.signal_gradient(c, torch.from_numpy(gc).cuda(), **kw)
    gs, gh, cn = gs.cpu().numpy(), gh.cpu().numpy(), c.cpu().numpy()
    M8 = oracle.design_matrix(ph.bvals, ph.bvecs, 8, 700.0, **ctx["kw"])
    nd, ld = oracle.regularization(8)
    for v in range(0, len(cn), 4):
        if reg == "l1":
            ws, wa, _ = oracle.l1_adjoint(M8, cn[v], gc[v])
            np.testing.assert_allclose(gh[v, 0], wa, rtol=1e-8, atol=1e-300)
        else:
            ws, (wn, wl), _ = oracle.l2_adjoint(M8, cn[v], gc[v], nd, ld, 0.05, 0.02)
            np.testing.assert_allclose(gh[v], [wn, wl], rtol=1e-8)
        np.testing.assert_allclose(gs[v], ws, rtol=0, atol=1e-8 * np.abs(ws).max() + 1e-300)
