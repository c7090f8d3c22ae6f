"""Oracle parity on the benchmark workloads and on the code paths the
benchmark times.

The small-phantom tests elsewhere pin the arithmetic; these pin the measured
configurations themselves:

* grid4k (20 x 20 x 10, every voxel masked, radial order 6, fixed alpha 0.01)
  in full against the oracle;
* a strided sample of brain300k (96 x 114 x 96, 299,432 masked voxels; every
  32nd masked voxel, 9,358 voxels spread over the whole mask) taken from
  whole-volume fits made exactly as the benchmark makes them:
  - the device-buffer FP64 fit (coefficients only: the two-pass FISTA
    schedule with the autotuned kernel shape),
  - the page-locked host fit (the pipelined chunked path),
  - the mixed-precision device fit,
  - Tikhonov (lambda_n = lambda_l = 0.05) and the amplitude-positivity QP
    on the same sample;
* per-voxel designs at radial order 8 on 1,024 voxels: coefficients, and
  the RTOP and GFA computed from them.

Tolerances are the parity bounds of the FP64 path: per-voxel coefficient
relative L2 <= 1e-5 for L1 (a stopping decision within rounding of tol may
end a voxel one iteration earlier or later, moving it by about tol |x|),
iteration counts within 1; <= 1e-8 for Tikhonov (a direct solve).  The
float32 coefficient volumes the benchmark produces are compared as they
are (float32 rounding is ~6e-8 relative, far below 1e-5).

KKT residuals (the form of the reference's tests/common/mod.rs:127-153:
max over the support of |g_j + alpha sign(c_j)| and max off it of
max(0, |g_j| - alpha), g = M^T (M c - s) / n) are reported for the GPU and
oracle outputs of the sample: the reference's stopping rule (tol 1e-6 on the
relative change) leaves both well above a converged optimum's, and the GPU's
distribution must match the oracle's.
"""

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L1 = dict(alpha_mode="fixed", alpha=0.01, max_iter=1000, tol=1e-6, radial_order=6, zeta=700.0)
STRIDE = 32           # brain300k sample: every 32nd masked voxel (9,358 voxels)


@pytest.fixture(scope="module")
def brain():
    from cs_dmri_b200.phantom import config_phantom
    return config_phantom("brain300k")


@pytest.fixture(scope="module")
def brain_rows(brain):
    """Masked voxel signals (V, N) float32 in canonical x-y-z order."""
    n = brain.data.shape[-1]
    return brain.data.reshape(-1, n)[brain.mask.ravel()]


@pytest.fixture(scope="module")
def l1_sample_oracle(brain, brain_rows, oracle):
    idx = np.arange(0, len(brain_rows), STRIDE)
    return idx, oracle_rows(oracle, brain, brain_rows[idx], **L1)


def oracle_rows(oracle, ph, rows, **kw):
    """Oracle fit of the given voxel signals (V, N), as a V x 1 x 1 volume."""
    V, n = rows.shape
    sub = np.ascontiguousarray(rows.reshape(V, 1, 1, n))
    return oracle.shore_fit(sub, ph.bvals, ph.bvecs, np.ones((V, 1, 1), bool), big_delta=ph.big_delta,
                            small_delta=ph.small_delta, diagnostics=True, **kw)


def rel_rows(a, b):
    nb = np.linalg.norm(b, axis=1)
    nz = nb > 0
    return np.linalg.norm(a - b, axis=1)[nz] / nb[nz]


def kkt_residuals(M, S, C, alpha):
    """(max_active, max_inactive) per voxel, tests/common/mod.rs:127-153."""
    n = M.shape[0]
    g = (C @ M.T - S) @ M / n
    act = np.abs(C) > 1e-10
    a = np.where(act, np.abs(g + alpha * np.sign(C)), 0.0).max(1)
    i = np.where(act, 0.0, np.maximum(np.abs(g) - alpha, 0.0)).max(1)
    return a, i


def masked_rows(volume, mask):
    return volume.reshape(-1, volume.shape[-1])[mask.ravel()]


def check_l1(got, ref, what):
    r = rel_rows(got, ref)
    assert r.max() <= 1e-5, (what, float(r.max()))


def test_grid4k_config_in_full(oracle):
    """The CPU-runnable configuration (20 x 20 x 10, 4,000 voxels) against the
    oracle: coefficients, iterations, convergence and the diagnostic maps."""
    from cs_dmri_b200 import shore_fit
    from cs_dmri_b200.phantom import config_phantom
    ph = config_phantom("grid4k")
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, diagnostics=True, **L1)
    gpu = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, return_coef64=True, **kw)
    ref = oracle.shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    assert gpu["n_voxels"] == ref["n_voxels"] == 4000
    check_l1(gpu["coef64"], ref["coef64"], "grid4k")
    it_g, it_o = gpu["iterations"][ph.mask].astype(int), ref["iterations"][ph.mask].astype(int)
    assert np.abs(it_g - it_o).max() <= 1 and np.mean(it_g == it_o) >= 0.99
    assert np.mean(gpu["converged"] == ref["converged"]) >= 0.999
    np.testing.assert_allclose(gpu["r2"], ref["r2"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(gpu["residual_l2"], ref["residual_l2"], rtol=1e-5)
    np.testing.assert_allclose(gpu["coefficients"], ref["coefficients"], rtol=1e-4, atol=1e-3)
    assert gpu["total_iterations"] == pytest.approx(ref["total_iterations"], rel=1e-3)


def test_brain300k_device_fit_as_benchmarked(brain, brain_rows, l1_sample_oracle):
    """The benchmark's `value` call: device-resident volume, coefficients only,
    FP64; the fit takes two FISTA passes with the autotuned kernel shape."""
    import torch
    from cs_dmri_b200 import _abi, shore_fit_device
    idx, ref = l1_sample_oracle
    d = torch.from_numpy(brain.data).cuda()
    m = torch.from_numpy(brain.mask).cuda()
    coef, res = shore_fit_device(d, m, brain.bvals, brain.bvecs, big_delta=brain.big_delta,
                                 small_delta=brain.small_delta, precision="fp64", **L1)
    t = _abi.last_timing(0)
    assert t.fista_parked > len(brain_rows) // 2 and t.fista_warps in (12, 16)
    got = masked_rows(coef.cpu().numpy(), brain.mask)[idx].astype(np.float64)
    check_l1(got, ref["coef64"], "device fp64")
    # total iteration count of the whole volume against the sample's mean
    per_voxel = res.total_iterations / len(brain_rows)
    assert abs(per_voxel - ref["total_iterations"] / len(idx)) < 0.05 * per_voxel
    del d, m, coef
    torch.cuda.empty_cache()


def test_brain300k_iterations_and_kkt(brain, brain_rows, l1_sample_oracle, oracle):
    """Per-voxel iteration counts of the whole-volume fit (same kernels and
    two-pass schedule; the diagnostics need the host entry point) against the
    oracle on the sample, and the KKT residual distribution of both."""
    from cs_dmri_b200 import shore_fit
    idx, ref = l1_sample_oracle
    gpu = shore_fit(brain.data, brain.bvals, brain.bvecs, brain.mask, big_delta=brain.big_delta,
                    small_delta=brain.small_delta, diagnostics=True, return_coef64=True, **L1)
    check_l1(gpu["coef64"][idx], ref["coef64"], "host fp64")
    it_g = gpu["iterations"][brain.mask][idx].astype(int)
    it_o = ref["iterations"].ravel().astype(int)
    assert np.abs(it_g - it_o).max() <= 1 and np.mean(it_g == it_o) >= 0.99
    M = oracle.design_matrix(brain.bvals, brain.bvecs, 6, 700.0, big_delta=brain.big_delta,
                             small_delta=brain.small_delta)
    S = brain_rows[idx].astype(np.float64)
    ga, gi = kkt_residuals(M, S, gpu["coef64"][idx], 0.01)
    oa, oi = kkt_residuals(M, S, ref["coef64"], 0.01)
    q = [50, 90, 99]
    print("\nKKT (reference stopping rule), sample of", len(idx), "voxels, percentiles", q)
    print("  gpu    active", np.percentile(ga, q), " inactive", np.percentile(gi, q))
    print("  oracle active", np.percentile(oa, q), " inactive", np.percentile(oi, q))
    for g, o in ((ga, oa), (gi, oi)):
        gm, om = np.median(g), np.median(o)
        assert abs(gm - om) <= 0.1 * max(om, 1e-30) + 1e-12


def test_brain300k_pipelined_host_fit_as_benchmarked(brain, brain_rows, l1_sample_oracle):
    """The benchmark's `e2e` call: page-locked input and output volumes
    through the host entry point (the pipelined chunked path)."""
    import torch
    from cs_dmri_b200 import _abi, shore_fit
    idx, ref = l1_sample_oracle
    pin = torch.empty(brain.data.shape, dtype=torch.float32, pin_memory=True)
    pin.numpy()[...] = brain.data
    out = torch.full(brain.data.shape[:3] + (72,), float("nan"), dtype=torch.float32, pin_memory=True)
    shore_fit(pin.numpy(), brain.bvals, brain.bvecs, brain.mask, big_delta=brain.big_delta,
              small_delta=brain.small_delta, coefficients_out=out.numpy(), precision="fp64", **L1)
    assert _abi.last_timing(0).ms_rhs == 0.0      # the pipelined path ran
    o = out.numpy()
    assert np.all(o[~brain.mask] == 0)
    check_l1(masked_rows(o, brain.mask)[idx].astype(np.float64), ref["coef64"], "pipelined host")
    del pin, out


def test_brain300k_mixed_fit_as_benchmarked(brain, l1_sample_oracle):
    """The benchmark's mixed-precision path on the same volume."""
    import torch
    from cs_dmri_b200 import shore_fit_device
    idx, ref = l1_sample_oracle
    d = torch.from_numpy(brain.data).cuda()
    m = torch.from_numpy(brain.mask).cuda()
    coef, _ = shore_fit_device(d, m, brain.bvals, brain.bvecs, big_delta=brain.big_delta,
                               small_delta=brain.small_delta, precision="mixed", **L1)
    got = masked_rows(coef.cpu().numpy(), brain.mask)[idx].astype(np.float64)
    check_l1(got, ref["coef64"], "mixed")
    del d, m, coef
    torch.cuda.empty_cache()


def test_brain300k_tikhonov_sample(brain, brain_rows, oracle):
    """Configuration 2's L2 fit (lambda_n = lambda_l = 0.05), whole volume on
    the device path, against the oracle on the 9,358-voxel sample."""
    import torch
    from cs_dmri_b200 import shore_fit_device
    kw = dict(regularization="l2", lambda_n=0.05, lambda_l=0.05, radial_order=6, zeta=700.0)
    d = torch.from_numpy(brain.data).cuda()
    m = torch.from_numpy(brain.mask).cuda()
    coef, _ = shore_fit_device(d, m, brain.bvals, brain.bvecs, big_delta=brain.big_delta,
                               small_delta=brain.small_delta, **kw)
    idx = np.arange(0, len(brain_rows), STRIDE)
    got = masked_rows(coef.cpu().numpy(), brain.mask)[idx].astype(np.float64)
    ref = oracle_rows(oracle, brain, brain_rows[idx], **kw)
    # float32 output: compare at float32 resolution, and the FP64 path itself
    # at 1e-8 through the host entry point on the same rows
    r = rel_rows(got, ref["coef64"])
    assert r.max() <= 1e-6, r.max()
    from cs_dmri_b200 import shore_fit
    sub = np.ascontiguousarray(brain_rows[idx].reshape(len(idx), 1, 1, -1))
    host = shore_fit(sub, brain.bvals, brain.bvecs, np.ones((len(idx), 1, 1), bool), big_delta=brain.big_delta,
                     small_delta=brain.small_delta, return_coef64=True, **kw)
    r = rel_rows(host["coef64"], ref["coef64"])
    assert r.max() <= 1e-8, r.max()
    del d, m, coef
    torch.cuda.empty_cache()


def test_brain300k_positivity_qp_sample(brain, brain_rows, oracle):
    """Configuration 2's amplitude-positivity QP (Goldfarb-Idnani), whole
    volume on the device path, against the oracle on the 9,358-voxel sample: the
    minimiser, feasibility on the constraint sphere and the objective."""
    import torch
    from cs_dmri_b200 import shore_fit, shore_fit_device
    kw = dict(regularization="nonneg", radial_order=6, zeta=700.0)
    d = torch.from_numpy(brain.data).cuda()
    m = torch.from_numpy(brain.mask).cuda()
    coef, _ = shore_fit_device(d, m, brain.bvals, brain.bvecs, big_delta=brain.big_delta,
                               small_delta=brain.small_delta, **kw)
    idx = np.arange(0, len(brain_rows), STRIDE)
    got32 = masked_rows(coef.cpu().numpy(), brain.mask)[idx].astype(np.float64)
    ref = oracle_rows(oracle, brain, brain_rows[idx], **kw)
    sub = np.ascontiguousarray(brain_rows[idx].reshape(len(idx), 1, 1, -1))
    host = shore_fit(sub, brain.bvals, brain.bvecs, np.ones((len(idx), 1, 1), bool), big_delta=brain.big_delta,
                     small_delta=brain.small_delta, return_coef64=True, diagnostics=True, **kw)
    assert rel_rows(got32, host["coef64"]).max() <= 1e-6     # the float32 volume of the same fit
    r = rel_rows(host["coef64"], ref["coef64"])
    assert np.median(r) <= 1e-8 and r.max() <= 1e-5, (np.median(r), r.max())
    M = oracle.design_matrix(brain.bvals, brain.bvecs, 6, 700.0, big_delta=brain.big_delta,
                             small_delta=brain.small_delta)
    Cm = oracle.sh2amp_cart(oracle.odf8_hemisphere(), 6) @ oracle.shore_to_tournier(6, 700.0, 6)
    amp = Cm @ host["coef64"].T
    assert amp.min() >= -1e-7 * max(np.abs(amp).max(), 1.0)
    S = brain_rows[idx].astype(np.float64)
    obj_g = 0.5 * ((host["coef64"] @ M.T - S) ** 2).sum(1)
    obj_o = 0.5 * ((ref["coef64"] @ M.T - S) ** 2).sum(1)
    np.testing.assert_allclose(obj_g, obj_o, rtol=1e-9)
    del d, m, coef
    torch.cuda.empty_cache()


def test_graddev_order8_per_voxel(oracle):
    """Configuration 3's per-voxel designs (gradient deviation, 0-15 % dropped
    samples), radial order 8, on 1,024 voxels: per-voxel relative L2 <= 1e-5,
    iterations within 1, L_v to 1e-12."""
    from cs_dmri_b200.graddev import graddev_phantom, shore_fit_graddev
    V = 1024
    S, bvals, bvecs, T, keep, big, small = graddev_phantom(V, seed=11)
    out = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.01, radial_order=8, big_delta=big,
                            small_delta=small)
    c = out["coefficients"].cpu().numpy()
    it = out["iterations"].cpu().numpy().astype(int)
    lip = out["lipschitz"].cpu().numpy()

    def one(v):
        want, wit, _, M = oracle.graddev_fit(S[v], bvals, bvecs, T[v], keep[v], 0.01, radial_order=8,
                                             big_delta=big, small_delta=small)
        return want, wit, oracle.sigma_max(M) ** 2 / M.shape[0]

    with ThreadPoolExecutor(max_workers=oracle.cpu_count()) as ex:
        res = list(ex.map(one, range(V)))
    want = np.stack([r[0] for r in res])
    wit = np.array([r[1] for r in res])
    wl = np.array([r[2] for r in res])
    np.testing.assert_allclose(lip, wl, rtol=1e-12)
    check_l1(c, want, "graddev order 8")
    assert np.abs(it - wit).max() <= 1 and np.mean(it == wit) >= 0.99
    # the outputs derived from the coefficients: RTOP (GPU map kernel on the
    # GPU fit, the oracle's on the oracle fit) and GFA (GPU ODF sampling
    # against the oracle's), each within the coefficients' 1e-5
    from cs_dmri_b200 import shore_microstructure, shore_odf_peaks
    vol_g = c.astype(np.float32).reshape(V, 1, 1, -1)
    vol_o = want.astype(np.float32).reshape(V, 1, 1, -1)
    m = np.ones((V, 1, 1), bool)
    rt_g = shore_microstructure(vol_g, 8, 700.0, m, outlier_factor=None)["rtop"].ravel()
    rt_o = oracle.shore_microstructure(vol_o, 8, 700.0, m, outlier_factor=None)["rtop"].ravel()
    np.testing.assert_allclose(rt_g, rt_o, rtol=1e-5, atol=1e-6 * np.abs(rt_o).max())
    gfa_g = shore_odf_peaks(vol_g[:256], 8, 700.0)["gfa"].ravel()
    gfa_o = np.array([oracle.odf_peaks(w, 8, 700.0)[0] for w in want[:256]])
    np.testing.assert_allclose(gfa_g, gfa_o, rtol=1e-5, atol=1e-6)
