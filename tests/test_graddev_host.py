"""Per-voxel designs, host side: the oracle's effective table
(src/graddev.rs:160-185) and the synthetic inputs of the workload."""

import numpy as np


def test_effective_table(oracle):
    from cs_dmri_b200.phantom import gradient_table
    bvals, bvecs = gradient_table(1)
    b, d = oracle.effective_table(bvals, bvecs, np.eye(3))
    np.testing.assert_allclose(b, bvals, rtol=1e-15)
    dwi = bvals > 50
    np.testing.assert_allclose(d[dwi], bvecs[dwi], atol=1e-15)
    b2, d2 = oracle.effective_table(bvals, bvecs, 2.0 * np.eye(3))
    np.testing.assert_allclose(b2[dwi], 4.0 * bvals[dwi], rtol=1e-14)
    np.testing.assert_allclose(d2[dwi], bvecs[dwi], atol=1e-15)
    assert np.array_equal(b2[~dwi], bvals[~dwi])
    R = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])  # q = R^T g
    b3, d3 = oracle.effective_table(bvals, bvecs, R)
    np.testing.assert_allclose(b3, bvals, rtol=1e-14)
    np.testing.assert_allclose(d3[dwi], bvecs[dwi] @ R, atol=1e-15)


def test_graddev_phantom():
    from cs_dmri_b200.graddev import graddev_phantom
    S, bvals, bvecs, T, keep, big, small = graddev_phantom(250, seed=5)
    assert S.shape == (250, bvals.size) and S.dtype == np.float32
    assert T.shape == (250, 3, 3) and abs(T.mean() - 1.0 / 3.0) < 0.01 and 0.01 < (T - np.eye(3)).std() < 0.03
    dwi = bvals > 50
    assert np.all(keep[:, ~dwi])
    drop = 1.0 - keep[:, dwi].mean(1)
    assert drop.max() <= 0.15 + 1e-9 and drop.min() >= 0.0 and drop.mean() > 0.03
    S2, *_ = graddev_phantom(250, seed=5)
    assert np.array_equal(S, S2)
