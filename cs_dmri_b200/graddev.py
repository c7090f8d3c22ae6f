"""SHORE fit with a design matrix per voxel: gradient-deviation tensors and
per-voxel dropped samples.

The reference computes each voxel's effective gradient table from a
deviation tensor T (src/graddev.rs:160-185: q = T^T g, b_eff = b |q|^2,
dir = q / |q|) but its SHORE fit uses one design for the whole volume.  This
fits every voxel on its own table, restricted to the samples it keeps, with
the reference's FISTA and a per-voxel Lipschitz constant: the per-voxel
Gram matrix, its largest eigenvalue and the iterations all run in one
persistent kernel (csd_shore_fit_graddev_device).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _core

__all__ = ["shore_fit_graddev", "graddev_phantom"]


def graddev_phantom(n_voxels, seed=3, sigma=0.02, drop_max=0.15):
    """Synthetic inputs of the per-voxel-design workload: the multi-tensor
    phantom's signals for ``n_voxels`` voxels (CS-DSI table), one deviation
    tensor per voxel T = I + N(0, sigma^2) per entry, and a sample mask that
    drops a fraction U[0, drop_max] of each voxel's diffusion-weighted samples.
    Returns (signals (V, N) float32, bvals, bvecs, T (V, 3, 3), keep (V, N)
    bool, big_delta, small_delta).  The signals are those of the nominal
    table: the deviation enters through the fit's design only."""
    from .phantom import make_phantom
    nx = int(np.ceil(n_voxels / 100.0))
    ph = make_phantom((nx, 10, 10), seed=seed)
    S = np.ascontiguousarray(ph.data.reshape(-1, ph.data.shape[-1])[:n_voxels])
    rng = np.random.default_rng(seed)
    T = np.eye(3)[None] + rng.normal(0.0, sigma, size=(n_voxels, 3, 3))
    dwi = np.flatnonzero(ph.bvals > 50.0)
    frac = rng.uniform(0.0, drop_max, size=n_voxels)
    n_drop = (frac * dwi.size).astype(np.int64)  # at most drop_max of the samples
    order = np.argsort(rng.random((n_voxels, dwi.size)), axis=1)  # a random permutation per voxel
    keep = np.ones(S.shape, bool)
    rows, cols = np.nonzero(np.arange(dwi.size)[None, :] < n_drop[:, None])
    keep[rows, dwi[order[rows, cols]]] = False
    return S, ph.bvals, ph.bvecs, T, keep, ph.big_delta, ph.small_delta


def shore_fit_graddev(signals, bvals, bvecs, graddev=None, sample_mask=None, *, alpha=0.01, radial_order=8,
                      zeta=700.0, big_delta=None, small_delta=None, b0_threshold=50.0, max_iter=1000, tol=1e-6,
                      non_negative=False, device: int = 0, precision: str = "fp64") -> dict:
    """L1 fit (fixed alpha, one per voxel allowed) of ``signals`` (V, N) on
    per-voxel designs.  ``graddev`` (V, 3, 3) deviation tensors (None =
    identity), ``sample_mask`` (V, N) bool of the samples each voxel keeps
    (None = all).  Inputs may be numpy arrays or CUDA tensors; outputs are
    CUDA tensors: ``coefficients`` (V, K) float64, ``iterations``,
    ``converged``, ``lipschitz`` (sigma_max(M_v)^2 / n_v) and ``n_samples``.
    ``precision="fp64-kkt"`` returns every voxel's KKT-certified LASSO
    optimum on its own design instead of the reference FISTA's stopped
    iterate; ``converged`` is then the certificate.  ``"mixed-kkt"`` returns
    the same optimum with the Lanczos estimate and the support iterations in
    FP32 (on the FP32 high part of each voxel's Gram matrix, held as high and
    low FP32 parts) and the polish and certificate in FP64 (on the two parts
    together, 48 bits of the matrix)."""
    import torch

    dev = torch.device("cuda", device)
    S = torch.as_tensor(signals, device=dev).to(torch.float32).contiguous()
    if S.dim() != 2:
        raise ValueError("signals must be (V, N)")
    V, N = S.shape
    g, keep_alive = _core.build_gtab(bvals, bvecs, b0_threshold, big_delta, small_delta)
    if g.n != N:
        raise ValueError(f"signals have {N} samples but the gradient table has {g.n}")
    T = None
    if graddev is not None:
        T = torch.as_tensor(graddev, device=dev).to(torch.float64).reshape(V, 9).contiguous()
    keep = None
    if sample_mask is not None:
        keep = torch.as_tensor(sample_mask, device=dev).to(torch.uint8).contiguous()
        if tuple(keep.shape) != (V, N):
            raise ValueError(f"sample_mask must have shape {(V, N)}")
    alpha_v = None
    if isinstance(alpha, (np.ndarray, torch.Tensor)) and np.ndim(alpha) == 1:
        alpha_v = torch.as_tensor(alpha, device=dev).to(torch.float64).contiguous()
        if alpha_v.shape[0] != V:
            raise ValueError("alpha must be a scalar or one value per voxel")
        alpha = 0.0
    spec = _core.build_spec(radial_order=radial_order, zeta=zeta, regularization="l1", alpha_mode="fixed",
                            alpha=float(alpha), max_iter=max_iter, tol=tol, non_negative=non_negative,
                            precision=precision)
    K = _abi.load().csd_shore_n_coeffs(int(radial_order))
    out = {"coefficients": torch.empty((V, max(K, 0)), dtype=torch.float64, device=dev),
           "iterations": torch.empty(V, dtype=torch.int32, device=dev),
           "converged": torch.empty(V, dtype=torch.uint8, device=dev),
           "lipschitz": torch.empty(V, dtype=torch.float64, device=dev),
           "n_samples": torch.empty(V, dtype=torch.int32, device=dev)}
    err = C.create_string_buffer(4096)
    ptr = (lambda t: None if t is None else t.data_ptr())
    code = _abi.load().csd_shore_fit_graddev_device(
        _abi.handle(device), S.data_ptr(), V, C.byref(g), C.byref(spec), ptr(T), ptr(keep), ptr(alpha_v),
        out["coefficients"].data_ptr(), out["iterations"].data_ptr(), out["converged"].data_ptr(),
        out["lipschitz"].data_ptr(), out["n_samples"].data_ptr(), torch.cuda.current_stream(dev).cuda_stream,
        err, len(err))
    del keep_alive
    _abi.check(code, err)
    out["converged"] = out["converged"].bool()
    return out
