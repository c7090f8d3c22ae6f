"""Per-voxel L1 weight chosen by hypergradient descent on held-out q-samples.

The reference chooses alpha per voxel from a warm-started path (PathBic and
PathL2Anchored, src/solver/alpha.rs:249-318).  This selects it by gradient
instead: a seeded 10 % of the diffusion-weighted samples is held out, the L1
fit runs on the rest, and alpha moves to lower the held-out prediction error
L(alpha) = ||M_ho c(alpha) - s_ho||^2, whose derivative comes from the
implicit adjoint of the fit (dc/dalpha = -n G_SS^-1 sign(c_S), computed by
csd_shore_fit_adjoint_device).  The step on log(alpha) is Rprop's
(Riedmiller & Braun, 1993): each voxel moves by its own step in the
direction opposite the gradient's sign, the step growing x1.2 while the sign
holds and halving when it flips.  Each step's fit starts from the previous
step's coefficients.  The alpha kept is the one with the lowest held-out
error seen; the final fit then uses every sample.

``select_alpha_hypergradient`` runs it on a volume and also scores the
reference's own selections (L2-anchored, the ``cs-fit`` default, and
path-BIC) and the fixed starting alpha on the same held-out samples.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _core
from .autograd import DifferentiableShore

__all__ = ["holdout_split", "HypergradientAlpha", "CapturedHypergradient", "select_alpha_hypergradient"]


def holdout_split(bvals, fraction=0.1, seed=0, b0_threshold=50.0):
    """Indices (train, held_out) of the samples: ``fraction`` of the
    diffusion-weighted samples (b > b0_threshold), chosen by a seeded
    permutation, are held out; b0 samples always train."""
    b = np.asarray(bvals, dtype=np.float64).ravel()
    dwi = np.flatnonzero(b > b0_threshold)
    n_ho = int(round(fraction * dwi.size))
    if not 0 < n_ho < dwi.size:
        raise ValueError(f"holdout fraction {fraction} leaves no held-out or no training samples")
    ho = np.sort(np.random.default_rng(seed).permutation(dwi)[:n_ho])
    train = np.setdiff1d(np.arange(b.size), ho)
    return train, ho


class HypergradientAlpha:
    """Hypergradient alpha selection for batches of voxel signals (float32
    CUDA tensors (V, N) on the full table ``bvals`` / ``bvecs``)."""

    def __init__(self, bvals, bvecs, *, big_delta=None, small_delta=None, b0_threshold=50.0, radial_order=6,
                 zeta=700.0, max_iter=1000, tol=1e-6, holdout_fraction=0.1, seed=0, device: int = 0, handle=None):
        self._args = (bvals, bvecs)
        self._kwargs = dict(big_delta=big_delta, small_delta=small_delta, b0_threshold=b0_threshold,
                            radial_order=radial_order, zeta=zeta, max_iter=max_iter, tol=tol,
                            holdout_fraction=holdout_fraction, seed=seed, device=device)
        self.bvals = np.asarray(bvals, dtype=np.float64).ravel()
        self.bvecs = np.asarray(bvecs, dtype=np.float64).reshape(-1, 3)
        self.train, self.held_out = holdout_split(self.bvals, holdout_fraction, seed, b0_threshold)
        kw = dict(big_delta=big_delta, small_delta=small_delta, b0_threshold=b0_threshold,
                  radial_order=radial_order, zeta=zeta, max_iter=max_iter, tol=tol, device=device, handle=handle)
        self.model = DifferentiableShore(self.bvals[self.train], self.bvecs[self.train], regularization="l1", **kw)
        self.full = DifferentiableShore(self.bvals, self.bvecs, regularization="l1", **kw)
        self.device = self.model.device
        self._idx = None  # sample indices on the device (made once, so a captured run copies nothing from the host)

    def capture(self, signals: torch.Tensor, **kw) -> "CapturedHypergradient":
        """The whole run (``run``'s keyword arguments) as one CUDA graph
        over ``signals``; see ``CapturedHypergradient``."""
        return CapturedHypergradient(self, signals, **kw)

    def heldout_loss(self, coef: torch.Tensor, s_ho: torch.Tensor) -> torch.Tensor:
        """Per-voxel squared prediction error on the held-out samples."""
        pred = self.model.predict(coef, self.bvals[self.held_out], self.bvecs[self.held_out])
        return (pred - s_ho).square().sum(1)

    def split(self, signals: torch.Tensor):
        """(training samples float32, held-out samples float64) of each voxel."""
        if self._idx is None or self._idx[0].device != signals.device:
            self._idx = (torch.as_tensor(self.train, device=signals.device),
                         torch.as_tensor(self.held_out, device=signals.device))
        tr, ho = self._idx
        return signals.index_select(1, tr).contiguous(), signals.index_select(1, ho).to(torch.float64)

    def run(self, signals: torch.Tensor, *, alpha0=0.01, steps=8, step0=0.5, alpha_range=(1e-3, 1e3)):
        """Returns (alpha (V,), held-out loss at that alpha (V,), the loss at
        alpha0 (V,), the per-step history of (alpha, loss, d loss / d ln alpha))."""
        s_tr, s_ho = self.split(signals)
        V = signals.shape[0]
        f64 = dict(dtype=torch.float64, device=self.device)
        alpha = torch.full((V,), float(alpha0), **f64)
        lo, hi = float(alpha0) * alpha_range[0], float(alpha0) * alpha_range[1]
        eta = torch.full((V,), float(step0), **f64)
        prev = torch.zeros(V, **f64)
        best_alpha, best_loss, loss0, warm, hist = alpha.clone(), None, None, None, []
        for t in range(int(steps)):
            a = alpha.clone().requires_grad_(True)
            c = self.model.fit(s_tr, a, warm=warm)
            loss = self.heldout_loss(c, s_ho)
            loss.sum().backward()
            g = a.grad * alpha  # d loss / d ln(alpha), per voxel
            loss = loss.detach()
            if best_loss is None:
                best_loss, loss0 = loss.clone(), loss.clone()
            better = loss < best_loss
            best_alpha = torch.where(better, alpha, best_alpha)
            best_loss = torch.where(better, loss, best_loss)
            hist.append((alpha.clone(), loss, g.detach()))
            sgn = torch.sign(g.detach())
            agree = sgn * prev
            eta = torch.where(agree > 0, eta * 1.2, torch.where(agree < 0, eta * 0.5, eta))
            alpha = (alpha * torch.exp(-eta * sgn)).clamp(lo, hi)
            prev = torch.where(agree < 0, torch.zeros_like(sgn), sgn)
            warm = c.detach()
        return best_alpha, best_loss, loss0, hist


class CapturedHypergradient:
    """``HypergradientAlpha.run`` captured in one CUDA graph: every fit,
    held-out prediction, adjoint and step of the run, replayed by
    ``replay()`` on the current contents of the signal tensor it was captured
    with.  ``outputs`` are that run's (alpha, loss, loss at alpha0) tensors,
    rewritten by each replay.  The run uses a library handle of its own, so
    no other call can free or resize the scratch memory the graph's kernels
    point at; the handle lives as long as this object."""

    def __init__(self, selector: "HypergradientAlpha", signals: torch.Tensor, **kw):
        from . import _abi
        self._handle = _abi.PrivateHandle(selector._kwargs["device"])
        self.selector = HypergradientAlpha(*selector._args, **selector._kwargs, handle=self._handle)
        self.signals = signals
        side = torch.cuda.Stream(signals.device)
        side.wait_stream(torch.cuda.current_stream(signals.device))
        with torch.cuda.stream(side):  # one untimed run sizes every buffer before capture
            self.selector.run(signals, **kw)
        torch.cuda.current_stream(signals.device).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            best, loss, loss0, _ = self.selector.run(signals, **kw)
        self.outputs = (best, loss, loss0)

    def replay(self):
        self.graph.replay()
        return self.outputs

    def __del__(self):
        self.graph = None  # the graph goes before the handle whose memory it uses
        self.selector = None


def select_alpha_hypergradient(data, bvals, bvecs, mask, *, big_delta=None, small_delta=None, b0_threshold=50.0,
                               radial_order=6, zeta=700.0, alpha0=0.01, steps=8, holdout_fraction=0.1, seed=0,
                               npeaks=3, compare_reference=True, device: int = 0) -> dict:
    """The whole pipeline on a volume: hypergradient alpha per voxel, the
    final L1 fit on every sample, ODF peaks and GFA (3 peaks), RTOP and MSD;
    with ``compare_reference`` the held-out error of the reference's own
    selections (L2-anchored and path-BIC on the training samples) and of the
    fixed alpha0, all on the same held-out samples.

    Returns a dict of volumes (``alpha``, ``coefficients``, ``gfa``,
    ``peak_dirs``, ``peak_values``, ``rtop``, ``msd``, ``heldout_loss``) and
    ``comparison`` (median held-out error per method)."""
    data = np.asarray(data)
    mask = np.asarray(mask).astype(bool)
    X, Y, Z, N = data.shape
    sel = HypergradientAlpha(bvals, bvecs, big_delta=big_delta, small_delta=small_delta, b0_threshold=b0_threshold,
                             radial_order=radial_order, zeta=zeta, holdout_fraction=holdout_fraction, seed=seed,
                             device=device)
    rows = np.flatnonzero(mask.ravel())  # masked voxels in x-y-z order
    flat = torch.from_numpy(np.ascontiguousarray(data.reshape(-1, N), dtype=np.float32))
    S = flat.index_select(0, torch.from_numpy(rows)).to(sel.device)  # a gather on all host threads
    alpha, loss, loss0, _ = sel.run(S, alpha0=alpha0, steps=steps)
    coef = sel.full.fit(S, alpha).detach()
    K = coef.shape[1]
    # the volumes are assembled on the device and copied back once each
    idx = torch.from_numpy(rows).to(sel.device)

    def volume(v: torch.Tensor, width: int) -> np.ndarray:
        full = torch.zeros((X * Y * Z, width), dtype=torch.float32, device=sel.device)
        full.index_copy_(0, idx, v.reshape(-1, width).to(torch.float32))
        return full.cpu().numpy().reshape((X, Y, Z) + ((width,) if width > 1 else ()))

    vol = volume(coef, K)
    out = {"alpha": volume(alpha, 1), "heldout_loss": volume(loss, 1),
           "coefficients": vol, "train_samples": sel.train, "heldout_samples": sel.held_out}
    pk = _core.shore_odf_peaks(vol, radial_order, zeta, mask, npeaks=npeaks, device=device)
    out.update(gfa=pk["gfa"], peak_dirs=pk["peak_dirs"], peak_values=pk["peak_values"])
    micro = _core.shore_microstructure(vol, radial_order, zeta, mask, units="mm", outlier_factor=None,
                                       device=device)
    out.update(rtop=micro["rtop"], msd=micro["msd"])
    comp = {"hypergradient": float(np.median(loss.cpu().numpy())), "fixed_alpha0": float(np.median(loss0.cpu().numpy()))}
    if compare_reference:
        s_tr, s_ho = sel.split(S)
        tr = np.zeros((int(mask.sum()), 1, 1, sel.train.size), np.float32)
        tr[:, 0, 0] = s_tr.cpu().numpy()
        ones = np.ones(tr.shape[:3], bool)
        for mode in ("l2-anchored", "path-bic"):
            r = _core.shore_fit(tr, sel.bvals[sel.train], sel.bvecs[sel.train], ones, big_delta=big_delta,
                                small_delta=small_delta, b0_threshold=b0_threshold, radial_order=radial_order,
                                zeta=zeta, regularization="l1", alpha_mode=mode, return_coef64=True, device=device)
            c = torch.from_numpy(r["coef64"]).to(sel.device)
            comp[mode] = float(np.median(sel.heldout_loss(c, s_ho).cpu().numpy()))
    out["comparison"] = comp
    return out
