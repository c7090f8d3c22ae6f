"""Differentiable SHORE fit on the GPU.

The reference computes no derivatives.  This module differentiates the
solution maps of its solvers - the LASSO fit of src/solver/fista.rs:70-143 and
the Tikhonov fit of src/solver/tikhonov.rs:26-76 - and the maps taken on their
coefficients (RTOP, src/scalars/microstructure.rs:98-118; ODF amplitudes on a
sphere, src/odf.rs:79-102; predicted signals, src/synth.rs:15-84), each as a
``torch.autograd.Function`` whose forward and backward run in libcsdshore.so:

* fit: ``csd_shore_fit_batch_device`` forward (the volume fit's kernels), and
  ``csd_shore_fit_adjoint_device`` backward - implicit differentiation on the
  converged support for L1 (w_S = G_SS^-1 g_S, grad_s = M w,
  grad_alpha = -N sign(c_S) . w_S), the transpose solve with the shared
  Cholesky factor for L2;
* RTOP: ``csd_shore_rtop_device`` / ``csd_shore_rtop_adjoint_device``;
* ODF amplitudes and predicted signals: ``csd_apply_rows_device`` with the
  matrix, and with its transpose for the adjoint.

Example::

    model = DifferentiableShore(bvals, bvecs, big_delta=0.0431, small_delta=0.0107)
    alpha = torch.tensor(0.01, dtype=torch.float64, device="cuda", requires_grad=True)
    c = model.fit(signals, alpha)          # (V, K) float64
    loss = model.rtop(c).sum() + model.odf(c).square().mean()
    loss.backward()                        # signals.grad (float32), alpha.grad

Signals are float32 CUDA tensors (V, N), coefficients float64 (V, K).  The
derivative of the L1 fit is that of the exact minimiser on the support the
iterations converged to; it is the derivative of the returned coefficients up
to the fit's own tolerance.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi, _core

__all__ = ["DifferentiableShore", "geodesic_sphere"]


def geodesic_sphere(frequency: int = 6, hemisphere: bool = False) -> np.ndarray:
    """Unit vertices (count, 3) of the class I geodesic sphere of
    ``frequency`` (10 f^2 + 2 vertices; 362 at the default 6)."""
    lib = _abi.load()
    n = lib.csd_geodesic_sphere(int(frequency), int(bool(hemisphere)), None, 0)
    if n < 0:
        raise ValueError(f"frequency must be in 1..64, got {frequency}")
    out = np.zeros((n, 3))
    lib.csd_geodesic_sphere(int(frequency), int(bool(hemisphere)), out.ctypes.data, n)
    return out


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _call(fn, *args) -> str:
    err = C.create_string_buffer(4096)
    _abi.check(fn(*args, err, len(err)), err)
    return err.value.decode("utf-8", "replace")


def _ptr(t):
    return None if t is None else t.data_ptr()


class _Fit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, signals, hyper, model, warm):
        spec = model._spec_for(hyper)
        coef = model._fit_raw(signals, hyper, spec, warm)
        ctx.model, ctx.spec, ctx.hyper_shape = model, spec, tuple(hyper.shape)
        ctx.save_for_backward(coef)
        return coef

    @staticmethod
    def backward(ctx, grad):
        (coef,) = ctx.saved_tensors
        model = ctx.model
        gs, gh = model._adjoint_raw(coef, grad, ctx.spec, signal32=ctx.needs_input_grad[0])
        ghyp = None
        if ctx.needs_input_grad[1]:
            if model.regularization == "l1":
                ghyp = gh[:, 0] if len(ctx.hyper_shape) == 1 else gh[:, 0].sum().reshape(ctx.hyper_shape)
            else:
                ghyp = gh.sum(0)
        return gs, ghyp, None, None


class _Apply(torch.autograd.Function):
    """out = in A^T for a fixed matrix A (rows, cols)."""

    @staticmethod
    def forward(ctx, x, A, At, model):
        ctx.model, ctx.A = model, A
        return model._apply_raw(At, A.shape[0], A.shape[1], x)

    @staticmethod
    def backward(ctx, grad):
        A = ctx.A
        return ctx.model._apply_raw(A, A.shape[1], A.shape[0], grad), None, None, None


class _Rtop(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coef, model):
        ctx.model = model
        ctx.save_for_backward(coef)
        return model._rtop_raw(coef)

    @staticmethod
    def backward(ctx, grad):
        (coef,) = ctx.saved_tensors
        return ctx.model._rtop_adjoint_raw(coef, grad), None


class DifferentiableShore:
    """SHORE fit of a batch of voxel signals with gradients.

    Keyword arguments follow ``_cs_dmri.shore_fit`` (python/src/models.rs:70-76):
    ``radial_order``, ``zeta``, ``regularization`` ("l1" or "l2"),
    ``max_iter``, ``tol``, ``non_negative``, ``precision``; the gradient
    table is ``bvals``, ``bvecs``, ``big_delta``, ``small_delta``,
    ``b0_threshold``.  L1 fits take a fixed alpha (one, or one per voxel).
    ``handle`` (an ``_abi.PrivateHandle``) gives the model library scratch of
    its own instead of the device's shared handle.  ``schedule="previous"``
    (the default) has each L1 fit of a batch take its voxels up in decreasing
    iteration count of the model's previous fit of a batch of the same size
    (repeated fits of one batch - training loops, hypergradient steps - then
    have no late-starting slow voxels); ``"index"`` keeps voxel order.  The
    results are the same either way."""

    def __init__(self, bvals, bvecs, *, big_delta=None, small_delta=None, b0_threshold=50.0, radial_order=6,
                 zeta=700.0, regularization="l1", max_iter=1000, tol=1e-6, non_negative=False, precision="fp64",
                 allow_single_shell=False, device: int = 0, handle=None, schedule="previous"):
        if regularization not in ("l1", "l2"):
            raise ValueError(f"regularization must be l1 or l2 for the differentiable fit, got {regularization!r}")
        self.regularization = regularization
        self.radial_order, self.zeta = int(radial_order), float(zeta)
        self.bvals = np.asarray(bvals, dtype=np.float64).ravel()
        self.bvecs = np.asarray(bvecs, dtype=np.float64).reshape(-1, 3)
        self.big_delta, self.small_delta, self.b0_threshold = big_delta, small_delta, b0_threshold
        self._g, self._keep = _core.build_gtab(self.bvals, self.bvecs, b0_threshold, big_delta, small_delta)
        self.N = int(self._g.n)
        self.K = _abi.load().csd_shore_n_coeffs(self.radial_order)
        if self.K <= 0:
            raise ValueError("radial_order must be a positive even integer")
        self._kw = dict(radial_order=self.radial_order, zeta=self.zeta, regularization=regularization,
                        alpha_mode="fixed", max_iter=max_iter, tol=tol, non_negative=non_negative,
                        precision=precision, allow_single_shell=allow_single_shell)
        self.device_index = int(device)
        self.device = torch.device("cuda", self.device_index)
        self._mats: dict = {}
        self._singular = torch.zeros(1, dtype=torch.int64, device=self.device)
        self._private = handle  # an _abi.PrivateHandle, or None for the process-wide handle of the device
        if schedule not in ("previous", "index"):
            raise ValueError(f"schedule must be 'previous' or 'index', got {schedule!r}")
        self.schedule = schedule
        self._iters = None  # iteration counts of the last L1 fit (int32, one per voxel)

    # ---------------------------------------------------------------- public
    def fit(self, signals: torch.Tensor, alpha=None, *, lambda_n=None, lambda_l=None, warm=None) -> torch.Tensor:
        """Coefficients (V, K) float64 of ``signals`` (V, N) float32.

        L1: ``alpha`` a float, a 0-d float64 tensor or a (V,) float64 tensor
        (one per voxel); gradients flow to it when it requires grad.  L2:
        ``lambda_n`` / ``lambda_l`` floats or 0-d tensors (defaults 1e-8).
        ``warm`` (V, K) float64 starts the L1 iterations (no gradient)."""
        self._check_signals(signals)
        if self.regularization == "l1":
            if alpha is None:
                raise ValueError("the L1 fit needs alpha")
            hyper = self._as_f64(alpha)
            if hyper.dim() not in (0, 1) or (hyper.dim() == 1 and hyper.shape[0] != signals.shape[0]):
                raise ValueError("alpha must be a scalar or one value per voxel")
        else:
            ln = self._as_f64(1e-8 if lambda_n is None else lambda_n)
            ll = self._as_f64(1e-8 if lambda_l is None else lambda_l)
            if ln.dim() != 0 or ll.dim() != 0:
                raise ValueError("lambda_n and lambda_l must be scalars")
            hyper = torch.stack([ln, ll])
        if warm is not None:
            if self.regularization != "l1":
                raise ValueError("warm starts apply to the L1 fit")
            warm = warm.detach().to(self.device, torch.float64).contiguous()
            if tuple(warm.shape) != (signals.shape[0], self.K):
                raise ValueError(f"warm must have shape {(signals.shape[0], self.K)}")
        return _Fit.apply(signals, hyper, self, warm)

    def rtop(self, coef: torch.Tensor) -> torch.Tensor:
        """RTOP (V,) of coefficients (V, K), millimetre units."""
        return _Rtop.apply(self._check_coef(coef), self)

    def odf(self, coef: torch.Tensor, directions=None) -> torch.Tensor:
        """ODF amplitudes (V, R) on ``directions`` (R, 3); default: the
        362-vertex geodesic sphere."""
        key = ("odf", None if directions is None else np.asarray(directions, dtype=np.float64).tobytes())
        if key not in self._mats:
            d = geodesic_sphere(6) if directions is None else np.ascontiguousarray(directions, dtype=np.float64)
            A = np.zeros((len(d), self.K))
            _call(_abi.load().csd_shore_odf_matrix, self._handle(), self.radial_order, self.zeta,
                  d.ctypes.data, len(d), A.ctypes.data)
            self._mats[key] = self._device_pair(A)
        A, At = self._mats[key]
        return _Apply.apply(self._check_coef(coef), A, At, self)

    def predict(self, coef: torch.Tensor, bvals, bvecs) -> torch.Tensor:
        """Signals (V, N_target) the coefficients predict on a target table
        (the fit's big / small delta and b0 threshold)."""
        bv = np.asarray(bvals, dtype=np.float64).ravel()
        bc = np.asarray(bvecs, dtype=np.float64).reshape(-1, 3)
        key = ("predict", bv.tobytes(), bc.tobytes())
        if key not in self._mats:
            A = _core.design_matrix(bv, bc, self.radial_order, self.zeta, big_delta=self.big_delta,
                                    small_delta=self.small_delta, b0_threshold=self.b0_threshold,
                                    device=self.device_index)
            self._mats[key] = self._device_pair(A)
        A, At = self._mats[key]
        return _Apply.apply(self._check_coef(coef), A, At, self)

    def signal_gradient(self, coef: torch.Tensor, grad_coef: torch.Tensor, *, alpha=None, lambda_n=1e-8,
                        lambda_l=1e-8):
        """FP64 adjoint outside autograd: (grad on the signals (V, N) float64,
        per-voxel hyper-parameter gradients (V, 2)) for coefficients ``coef``
        and an upstream gradient ``grad_coef``."""
        hyper = self._as_f64(0.0 if alpha is None else alpha) if self.regularization == "l1" else \
            torch.stack([self._as_f64(lambda_n), self._as_f64(lambda_l)])
        spec = self._spec_for(hyper)
        return self._adjoint_raw(self._check_coef(coef).detach(), grad_coef, spec, signal32=False, signal64=True)

    # -------------------------------------------------------------- internals
    def _handle(self):
        return self._private.h if self._private is not None else _abi.handle(self.device_index)

    def _as_f64(self, v) -> torch.Tensor:
        if isinstance(v, torch.Tensor):
            return v.to(self.device, torch.float64)
        return torch.tensor(float(v), dtype=torch.float64, device=self.device)

    def _check_signals(self, s: torch.Tensor) -> None:
        if not (isinstance(s, torch.Tensor) and s.is_cuda and s.dtype == torch.float32 and s.dim() == 2):
            raise ValueError("signals must be a float32 CUDA tensor (V, N)")
        if s.shape[1] != self.N:
            raise ValueError(f"signals have {s.shape[1]} samples but the gradient table has {self.N}")

    def _check_coef(self, c: torch.Tensor) -> torch.Tensor:
        if not (isinstance(c, torch.Tensor) and c.is_cuda and c.dtype == torch.float64 and c.dim() == 2
                and c.shape[1] == self.K):
            raise ValueError(f"coefficients must be a float64 CUDA tensor (V, {self.K})")
        return c

    def _device_pair(self, A: np.ndarray):
        At = torch.from_numpy(np.ascontiguousarray(A.T)).to(self.device)
        return torch.from_numpy(np.ascontiguousarray(A)).to(self.device), At

    def _spec_for(self, hyper: torch.Tensor) -> _abi.Spec:
        kw = dict(self._kw)
        if self.regularization == "l1":
            kw["alpha"] = 0.0  # the fit reads alpha per voxel from the device (no host round trip)
        else:
            h = hyper.detach().cpu().numpy()
            kw["lambda_n"], kw["lambda_l"] = float(h[0]), float(h[1])
        return _core.build_spec(**kw)

    def _fit_raw(self, signals, hyper, spec, warm) -> torch.Tensor:
        s = signals.detach().contiguous()
        V = s.shape[0]
        alpha_v = hyper.detach().expand(V).contiguous() if self.regularization == "l1" else None
        coef = torch.empty((V, self.K), dtype=torch.float64, device=self.device)
        order = None
        if self.regularization == "l1" and self.schedule == "previous":
            # voxels in decreasing iteration count of this model's previous fit of a batch this size
            if self._iters is not None and self._iters.shape[0] == V:
                order = torch.argsort(self._iters, descending=True, stable=True)
            else:
                self._iters = torch.zeros(V, dtype=torch.int32, device=self.device)
        lib = _abi.load()
        _call(lib.csd_shore_fit_batch_device, self._handle(), s.data_ptr(), V, C.byref(self._g),
              C.byref(spec), _ptr(alpha_v), _ptr(warm), _ptr(order), coef.data_ptr(),
              _ptr(self._iters if self.schedule == "previous" and self.regularization == "l1" else None), _stream(s))
        return coef

    def _adjoint_raw(self, coef, grad, spec, *, signal32=True, signal64=False):
        g = grad.detach().to(self.device, torch.float64).contiguous()
        V = coef.shape[0]
        gs32 = torch.empty((V, self.N), dtype=torch.float32, device=self.device) if signal32 else None
        gs64 = torch.empty((V, self.N), dtype=torch.float64, device=self.device) if signal64 else None
        gh = torch.empty((V, 2), dtype=torch.float64, device=self.device)
        _call(_abi.load().csd_shore_fit_adjoint_device, self._handle(), C.byref(self._g),
              C.byref(spec), coef.contiguous().data_ptr(), g.data_ptr(), V, _ptr(gs32), _ptr(gs64),
              gh.data_ptr(), _ptr(self._singular), _stream(g))
        return (gs64 if signal64 else gs32), gh

    @property
    def singular_voxels(self) -> int:
        """Voxels, over every backward pass so far, whose support Gram matrix
        was not positive definite (their gradients are NaN)."""
        return int(self._singular.item())

    def _apply_raw(self, At, rows, cols, x) -> torch.Tensor:
        x = x.detach().to(self.device, torch.float64).contiguous()
        out = torch.empty((x.shape[0], rows), dtype=torch.float64, device=self.device)
        _call(_abi.load().csd_apply_rows_device, self._handle(), At.data_ptr(), rows, cols,
              x.data_ptr(), x.shape[0], out.data_ptr(), _stream(x))
        return out

    def _rtop_raw(self, coef) -> torch.Tensor:
        c = coef.detach().contiguous()
        out = torch.empty(c.shape[0], dtype=torch.float64, device=self.device)
        _call(_abi.load().csd_shore_rtop_device, self._handle(), self.radial_order, self.zeta,
              c.data_ptr(), c.shape[0], out.data_ptr(), _stream(c))
        return out

    def _rtop_adjoint_raw(self, coef, grad) -> torch.Tensor:
        c = coef.detach().contiguous()
        g = grad.detach().to(self.device, torch.float64).contiguous()
        out = torch.empty_like(c)
        _call(_abi.load().csd_shore_rtop_adjoint_device, self._handle(), self.radial_order,
              self.zeta, c.data_ptr(), c.shape[0], g.data_ptr(), out.data_ptr(), _stream(c))
        return out
