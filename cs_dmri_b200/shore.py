"""3D-SHORE model and fit objects with the reference's Python interface
(``cs_dmri.ShoreModel`` / ``cs_dmri.ShoreFit``, python/cs_dmri/shore.py:25-299),
fitted by the CUDA library."""

from __future__ import annotations

import json
import warnings
from pathlib import Path

import numpy as np

from . import _core
from .gradients import as_gradient_table

__all__ = ["ShoreModel", "ShoreFit"]

_REGULARIZATIONS = ("l1", "l2", "nonneg")
_ALPHA_MODES = ("l2-anchored", "path-bic", "alpha-ratio", "fixed")
_FRAMES = ("auto", "world", "image")


def _fit_frame(bvec_frame: str, affine):
    """("world" | "image", R) with R rotating image-axis vectors into the fit
    frame (python/cs_dmri/_frame.py:13-31)."""
    if bvec_frame not in _FRAMES:
        raise ValueError(f"bvec_frame must be one of {_FRAMES}, got {bvec_frame!r}")
    if bvec_frame == "auto":
        bvec_frame = "world" if affine is not None else "image"
    if bvec_frame == "world":
        if affine is None:
            raise ValueError("bvec_frame='world' needs an affine (fit a DWI, or pass affine=)")
        return "world", _core.affine_rotation(np.asarray(affine, dtype=np.float64))
    return "image", np.eye(3)


def _stem(path: Path) -> str:
    """foo.nii.gz -> foo, foo.nii -> foo (src/io/coeffs.rs:152-160)."""
    return str(path)[: -len(".nii.gz")] if str(path).endswith(".nii.gz") else str(path.with_suffix(""))


def _rotate(vectors, R):
    return np.ascontiguousarray(np.asarray(vectors, dtype=np.float64) @ R.T)


class ShoreModel:
    """3D-SHORE model (Merlet & Deriche 2013; Ozarslan et al. 2013).

    Same parameters and defaults as ``cs_dmri.ShoreModel``: ``radial_order``
    (even; 6 gives 72 coefficients), ``zeta`` (700), ``regularization`` in
    ``{"l1", "l2", "nonneg"}``, ``alpha_mode`` in ``{"l2-anchored",
    "path-bic", "alpha-ratio", "fixed"}``, the L1 path settings, the Tikhonov
    weights ``lambda_n`` / ``lambda_l``, the amplitude-ICLS settings,
    ``bvec_frame`` and ``allow_single_shell``.  ``device`` picks the GPU.
    """

    def __init__(self, gtab, *, radial_order: int = 6, zeta: float = 700.0, regularization: str = "l1",
                 alpha_mode: str = "l2-anchored", alpha: float = 1.0, alpha_ratio: float = 1e-3,
                 path_n_alphas: int = 20, path_eps: float | None = None, slack: float = 0.05,
                 max_iter: int = 1000, tol: float = 1e-6, non_negative: bool = False,
                 lambda_n: float = 1e-8, lambda_l: float = 1e-8, nonneg_max_iter: int = 200,
                 nonneg_tol: float = 1e-9, nonneg_epsilon: float = 1e-10, bvec_frame: str = "auto",
                 allow_single_shell: bool = False, device: int = 0, precision: str = "fp64"):
        if regularization not in _REGULARIZATIONS:
            raise ValueError(f"regularization must be one of {_REGULARIZATIONS}, got {regularization!r}")
        if alpha_mode not in _ALPHA_MODES:
            raise ValueError(f"alpha_mode must be one of {_ALPHA_MODES}, got {alpha_mode!r}")
        self.gtab = as_gradient_table(gtab)
        self.radial_order = radial_order
        self.zeta = zeta
        self.regularization = regularization
        self.bvec_frame = bvec_frame
        self.device = device
        self._solver = dict(
            alpha_mode=alpha_mode, alpha=alpha, alpha_ratio=alpha_ratio, path_n_alphas=path_n_alphas,
            path_eps=path_eps, slack=slack, max_iter=max_iter, tol=tol, non_negative=non_negative,
            lambda_n=lambda_n, lambda_l=lambda_l, nonneg_max_iter=nonneg_max_iter, nonneg_tol=nonneg_tol,
            nonneg_epsilon=nonneg_epsilon, allow_single_shell=allow_single_shell, precision=precision)

    def fit(self, data, mask=None, *, affine=None, diagnostics: bool = True,
            n_threads: int | None = None) -> "ShoreFit":
        """Fit every voxel in ``mask`` ((X, Y, Z) bool; required for arrays)."""
        vol = np.asarray(data, dtype=np.float32)
        if vol.ndim != 4:
            raise ValueError(f"expected a 4-D (X, Y, Z, N) array, got shape {vol.shape}")
        if mask is None:
            raise ValueError("a mask is required")
        m = np.asarray(mask)
        if m.dtype != bool:
            m = m > 0
        if m.shape != vol.shape[:3]:
            raise ValueError(f"mask shape {m.shape} does not match data spatial shape {vol.shape[:3]}")
        affine = None if affine is None else np.asarray(affine, dtype=np.float64)
        frame, R = _fit_frame(self.bvec_frame, affine)
        out = _core.shore_fit(
            vol, self.gtab.bvals, _rotate(self.gtab.bvecs, R), m,
            big_delta=self.gtab.big_delta, small_delta=self.gtab.small_delta,
            b0_threshold=self.gtab.b0_threshold,
            bvec_frame="world-ras" if frame == "world" else "image-axis",
            radial_order=self.radial_order, zeta=self.zeta, regularization=self.regularization,
            diagnostics=diagnostics, n_threads=n_threads, device=self.device, **self._solver)
        for message in out.pop("warnings", ()):
            warnings.warn(message, stacklevel=2)
        return ShoreFit(out, model=self, mask=m, affine=affine, frame=frame, rotation=R)


class ShoreFit:
    """Result of :meth:`ShoreModel.fit`: ``coefficients`` (X, Y, Z, K) float32,
    the diagnostic maps (``r2, rmse, residual_l2, iterations,
    regularization_kind``, and ``alpha, bic, rss_l2`` where the solver has
    them), ``sidecar`` and ``frame``."""

    def __init__(self, arrays: dict, *, model=None, mask=None, affine=None, frame="image", rotation=None):
        self.coefficients = arrays["coefficients"]
        self.sidecar = arrays["sidecar"]
        self.alpha_distribution = arrays.get("alpha_distribution")
        for k in ("r2", "rmse", "residual_l2", "iterations", "regularization_kind", "alpha", "bic", "rss_l2"):
            setattr(self, k, arrays.get(k))
        self.model = model
        self.mask = mask if mask is not None else np.any(self.coefficients != 0, axis=-1)
        self.affine = affine
        self.frame = frame
        self._rotation = np.eye(3) if rotation is None else rotation
        basis = self.sidecar["basis"]
        self.radial_order = int(basis["radial_order"])
        self.zeta = float(basis["zeta"])

    @property
    def dwi_shells(self):
        shells = self.sidecar.get("dwi_shells")
        return None if shells is None else [float(b) for b in shells]

    @property
    def single_shell(self) -> bool:
        return self.dwi_shells is not None and len(self.dwi_shells) < 2

    @property
    def sparsity(self) -> np.ndarray:
        """Fraction of non-zero coefficients per voxel (L1 sparsity)."""
        out = np.zeros(self.coefficients.shape[:3], np.float32)
        out[self.mask] = (self.coefficients[self.mask] != 0).mean(-1)
        return out

    def odf_sh(self, lmax: int | None = None, *, n_threads=None) -> np.ndarray:
        """Tournier (MRtrix) SH coefficients of the ODF, (X, Y, Z, n_sh);
        ``lmax`` defaults to the largest even value <= the radial order
        (python/cs_dmri/shore.py:152-157)."""
        lmax = self.radial_order - self.radial_order % 2 if lmax is None else lmax
        return _core.shore_odf_sh(self.coefficients, self.radial_order, self.zeta, lmax, self.mask, n_threads=n_threads)

    def predict(self, gtab=None, *, clip: bool = True, n_threads=None) -> np.ndarray:
        """Signal for ``gtab`` (default: the fit's own), (X, Y, Z, N); ``gtab``
        is in the image's voxel-axis frame and is rotated into the fit frame
        (python/cs_dmri/shore.py:159-181)."""
        if gtab is None:
            if self.model is None:
                raise ValueError("pass a gradient table: this fit has no model")
            gtab = self.model.gtab
        gtab = as_gradient_table(gtab)
        if self.single_shell:
            fitted = self.dwi_shells[0]
            dw = gtab.bvals[gtab.bvals > gtab.b0_threshold]
            if np.any(np.abs(dw - fitted) > 50):
                warnings.warn(
                    f"this fit used a single shell (b = {fitted:.0f}); signals at other b-values are "
                    "extrapolated by the regularization, not the measurements", stacklevel=2)
        out = _core.shore_predict(self.coefficients, self.radial_order, self.zeta, gtab.bvals,
                                  _rotate(gtab.bvecs, self._rotation), big_delta=self.sidecar["big_delta_seconds"],
                                  small_delta=self.sidecar["small_delta_seconds"], n_threads=n_threads)
        return np.maximum(out, 0) if clip else out

    def peaks(self, *, npeaks: int = 5, relative_peak_threshold: float = 0.5, min_separation_angle: float = 25.0,
              sphere_frequency: int = 6) -> dict:
        """GFA and ODF peaks inside the mask (``shore_odf_peaks``; the
        quantities of the reference's ODX export, src/io/odx_out.rs:1008-1090).
        Peak directions are returned in the image's voxel-axis frame."""
        out = _core.shore_odf_peaks(self.coefficients, self.radial_order, self.zeta, self.mask,
                                    sphere_frequency=sphere_frequency, npeaks=npeaks,
                                    relative_peak_threshold=relative_peak_threshold,
                                    min_separation_angle=min_separation_angle)
        d = out["peak_dirs"]
        out["peak_dirs"] = _rotate(d.reshape(-1, 3), self._rotation.T).reshape(d.shape).astype(np.float32)
        return out

    def microstructure(self, directions=None, *, units: str = "um", outlier_factor: float | None = 10.0,
                       n_threads=None) -> dict:
        """RTOP, RTAP, RTPP, MSD, QIV and NG maps (python/cs_dmri/shore.py:183-205).
        RTAP / RTPP need ``directions`` (X, Y, Z, 3) in the image's voxel-axis
        frame; without them they are NaN.  Raises ``ValueError`` for a
        single-shell fit, whose radial decay the data do not determine."""
        if self.single_shell:
            raise ValueError(
                "propagator-derived scalars are not determined by single-shell data "
                f"(this fit used b = {self.dwi_shells[0]:.0f} only)")
        if directions is not None:
            directions = _rotate(directions, self._rotation).astype(np.float32)
        return _core.shore_microstructure(self.coefficients, self.radial_order, self.zeta, self.mask, directions,
                                          units=units, outlier_factor=outlier_factor, n_threads=n_threads)

    def save(self, path, *, overwrite: bool = False) -> None:
        """Write the coefficient NIfTI, its JSON sidecar and the diagnostic
        siblings (``<stem>_r2.nii.gz``, ``_rmse``, ``_alpha``, ``_bic``,
        ``_rss_l2``, ``_sparsity``) in the layout ``cs-fit`` uses
        (python/cs_dmri/shore.py:249-271, src/io/coeffs.rs:92-130)."""
        from . import nifti

        if self.affine is None:
            raise ValueError("saving needs an affine")
        path = Path(path)
        stem = _stem(path)
        outputs = {path: self.coefficients, Path(stem + ".json"): None}
        for name in ("r2", "rmse", "alpha", "bic", "rss_l2"):
            if getattr(self, name) is not None:
                outputs[Path(f"{stem}_{name}.nii.gz")] = np.asarray(getattr(self, name), dtype=np.float32)
        if self.r2 is not None:
            outputs[Path(f"{stem}_sparsity.nii.gz")] = self.sparsity
        if not overwrite:
            existing = [str(p) for p in outputs if p.exists()]
            if existing:
                raise FileExistsError(f"refusing to overwrite {existing}; pass overwrite=True")
        for p, arr in outputs.items():
            if arr is None:
                p.write_text(json.dumps(self.sidecar, indent=2))
            else:
                nifti.write(p, arr, self.affine)

    @classmethod
    def load(cls, path, mask=None) -> "ShoreFit":
        """Read a coefficient NIfTI written by :meth:`save` or ``cs-fit``
        (python/cs_dmri/shore.py:273-292)."""
        from . import nifti

        path = Path(path)
        stem = _stem(path)
        img = nifti.read(path)
        sidecar = json.loads(Path(stem + ".json").read_text())
        arrays = {"coefficients": np.asarray(img.data, dtype=np.float32), "sidecar": sidecar}
        for name in ("r2", "rmse", "alpha", "bic", "rss_l2"):
            p = Path(f"{stem}_{name}.nii.gz")
            if p.exists():
                arrays[name] = np.asarray(nifti.read(p).data, dtype=np.float32)
        frame = "world" if sidecar.get("bvec_frame") == "world-ras" else "image"
        rotation = _core.affine_rotation(img.affine) if frame == "world" else None
        return cls(arrays, mask=mask, affine=img.affine, frame=frame, rotation=rotation)

    def __repr__(self) -> str:
        r2 = "" if self.r2 is None else f", mean R² {float(self.r2[self.mask].mean()):.3f}"
        return f"ShoreFit(radial_order={self.radial_order}, {int(self.mask.sum())} voxels{r2}, frame={self.frame})"
