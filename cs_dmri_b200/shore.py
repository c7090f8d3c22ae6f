"""3D-SHORE model and fit objects with the reference's Python interface
(``cs_dmri.ShoreModel`` / ``cs_dmri.ShoreFit``, python/cs_dmri/shore.py:25-299),
fitted by the CUDA library.

The classes keep the reference's names, keyword arguments, defaults, result
attributes and ``ValueError`` messages; underneath, a model is a table of
solver settings handed to ``_core.shore_fit`` and a fit is a coefficient
volume plus a dictionary of diagnostic maps.  The on-disk layout of
``save`` / ``load`` is the one ``cs-fit`` writes (src/io/coeffs.rs:92-170).
"""

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

# Keyword arguments of ShoreModel that go to the solver unchanged.
_SOLVER_KEYS = ("alpha_mode", "alpha", "alpha_ratio", "path_n_alphas", "path_eps", "slack", "max_iter", "tol",
                "non_negative", "lambda_n", "lambda_l", "nonneg_max_iter", "nonneg_tol", "nonneg_epsilon",
                "allow_single_shell", "precision")
# Per-voxel maps a fit may carry, and the ones written next to the
# coefficient file (in this order, then the sparsity map when R^2 exists).
_MAP_NAMES = ("r2", "rmse", "residual_l2", "iterations", "regularization_kind", "alpha", "bic", "rss_l2")
_SAVED_MAPS = ("r2", "rmse", "alpha", "bic", "rss_l2")


def _choice(name: str, value, allowed) -> None:
    if value not in allowed:
        raise ValueError(f"{name} must be one of {allowed}, got {value!r}")


def _frame_rotation(bvec_frame: str, affine):
    """The fit frame ("world" | "image") and the rotation R taking image-axis
    vectors into it (python/cs_dmri/_frame.py:13-31): world RAS needs the
    affine's column-normalised rotation; "auto" picks world when an affine is
    known."""
    _choice("bvec_frame", bvec_frame, _FRAMES)
    world = bvec_frame == "world" or (bvec_frame == "auto" and affine is not None)
    if not world:
        return "image", np.eye(3)
    if affine is None:
        raise ValueError("bvec_frame='world' needs an affine (fit a DWI, or pass affine=)")
    return "world", _core.affine_rotation(affine)


def _in_frame(vectors, R) -> np.ndarray:
    """Row vectors rotated by R (v -> R v for every row)."""
    return np.ascontiguousarray(np.einsum("ij,...j->...i", R, np.asarray(vectors, dtype=np.float64)))


def _volume_and_mask(data, mask):
    vol = np.asarray(data, dtype=np.float32)
    if vol.ndim != 4:
        raise ValueError(f"expected a 4-D (X, Y, Z, N) array, got shape {vol.shape}")
    if mask is None:
        raise ValueError("a mask is required")
    m = np.asarray(mask)
    m = m if m.dtype == bool else m > 0
    if m.shape != vol.shape[:3]:
        raise ValueError(f"mask shape {m.shape} does not match data spatial shape {vol.shape[:3]}")
    return vol, m


class ShoreModel:
    """3D-SHORE model (Merlet & Deriche 2013; Ozarslan et al. 2013).

    Parameters and defaults are those of ``cs_dmri.ShoreModel``:
    ``radial_order`` (even; 6 gives 72 coefficients), ``zeta`` (700),
    ``regularization`` in ``{"l1", "l2", "nonneg"}``, ``alpha_mode`` in
    ``{"l2-anchored", "path-bic", "alpha-ratio", "fixed"}``, the L1 path
    settings, the Tikhonov weights ``lambda_n`` / ``lambda_l``, the
    amplitude-ICLS settings, ``bvec_frame`` and ``allow_single_shell``.  Two
    keywords are added: ``device`` (the GPU) and ``precision`` ("fp64", the
    reference arithmetic; "mixed"; "mixed-kkt" / "fp64-kkt" for the
    KKT-certified optimum, see ``_core.shore_fit``).
    """

    def __init__(self, gtab, *, radial_order: int = 6, zeta: float = 700.0, regularization: str = "l1",
                 alpha_mode: str = "l2-anchored", alpha: float = 1.0, alpha_ratio: float = 1e-3,
                 path_n_alphas: int = 20, path_eps: float | None = None, slack: float = 0.05,
                 max_iter: int = 1000, tol: float = 1e-6, non_negative: bool = False,
                 lambda_n: float = 1e-8, lambda_l: float = 1e-8, nonneg_max_iter: int = 200,
                 nonneg_tol: float = 1e-9, nonneg_epsilon: float = 1e-10, bvec_frame: str = "auto",
                 allow_single_shell: bool = False, device: int = 0, precision: str = "fp64"):
        settings = dict(locals())
        _choice("regularization", regularization, _REGULARIZATIONS)
        _choice("alpha_mode", alpha_mode, _ALPHA_MODES)
        self.gtab = as_gradient_table(gtab)
        self.radial_order, self.zeta = radial_order, zeta
        self.regularization, self.bvec_frame, self.device = regularization, bvec_frame, device
        self._solver = {k: settings[k] for k in _SOLVER_KEYS}

    def fit(self, data, mask=None, *, affine=None, diagnostics: bool = True,
            n_threads: int | None = None) -> "ShoreFit":
        """Fit every voxel of ``mask`` ((X, Y, Z); required for arrays)."""
        vol, m = _volume_and_mask(data, mask)
        if affine is not None:
            affine = np.asarray(affine, dtype=np.float64)
        frame, R = _frame_rotation(self.bvec_frame, affine)
        g = self.gtab
        result = _core.shore_fit(vol, g.bvals, _in_frame(g.bvecs, R), m, big_delta=g.big_delta,
                                 small_delta=g.small_delta, b0_threshold=g.b0_threshold,
                                 bvec_frame={"world": "world-ras", "image": "image-axis"}[frame],
                                 radial_order=self.radial_order, zeta=self.zeta,
                                 regularization=self.regularization, diagnostics=diagnostics,
                                 n_threads=n_threads, device=self.device, **self._solver)
        for text in result.pop("warnings", ()):
            warnings.warn(text, stacklevel=2)
        return ShoreFit(result, model=self, mask=m, affine=affine, frame=frame, rotation=R)


class ShoreFit:
    """Result of :meth:`ShoreModel.fit` (or :meth:`load`): ``coefficients``
    (X, Y, Z, K) float32, the diagnostic maps (``r2, rmse, residual_l2,
    iterations, regularization_kind``, and ``alpha, bic, rss_l2`` where the
    solver makes them; ``None`` otherwise), ``sidecar``, ``alpha_distribution``
    and ``frame``."""

    def __init__(self, arrays: dict, *, model=None, mask=None, affine=None, frame="image", rotation=None):
        self.coefficients = arrays["coefficients"]
        self.sidecar = arrays["sidecar"]
        self.alpha_distribution = arrays.get("alpha_distribution")
        self._maps = {name: arrays.get(name) for name in _MAP_NAMES}
        self.model, self.affine, self.frame = model, affine, frame
        self.mask = mask if mask is not None else np.count_nonzero(self.coefficients, axis=-1) > 0
        self._rotation = np.eye(3) if rotation is None else np.asarray(rotation, dtype=np.float64)
        self.radial_order = int(self.sidecar["basis"]["radial_order"])
        self.zeta = float(self.sidecar["basis"]["zeta"])

    def __getattr__(self, name):
        maps = self.__dict__.get("_maps")
        if maps is not None and name in maps:
            return maps[name]
        raise AttributeError(f"{type(self).__name__!s} has no attribute {name!r}")

    @property
    def dwi_shells(self):
        """Mean b of the non-zero shells the fit used (None if not recorded)."""
        shells = self.sidecar.get("dwi_shells")
        return None if shells is None else list(map(float, shells))

    @property
    def single_shell(self) -> bool:
        shells = self.dwi_shells
        return shells is not None and len(shells) <= 1

    @property
    def sparsity(self) -> np.ndarray:
        """Fraction of non-zero coefficients per voxel (0 outside the mask)."""
        c = self.coefficients
        frac = np.count_nonzero(c, axis=-1) / np.float32(max(c.shape[-1], 1))
        return np.where(self.mask, frac, 0.0).astype(np.float32)

    def odf_sh(self, lmax: int | None = None, *, n_threads=None) -> np.ndarray:
        """Tournier (MRtrix) SH coefficients of the ODF, (X, Y, Z, n_sh); the
        default ``lmax`` is the largest even value <= the radial order."""
        if lmax is None:
            lmax = 2 * (self.radial_order // 2)
        return _core.shore_odf_sh(self.coefficients, self.radial_order, self.zeta, lmax, self.mask,
                                  n_threads=n_threads)

    def predict(self, gtab=None, *, clip: bool = True, n_threads=None) -> np.ndarray:
        """Signal on ``gtab`` (default: the model's table), (X, Y, Z, N).  The
        table is in the image's voxel-axis frame and is rotated into the fit
        frame here."""
        if gtab is None and self.model is None:
            raise ValueError("pass a gradient table: this fit has no model")
        g = as_gradient_table(self.model.gtab if gtab is None else gtab)
        if self.single_shell:
            b_fit = self.dwi_shells[0]
            b_new = g.bvals[~g.b0s_mask]
            if b_new.size and float(np.abs(b_new - b_fit).max()) > 50.0:
                warnings.warn(f"single-shell fit (b = {b_fit:.0f}): the prediction at other b-values comes "
                              "from the regularization, not from measurements", stacklevel=2)
        sig = _core.shore_predict(self.coefficients, self.radial_order, self.zeta, g.bvals,
                                  _in_frame(g.bvecs, self._rotation),
                                  big_delta=self.sidecar["big_delta_seconds"],
                                  small_delta=self.sidecar["small_delta_seconds"], n_threads=n_threads)
        if clip:
            np.maximum(sig, 0, out=sig)
        return sig

    def peaks(self, *, npeaks: int = 5, relative_peak_threshold: float = 0.5, min_separation_angle: float = 25.0,
              sphere_frequency: int = 6) -> dict:
        """GFA and ODF peaks inside the mask (``shore_odf_peaks``; the
        quantities of the reference's ODX export, src/io/odx_out.rs:1008-1090).
        Peak directions come back in the image's voxel-axis frame."""
        out = _core.shore_odf_peaks(self.coefficients, self.radial_order, self.zeta, self.mask,
                                    sphere_frequency=sphere_frequency, npeaks=npeaks,
                                    relative_peak_threshold=relative_peak_threshold,
                                    min_separation_angle=min_separation_angle)
        out["peak_dirs"] = _in_frame(out["peak_dirs"], self._rotation.T).astype(np.float32)
        return out

    def microstructure(self, directions=None, *, units: str = "um", outlier_factor: float | None = 10.0,
                       n_threads=None) -> dict:
        """RTOP, RTAP, RTPP, MSD, QIV and NG maps.  RTAP / RTPP need
        ``directions`` (X, Y, Z, 3) in the image's voxel-axis frame and are
        NaN without them.  A single-shell fit raises ``ValueError``: the data
        do not determine its radial decay."""
        if self.single_shell:
            raise ValueError(
                "propagator-derived scalars are not determined by single-shell data "
                f"(this fit used b = {self.dwi_shells[0]:.0f} only)")
        dirs = None if directions is None else _in_frame(directions, self._rotation).astype(np.float32)
        return _core.shore_microstructure(self.coefficients, self.radial_order, self.zeta, self.mask, dirs,
                                          units=units, outlier_factor=outlier_factor, n_threads=n_threads)

    # ---- the cs-fit file layout: <stem>.nii.gz, <stem>.json, <stem>_<map>.nii.gz

    @staticmethod
    def _stem(path: Path) -> str:
        name = str(path)
        for ext in (".nii.gz", ".nii"):
            if name.endswith(ext):
                return name[: -len(ext)]
        return str(path.with_suffix(""))

    def _files(self, path: Path):
        """(path, array or None for the sidecar) of everything save writes."""
        stem = self._stem(path)
        yield path, self.coefficients
        yield Path(stem + ".json"), None
        for name in _SAVED_MAPS:
            if self._maps.get(name) is not None:
                yield Path(f"{stem}_{name}.nii.gz"), np.asarray(self._maps[name], dtype=np.float32)
        if self._maps.get("r2") is not None:
            yield Path(f"{stem}_sparsity.nii.gz"), self.sparsity

    def save(self, path, *, overwrite: bool = False) -> None:
        """Write the coefficient NIfTI, its JSON sidecar and the diagnostic
        siblings in the layout ``cs-fit`` uses."""
        from . import nifti

        if self.affine is None:
            raise ValueError("saving needs an affine")
        files = list(self._files(Path(path)))
        clash = [str(p) for p, _ in files if p.exists()]
        if clash and not overwrite:
            raise FileExistsError(f"refusing to overwrite {clash}; pass overwrite=True")
        for p, arr in files:
            if arr is None:
                p.write_text(json.dumps(self.sidecar, indent=2))
            else:
                nifti.write(p, arr, self.affine)

    @classmethod
    def load(cls, path, mask=None) -> "ShoreFit":
        """Read a coefficient NIfTI written by :meth:`save` or ``cs-fit``, with
        its sidecar and whichever diagnostic siblings exist."""
        from . import nifti

        path = Path(path)
        stem = cls._stem(path)
        img = nifti.read(path)
        arrays = {"coefficients": np.asarray(img.data, dtype=np.float32),
                  "sidecar": json.loads(Path(stem + ".json").read_text())}
        for name in _SAVED_MAPS:
            sib = Path(f"{stem}_{name}.nii.gz")
            if sib.exists():
                arrays[name] = np.asarray(nifti.read(sib).data, dtype=np.float32)
        world = arrays["sidecar"].get("bvec_frame") == "world-ras"
        return cls(arrays, mask=mask, affine=img.affine, frame="world" if world else "image",
                   rotation=_core.affine_rotation(img.affine) if world else None)

    def __repr__(self) -> str:
        n = int(np.count_nonzero(self.mask))
        r2 = self._maps.get("r2")
        tail = "" if r2 is None else f", mean R² {float(np.mean(r2[self.mask])):.3f}"
        return f"ShoreFit(radial_order={self.radial_order}, {n} voxels{tail}, frame={self.frame})"
