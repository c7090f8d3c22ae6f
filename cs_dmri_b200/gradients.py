"""Gradient tables (mirror of cs_dmri.gradients, python/cs_dmri/gradients.py)."""

from __future__ import annotations

from os import PathLike

import numpy as np

__all__ = ["GradientTable", "as_gradient_table", "read_bvals_bvecs"]


def read_bvals_bvecs(bval_file: str | PathLike, bvec_file: str | PathLike):
    """Read FSL-style ``.bval`` / ``.bvec`` files; bvecs may be 3xN or Nx3."""
    bvals = np.loadtxt(bval_file, dtype=np.float64, ndmin=1).ravel()
    bvecs = np.loadtxt(bvec_file, dtype=np.float64, ndmin=2)
    return bvals, _bvecs_n3(bvecs, len(bvals))


def _bvecs_n3(bvecs, n: int) -> np.ndarray:
    bvecs = np.asarray(bvecs, dtype=np.float64)
    if bvecs.shape == (n, 3):
        return np.ascontiguousarray(bvecs)
    if bvecs.shape == (3, n):
        return np.ascontiguousarray(bvecs.T)
    raise ValueError(f"bvecs must have shape ({n}, 3) or (3, {n}), got {bvecs.shape}")


class GradientTable:
    """b-values and gradient directions of a DWI series.

    Directions are taken as given (never flipped or rotated).  ``big_delta`` /
    ``small_delta`` are diffusion times in seconds; if either is missing both
    are estimated from the maximum b-value (TORTOISE's heuristic) inside the
    fit, as the reference does (python/cs_dmri/gradients.py:32-61).
    """

    def __init__(self, bvals, bvecs, *, b0_threshold: float = 50.0,
                 big_delta: float | None = None, small_delta: float | None = None):
        bvals = np.ascontiguousarray(np.asarray(bvals, dtype=np.float64).ravel())
        self._bvals = bvals
        self._bvecs = _bvecs_n3(bvecs, len(bvals))
        self._bvals.setflags(write=False)
        self._bvecs.setflags(write=False)
        self.b0_threshold = float(b0_threshold)
        self.big_delta = big_delta
        self.small_delta = small_delta

    @classmethod
    def from_files(cls, bval_file, bvec_file, **kwargs) -> "GradientTable":
        return cls(*read_bvals_bvecs(bval_file, bvec_file), **kwargs)

    @classmethod
    def from_dipy(cls, gtab, **kwargs) -> "GradientTable":
        kwargs.setdefault("b0_threshold", getattr(gtab, "b0_threshold", 50.0))
        return cls(gtab.bvals, gtab.bvecs, **kwargs)

    @property
    def bvals(self) -> np.ndarray:
        return self._bvals

    @property
    def bvecs(self) -> np.ndarray:
        return self._bvecs

    @property
    def b0s_mask(self) -> np.ndarray:
        return self._bvals <= self.b0_threshold

    def __len__(self) -> int:
        return len(self._bvals)

    def __repr__(self) -> str:
        return f"GradientTable({len(self)} volumes, {int(self.b0s_mask.sum())} b0)"


def as_gradient_table(gtab) -> GradientTable:
    """Accept a GradientTable, anything with ``bvals``/``bvecs``, or a
    ``(bvals, bvecs)`` pair."""
    if isinstance(gtab, GradientTable):
        return gtab
    if hasattr(gtab, "bvals") and hasattr(gtab, "bvecs"):
        return GradientTable.from_dipy(gtab)
    if isinstance(gtab, (tuple, list)) and len(gtab) == 2:
        return GradientTable(*gtab)
    raise TypeError(f"cannot build a gradient table from {type(gtab).__name__}")
