"""Gradient tables for the SHORE fit.

A table is the b-values (s/mm^2) and gradient directions of a DWI series, in
the image's voxel-axis frame, plus the b=0 threshold and the optional
diffusion times.  The public names and keyword arguments are those of the
reference's ``cs_dmri.gradients`` module (python/cs_dmri/gradients.py), so
code written against it runs unchanged; the table itself is held here as one
read-only (N, 4) array of rows (b, gx, gy, gz).
"""

from __future__ import annotations

from os import PathLike
from pathlib import Path

import numpy as np

__all__ = ["GradientTable", "as_gradient_table", "read_bvals_bvecs"]


def _numbers(path: str | PathLike) -> np.ndarray:
    """The whitespace-separated numbers of a text file as a 2-D array, one
    row per non-empty line (FSL's .bval / .bvec layout)."""
    rows = [line.split() for line in Path(path).read_text().splitlines() if line.strip()]
    if not rows:
        return np.zeros((0, 0))
    widths = {len(r) for r in rows}
    if len(widths) != 1:
        raise ValueError(f"{path}: rows of different lengths {sorted(widths)}")
    return np.array(rows, dtype=np.float64)


def _direction_rows(bvecs, n: int) -> np.ndarray:
    """Directions as (n, 3) rows, from an (n, 3) or (3, n) array."""
    a = np.array(bvecs, dtype=np.float64)
    for candidate in (a, a.T if a.ndim == 2 else a):
        if candidate.shape == (n, 3):
            return candidate
    raise ValueError(f"bvecs must have shape ({n}, 3) or (3, {n}), got {a.shape}")


def read_bvals_bvecs(bval_file: str | PathLike, bvec_file: str | PathLike):
    """Read FSL-style ``.bval`` / ``.bvec`` files.  Returns ``(bvals (N,),
    bvecs (N, 3))``; the bvec file may hold 3 rows of N values (FSL) or N rows
    of 3."""
    bvals = _numbers(bval_file).reshape(-1)
    return bvals, _direction_rows(_numbers(bvec_file), bvals.size)


class GradientTable:
    """b-values and gradient directions of a DWI series.

    Directions are used as given (never flipped or rotated).  ``big_delta`` /
    ``small_delta`` are the diffusion times in seconds; when either is left
    out the fit estimates both from the largest b-value (TORTOISE's rule).
    Volumes with ``b <= b0_threshold`` are b=0 volumes.
    """

    def __init__(self, bvals, bvecs, *, b0_threshold: float = 50.0,
                 big_delta: float | None = None, small_delta: float | None = None):
        b = np.array(bvals, dtype=np.float64).reshape(-1)
        table = np.empty((b.size, 4))
        table[:, 0] = b
        table[:, 1:] = _direction_rows(bvecs, b.size)
        table.flags.writeable = False
        self._table = table
        self.b0_threshold = float(b0_threshold)
        self.big_delta = big_delta
        self.small_delta = small_delta

    @classmethod
    def from_files(cls, bval_file, bvec_file, **kwargs) -> "GradientTable":
        """Build from FSL ``.bval`` / ``.bvec`` files."""
        bvals, bvecs = read_bvals_bvecs(bval_file, bvec_file)
        return cls(bvals, bvecs, **kwargs)

    @classmethod
    def from_dipy(cls, gtab, **kwargs) -> "GradientTable":
        """Build from a dipy gradient table (anything with ``bvals`` and
        ``bvecs``), keeping its b=0 threshold unless one is given."""
        if "b0_threshold" not in kwargs and hasattr(gtab, "b0_threshold"):
            kwargs["b0_threshold"] = gtab.b0_threshold
        return cls(gtab.bvals, gtab.bvecs, **kwargs)

    @property
    def bvals(self) -> np.ndarray:
        return np.ascontiguousarray(self._table[:, 0])

    @property
    def bvecs(self) -> np.ndarray:
        return np.ascontiguousarray(self._table[:, 1:])

    @property
    def b0s_mask(self) -> np.ndarray:
        return self._table[:, 0] <= self.b0_threshold

    @property
    def max_b(self) -> float:
        return float(self._table[:, 0].max(initial=0.0))

    def __len__(self) -> int:
        return self._table.shape[0]

    def __repr__(self) -> str:
        b0 = int(np.count_nonzero(self.b0s_mask))
        return f"GradientTable(N={len(self)}, b0={b0}, dwi={len(self) - b0}, bmax={self.max_b:g})"


def as_gradient_table(gtab, **kwargs) -> GradientTable:
    """A GradientTable from one, from a dipy gradient table, or from a
    ``(bvals, bvecs)`` pair."""
    if isinstance(gtab, GradientTable):
        return gtab
    if isinstance(gtab, (tuple, list)) and len(gtab) == 2:
        return GradientTable(gtab[0], gtab[1], **kwargs)
    if all(hasattr(gtab, a) for a in ("bvals", "bvecs")):
        return GradientTable.from_dipy(gtab, **kwargs)
    raise TypeError(f"cannot make a gradient table from a {type(gtab).__name__}")
