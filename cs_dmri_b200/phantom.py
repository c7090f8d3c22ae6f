"""Seeded synthetic diffusion volumes for tests and benchmarks.

The reference measures no public dataset; its benchmark configurations are
synthetic CS-DSI acquisitions, restated here:

* gradient table: integer q-space grid points with |q| <= 5 (515 points with
  the origin); the origin is dropped, a seeded subset of 258 is kept and one
  b=0 volume is put first (N = 259).  b = 5000 |q|^2 / 25 s/mm^2 (bmax 5000),
  bvecs = q / |q|.  Delta / delta are explicit (43 ms / 11 ms) so every
  implementation computes identical q-values.
* signal per voxel: S0 * [sum_i (1 - f_iso) f_i exp(-b g'D_i g)
  + f_iso exp(-b 3e-3)] with 1-3 fibres of eigenvalues (1.7, 0.3, 0.3)e-3
  mm^2/s, uniform random orientations, Dirichlet(1) fractions, f_iso in
  U[0, 0.3], Rician noise at SNR 25 (sigma = S0 / 25), stored as float32.
  S0 = 1000 (raw DWI magnitude): the reference fits raw signals, and at S0 = 1
  the L1 weight alpha = 0.01 exceeds alpha_max (~3e-4) so every voxel's L1 fit
  would be exactly zero.
* mask: every voxel of a small grid, or an ellipsoid inside a
  96 x 114 x 96 brain-sized grid holding ~300k voxels.

All randomness comes from a counter-based SplitMix64 stream keyed by
(seed, voxel index, draw index), so any voxel can be generated independently
and any implementation of the same hash reproduces the volume bit for bit.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["Phantom", "gradient_table", "brain_mask", "make_phantom", "CONFIGS"]

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
BIG_DELTA = 0.043
SMALL_DELTA = 0.011
S0 = 1000.0
SNR = 25.0
LAMBDA_PAR, LAMBDA_PERP, D_ISO = 1.7e-3, 0.3e-3, 3.0e-3


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, counters: np.ndarray) -> np.ndarray:
    """U[0, 1) doubles for the given 64-bit counters of stream `seed`."""
    key = np.asarray(counters, dtype=np.uint64) + (np.uint64(seed) << np.uint64(40))
    return (_splitmix64(key) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def gradient_table(seed: int = 1, n_dirs: int = 258):
    """CS-DSI table: (bvals (N,), bvecs (N, 3)) with the b=0 volume first."""
    r = np.arange(-5, 6)
    q = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    q = q[(q * q).sum(1) <= 25]
    q = q[np.any(q != 0, axis=1)]
    keys = uniform(seed, np.arange(len(q), dtype=np.uint64) + np.uint64(1 << 39))
    sel = q[np.sort(np.argsort(keys, kind="stable")[:n_dirs])].astype(np.float64)
    norm = np.linalg.norm(sel, axis=1)
    bvals = np.concatenate([[0.0], 5000.0 * norm ** 2 / 25.0])
    bvecs = np.vstack([np.zeros((1, 3)), sel / norm[:, None]])
    return bvals, bvecs


def brain_mask(shape=(96, 114, 96), fill: float = 0.8165) -> np.ndarray:
    """Ellipsoid with semi-axes `fill` x half the grid (~300k of 1.05M voxels)."""
    axes = [(np.arange(n) - (n - 1) / 2.0) / (fill * n / 2.0) for n in shape]
    x, y, z = np.meshgrid(*axes, indexing="ij")
    return (x * x + y * y + z * z) <= 1.0


def signals(seed: int, voxel_ids: np.ndarray, bvals: np.ndarray, bvecs: np.ndarray,
            s0: float = S0, snr: float = SNR) -> np.ndarray:
    """Multi-tensor + free-water Rician signals (len(voxel_ids), N) float32."""
    n = len(bvals)
    stride = np.uint64(16 + 2 * n)
    v = np.asarray(voxel_ids, dtype=np.uint64)[:, None] * stride

    def draw(slot, count=1):
        return uniform(seed, v + np.uint64(slot) + np.arange(count, dtype=np.uint64)[None, :])

    u_nf = draw(0)[:, 0]
    nf = 1 + np.minimum((u_nf * 3).astype(np.int64), 2)
    e = -np.log1p(-draw(1, 3))                       # Exp(1) draws -> Dirichlet(1)
    active = np.arange(3)[None, :] < nf[:, None]
    e = np.where(active, e, 0.0)
    frac = e / e.sum(1, keepdims=True)
    f_iso = 0.3 * draw(4)[:, 0]
    uz = 2.0 * draw(5, 3) - 1.0
    uphi = 2.0 * np.pi * draw(8, 3)
    rxy = np.sqrt(np.maximum(1.0 - uz * uz, 0.0))
    u = np.stack([rxy * np.cos(uphi), rxy * np.sin(uphi), uz], -1)      # (V, 3 fibres, 3)
    cos2 = np.einsum("vfc,nc->vfn", u, bvecs) ** 2                        # (V, 3, N)
    adc = LAMBDA_PERP + (LAMBDA_PAR - LAMBDA_PERP) * cos2
    att = np.exp(-bvals[None, None, :] * adc)
    s = ((1.0 - f_iso)[:, None, None] * frac[:, :, None] * att).sum(1)
    s += f_iso[:, None] * np.exp(-bvals * D_ISO)[None, :]
    s *= s0
    sigma = s0 / snr
    u1 = 1.0 - draw(16, n)
    u2 = draw(16 + n, n)
    rad = np.sqrt(-2.0 * np.log(u1))
    n1 = rad * np.cos(2.0 * np.pi * u2)
    n2 = rad * np.sin(2.0 * np.pi * u2)
    return np.sqrt((s + sigma * n1) ** 2 + (sigma * n2) ** 2).astype(np.float32)


@dataclass
class Phantom:
    data: np.ndarray      # (X, Y, Z, N) float32
    mask: np.ndarray      # (X, Y, Z) bool
    bvals: np.ndarray
    bvecs: np.ndarray
    big_delta: float = BIG_DELTA
    small_delta: float = SMALL_DELTA
    seed: int = 1

    @property
    def n_voxels(self) -> int:
        return int(self.mask.sum())


def make_phantom(shape=(20, 20, 10), mask: np.ndarray | None = None, seed: int = 1,
                 chunk: int = 32768, s0: float = S0) -> Phantom:
    """Volume of `shape` with signals in the mask (default: every voxel) and
    zeros elsewhere."""
    bvals, bvecs = gradient_table(seed)
    if mask is None:
        mask = np.ones(shape, dtype=bool)
    n = len(bvals)
    data = np.zeros(tuple(shape) + (n,), dtype=np.float32)
    flat = data.reshape(-1, n)
    ids = np.flatnonzero(mask.ravel())
    for i in range(0, len(ids), chunk):
        part = ids[i:i + chunk]
        flat[part] = signals(seed, part, bvals, bvecs, s0=s0)
    return Phantom(data=data, mask=mask, bvals=bvals, bvecs=bvecs, seed=seed)


# Benchmark configurations (synthetic stand-ins of the reference's workloads).
CONFIGS = {
    "grid4k": dict(shape=(20, 20, 10), mask=None, seed=1),
    "brain300k": dict(shape=(96, 114, 96), mask="brain", seed=2),
    "grid64k": dict(shape=(40, 40, 40), mask=None, seed=3),
}


def config_phantom(name: str) -> Phantom:
    cfg = dict(CONFIGS[name])
    mask = brain_mask(cfg["shape"]) if cfg["mask"] == "brain" else None
    return make_phantom(cfg["shape"], mask=mask, seed=cfg["seed"])
