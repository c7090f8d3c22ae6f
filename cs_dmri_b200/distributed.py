"""One volume fitted across several GPUs, one process per GPU.

The fit is independent per voxel, so a volume shards without any exchange in
the solve: rank r fits a contiguous chunk of the masked voxels (canonical
x-y-z order, src/voxel_loop.rs:28-42) on its own GPU.  Two collectives
assemble the result, both outside the solve:

* each rank's rows - the coefficients and diagnostic values of its own
  masked voxels, V_r x (K + maps) - are gathered to the destination rank,
  which places them into the volume by the mask (the shards are contiguous
  runs of the canonical order, so the rows arrive in order); the result is
  the single-GPU result bit for bit, and only V x (K + maps) values cross the
  interconnect, not world x the volume;
* the per-voxel alphas are gathered so the alpha distribution (median, p10,
  p90 by nearest rank, src/fit.rs:334-352) is taken over the whole mask.

Works with any torch.distributed backend (NCCL across GPUs, gloo on CPU).
"""

from __future__ import annotations

import numpy as np

__all__ = ["shard_mask", "fit_sharded", "alpha_distribution"]


def _torch_dtype(dt: np.dtype):
    import torch
    return {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
            np.dtype(np.uint32): torch.int64, np.dtype(np.uint8): torch.uint8,
            np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64}[np.dtype(dt)]


_MAPS = ("r2", "rmse", "residual_l2", "iterations", "regularization_kind", "alpha", "bic", "rss_l2")


def shard_mask(mask: np.ndarray, rank: int, world: int) -> np.ndarray:
    """Mask of rank `rank`'s shard: masked voxels [lo, hi) of the canonical
    order, with counts differing by at most one between ranks."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    flat = np.asarray(mask, dtype=bool).ravel()
    ids = np.flatnonzero(flat)
    lo = (len(ids) * rank) // world
    hi = (len(ids) * (rank + 1)) // world
    out = np.zeros_like(flat)
    out[ids[lo:hi]] = True
    return out.reshape(np.shape(mask))


def alpha_distribution(alphas: np.ndarray):
    """(median, p10, p90) by nearest rank, src/fit.rs:337-350."""
    a = np.sort(np.asarray(alphas, dtype=np.float64))
    if a.size == 0:
        return (0.0, 0.0, 0.0)

    def pct(q):
        i = int(np.floor((a.size - 1) * q + 0.5))  # f64::round: half away from zero (non-negative here)
        return float(a[min(i, a.size - 1)])

    return (pct(0.5), pct(0.10), pct(0.90))


def fit_sharded(data, bvals, bvecs, mask, *, group=None, dst: int = 0, fit_fn=None, **kw) -> dict | None:
    """Fit `mask` across the ranks of `group`; rank `dst` returns the whole
    result dict (the others return None).

    `fit_fn(data, bvals, bvecs, mask, **kw) -> dict` defaults to
    :func:`cs_dmri_b200.shore_fit` on this rank's GPU.  Everything but the
    alpha distribution is the single-process result bit for bit; the
    distribution is taken over the f32 alpha maps, and because f32 rounding is
    monotonic each percentile is the f32 rounding of the single-process one.
    """
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    if fit_fn is None:
        from . import shore_fit

        fit_fn = shore_fit
    diag = bool(kw.get("diagnostics", False))
    per_voxel_alpha = kw.get("regularization", "l1") == "l1" and kw.get("alpha_mode", "l2-anchored") != "fixed"
    local = shard_mask(mask, rank, world)
    out = fit_fn(data, bvals, bvecs, local, **dict(kw, diagnostics=diag or per_voxel_alpha))
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    sel = local.ravel()
    counts_all = [int(shard_mask(mask, r, world).sum()) for r in range(world)]  # the same on every rank
    n_max = max(1, max(counts_all))

    def gather_rows(a: np.ndarray, width: int) -> np.ndarray | None:
        """This rank's masked rows of `a` (flattened to (voxels, width)),
        gathered on `dst` in rank order: (V, width), or None elsewhere."""
        rows = np.asarray(a).reshape(-1, width)[sel]
        buf = torch.zeros((n_max, width), dtype=_torch_dtype(rows.dtype), device=dev)
        send = rows.astype(np.int64) if rows.dtype == np.uint32 else rows  # no uint32 collectives
        buf[: rows.shape[0]] = torch.from_numpy(np.ascontiguousarray(send)).to(dev)
        parts = [torch.empty_like(buf) for _ in range(world)] if rank == dst else None
        dist.gather(buf, gather_list=parts, dst=dst, group=group)
        if rank != dst:
            return None
        return np.concatenate([p[:c].cpu().numpy() for p, c in zip(parts, counts_all)]).astype(rows.dtype, copy=False)

    def place(rows: np.ndarray | None, like: np.ndarray) -> np.ndarray | None:
        if rows is None:
            return None
        full = np.zeros_like(like)
        flat = full.reshape(len(sel), -1)
        flat[np.asarray(mask, dtype=bool).ravel()] = rows.reshape(rows.shape[0], -1)
        return full

    K = out["coefficients"].shape[-1]
    result = {"coefficients": place(gather_rows(out["coefficients"], K), out["coefficients"])}
    if diag:
        for k in _MAPS:
            if out.get(k) is not None:
                result[k] = place(gather_rows(out[k], 1), out[k])
    counts = torch.tensor([out.get("total_iterations", 0), out.get("n_voxels", int(local.sum()))],
                          dtype=torch.int64, device=dev)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    result["total_iterations"], result["n_voxels"] = (int(v) for v in counts.tolist())
    dist_all = None
    if per_voxel_alpha:
        a_local = torch.from_numpy(np.asarray(out["alpha"][local], dtype=np.float64)).to(dev)
        sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
        dist.all_gather(sizes, torch.tensor([a_local.numel()], dtype=torch.int64, device=dev), group=group)
        n_max = max(1, int(max(s.item() for s in sizes)))
        padded = torch.zeros(n_max, dtype=torch.float64, device=dev)
        padded[: a_local.numel()] = a_local
        parts = [torch.zeros(n_max, dtype=torch.float64, device=dev) for _ in range(world)]
        dist.all_gather(parts, padded, group=group)
        alphas = np.concatenate([p[: int(s.item())].cpu().numpy() for p, s in zip(parts, sizes)])
        dist_all = alpha_distribution(alphas)
    result["alpha_distribution"] = dist_all if per_voxel_alpha else out.get("alpha_distribution")
    if rank != dst:
        return None
    side = dict(out["sidecar"])
    if per_voxel_alpha:
        med, p10, p90 = dist_all
        side["solver"] = dict(side["solver"],
                              chosen_alpha={"scope": "per-voxel", "median": med, "p10": p10, "p90": p90})
    result["sidecar"] = side
    result["warnings"] = out.get("warnings", [])
    return result
