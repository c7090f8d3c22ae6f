"""Small, fixed workloads that run one pass of a kernel family, for
profiling under ncu (one launch of each kernel of interest, a few hundred MB
on the device at most):

    python -m cs_dmri_b200.profile_cases graddev2k   # k_graddev_fit, 2,000 voxels, radial order 8
    python -m cs_dmri_b200.profile_cases diff50k     # differentiable fit step: k_l1_adjoint, k_apply_dmma, ...
    python -m cs_dmri_b200.profile_cases peaks108k   # k_odf_peaks on a 60 x 60 x 30 coefficient volume
    python -m cs_dmri_b200.profile_cases fista125k   # the two-pass FISTA schedule on 125,000 voxels

fista125k runs its measured fit inside an NVTX range of that name
(``ncu --nvtx --nvtx-include "fista125k/"`` selects its launches).
"""

from __future__ import annotations

import sys

import numpy as np


def graddev2k() -> None:
    import torch

    from .graddev import graddev_phantom, shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = graddev_phantom(2000, seed=3)
    out = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.01, radial_order=8, big_delta=big, small_delta=small)
    torch.cuda.synchronize()
    print("graddev2k: mean iterations", float(out["iterations"].double().mean()))


def diff50k() -> None:
    import torch

    from .autograd import DifferentiableShore
    from .phantom import make_phantom
    ph = make_phantom((50, 50, 20), seed=4)
    S = torch.from_numpy(ph.data.reshape(-1, ph.data.shape[-1])).cuda().requires_grad_(True)
    m = DifferentiableShore(ph.bvals, ph.bvecs, big_delta=ph.big_delta, small_delta=ph.small_delta)
    a = torch.tensor(0.01, dtype=torch.float64, device="cuda", requires_grad=True)
    c = m.fit(S, a)
    (m.rtop(c).sum() + 1e-3 * m.odf(c).square().sum()).backward()
    torch.cuda.synchronize()
    print("diff50k: d loss / d alpha", float(a.grad))


def peaks108k() -> None:
    from ._core import shore_odf_peaks
    rng = np.random.default_rng(1)
    vol = rng.normal(size=(60, 60, 30, 72)).astype(np.float32)
    vol[..., 0] = np.abs(vol[..., 0]) + 5.0
    out = shore_odf_peaks(vol, 6, 700.0)
    print("peaks108k: mean GFA", float(out["gfa"].mean()))


def fista125k() -> None:
    """A fixed-alpha fit of a 50^3 phantom (125,000 voxels, K = 72) through the
    device entry point: enough voxels per FISTA slot for the two-pass
    schedule (pass 1 to iteration 80, bucket sort, pass 2).  A first fit
    (gradient-table set-up, autotuning) runs outside the NVTX range."""
    import torch

    from . import _abi
    from ._core import shore_fit_device
    from .phantom import make_phantom
    ph = make_phantom((50, 50, 50), seed=6)
    d = torch.from_numpy(ph.data).cuda()
    m = torch.from_numpy(ph.mask).cuda()
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01)
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("fista125k")
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    t = _abi.last_timing(0)
    print(f"fista125k: solve {t.ms_solve_kernel:.3f} ms, parked {t.fista_parked} of {int(ph.mask.sum())} voxels")


CASES = {"graddev2k": graddev2k, "diff50k": diff50k, "peaks108k": peaks108k, "fista125k": fista125k}

if __name__ == "__main__":
    if len(sys.argv) != 2 or sys.argv[1] not in CASES:
        sys.exit(f"usage: python -m cs_dmri_b200.profile_cases {{{'|'.join(CASES)}}}")
    CASES[sys.argv[1]]()
