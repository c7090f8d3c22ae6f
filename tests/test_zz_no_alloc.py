"""The allocation-free batch entry point, checked against the volume fit.

csd_shore_fista_batch_noalloc is for callers that cannot let the library
call cudaMalloc (their device memory belongs to their own pool allocator, or
they cannot afford cudaFree's device-wide synchronisation): it keeps all its
scratch in one static device array.  This test drives it through the C ABI
with caller-owned device buffers on several calls in a row of different sizes,
which also shows that a call does not read stale scratch left by the previous
one, and compares each result with csd_shore_fit_volume's coefficients at the
parity tolerance of the other GPU tests (relative L2 <= 1e-5 per voxel).
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_VOXELS = 8192


def _noalloc(lib, gtab, spec, sig, out, its, stream):
    err = C.create_string_buffer(1024)
    code = lib.csd_shore_fista_batch_noalloc(C.byref(gtab), C.byref(spec), C.c_void_p(sig.data_ptr()),
                                             sig.shape[0], C.c_void_p(out.data_ptr()),
                                             C.c_void_p(its.data_ptr()), C.c_void_p(stream), err, len(err))
    return code, err.value.decode()


@pytest.mark.parametrize("order", [2, 4, 6])
def test_noalloc_batch_matches_volume_fit(order):
    """Radial orders 2, 4 and 6 (K = 8, 29, 72): the 8- and 32-row padded
    layouts of the right-hand sides and iterates, and the 72-row one."""
    import torch

    from cs_dmri_b200 import _abi, shore_fit
    from cs_dmri_b200._core import build_gtab, build_spec
    from cs_dmri_b200.phantom import make_phantom

    lib = _abi.load()
    kw = dict(alpha_mode="fixed", alpha=0.01, radial_order=order)
    K = lib.csd_shore_n_coeffs(order)
    stream = torch.cuda.current_stream().cuda_stream
    first = None
    for seed, shape in ((21, (12, 10, 8)), (22, (16, 16, 5)), (21, (12, 10, 8))):
        ph = make_phantom(shape, seed=seed)
        ref = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                        return_coef64=True, diagnostics=True, **kw)
        V = ph.n_voxels
        sig = torch.from_numpy(np.ascontiguousarray(ph.data.reshape(V, -1))).cuda()
        out = torch.full((V, K), float("nan"), dtype=torch.float32, device="cuda")
        its = torch.zeros(V, dtype=torch.int32, device="cuda")
        gtab, keep = build_gtab(ph.bvals, ph.bvecs, 50.0, ph.big_delta, ph.small_delta)
        spec = build_spec(**kw)
        torch.cuda.synchronize()
        code, msg = _noalloc(lib, gtab, spec, sig, out, its, stream)
        assert code == 0, msg
        c = out.cpu().numpy().astype(np.float64)
        rel = np.linalg.norm(c - ref["coef64"], axis=1) / np.maximum(np.linalg.norm(ref["coef64"], axis=1), 1e-300)
        assert rel.max() <= 1e-5, rel.max()
        it = its.cpu().numpy().astype(np.int64)
        assert np.abs(it - ref["iterations"].reshape(-1).astype(np.int64)).max() <= 1
        if first is None:
            first = (shape, c)
        elif shape == first[0]:
            assert np.array_equal(c, first[1])     # same input, same result after other calls


def test_noalloc_rejects_oversize_batches():
    import torch

    from cs_dmri_b200 import _abi
    from cs_dmri_b200._core import build_gtab, build_spec
    from cs_dmri_b200.phantom import gradient_table

    lib = _abi.load()
    bvals, bvecs = gradient_table(1)
    gtab, keep = build_gtab(bvals, bvecs, 50.0, 0.043, 0.011)
    sig = torch.zeros((MAX_VOXELS + 1, len(bvals)), dtype=torch.float32, device="cuda")
    out = torch.zeros((MAX_VOXELS + 1, 72), dtype=torch.float32, device="cuda")
    its = torch.zeros(MAX_VOXELS + 1, dtype=torch.int32, device="cuda")
    code, msg = _noalloc(lib, gtab, build_spec(alpha_mode="fixed", alpha=0.01), sig, out, its, 0)
    assert code == _abi.ERR_INVALID and "at most 8192 voxels" in msg
    code, msg = _noalloc(lib, gtab, build_spec(alpha_mode="l2-anchored"), sig[:4], out[:4], its[:4], 0)
    assert code == _abi.ERR_INVALID and "fixed alpha" in msg
    code, msg = _noalloc(lib, gtab, build_spec(alpha_mode="fixed", alpha=0.01, radial_order=8), sig[:4], out[:4],
                         its[:4], 0)
    assert code == _abi.ERR_INVALID and "radial order" in msg
    code, msg = _noalloc(lib, gtab, build_spec(alpha_mode="fixed", alpha=0.01, precision="mixed"), sig[:4],
                         out[:4], its[:4], 0)
    assert code == _abi.ERR_INVALID and "FP64 only" in msg
