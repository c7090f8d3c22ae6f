"""The C-ABI library loads on any machine and exports every function that
include/csd_shore.h declares (no compute call needs a GPU here)."""

import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "csd_shore.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(csd_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("csd_create", "csd_destroy", "csd_shore_fit_volume", "csd_shore_fit_volume_device"):
        assert n in names


def test_library_exports_every_declared_symbol(lib_built):
    from cs_dmri_b200 import _abi
    lib = C.CDLL(str(_abi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_abi.EXPORTS) == set(declared_functions())


def test_pure_functions_without_gpu(lib_built):
    from cs_dmri_b200 import _abi
    lib = _abi.load()
    assert lib.csd_abi_version() == 1
    assert lib.csd_shore_n_coeffs(6) == 72 and lib.csd_shore_n_coeffs(8) == 145
    s = _abi.default_spec()
    assert (s.radial_order, s.zeta, s.regularization, s.alpha_mode) == (6, 700.0, _abi.REG_L1,
                                                                        _abi.ALPHA_L2_ANCHORED)
    assert (s.max_iter, s.tol, s.path_n_alphas, s.slack) == (1000, 1e-6, 20, 0.05)
    assert (s.lambda_n, s.lambda_l, s.nonneg_max_iter, s.nonneg_tol) == (1e-8, 1e-8, 200, 1e-9)


def test_struct_layout_matches_header(lib_built):
    """Compile a tiny C probe of sizeof/offsetof and compare with ctypes."""
    import subprocess
    import tempfile
    from cs_dmri_b200 import _abi
    fields = {"csd_shore_spec": (_abi.Spec, ["zeta", "alpha", "path_eps", "precision"]),
              "csd_fit_result": (_abi.FitResult, ["n_coeffs", "n_voxels", "alpha_distribution",
                                                  "dwi_shells", "total_iterations", "warnings"]),
              "csd_gtab": (_abi.Gtab, ["n", "big_delta", "b0_threshold"]),
              "csd_fit_timing": (_abi.Timing, ["launches", "ms_solve_kernel", "tensor_flops", "ms_mixed_kernel",
                                                  "int8_tensor_ops", "fp64_rerun_voxels"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT}/include/csd_shore.h"',
             'int main(void){']
    for st, (_, fs) in fields.items():
        lines.append(f'printf("%zu\\n", sizeof({st}));')
        for f in fs:
            lines.append(f'printf("%zu\\n", offsetof({st}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = Path(d) / "p.c"
        src.write_text("\n".join(lines))
        exe = Path(d) / "p"
        subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
        vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    it = iter(vals)
    for st, (cls, fs) in fields.items():
        assert next(it) == C.sizeof(cls), st
        for f in fs:
            assert next(it) == getattr(cls, f).offset, (st, f)
