"""Regenerate the golden fixtures under tests/golden/.

Run where a checkout of the cs_dmri reference is available, giving its path
as the first argument or in CS_DMRI_REFERENCE.  Two sets are written:

1. lasso_fixtures.npz - the reference's eight scikit-learn LASSO fixtures
   (tests/data/lasso_fixtures/*.bin, format of tests/optimization_sklearn.rs:
   32-35, 68-127: "<IIIIB7xddd" header, row-major design, signal, expected
   coefficients), decoded into arrays.  They pin the oracle's FISTA to the
   reference's own external golden vectors.
2. shore_lasso.npz - new scikit-learn Lasso golds (fit_intercept=False,
   tol 1e-12, the objective (1/(2n))||Mc - s||^2 + alpha ||c||_1 of
   src/solver/fista.rs:4-7) on the real order-4 SHORE design of the synthetic
   CS-DSI table, for phantom voxels at S0 = 1000: the same objective at N = 259
   on the basis the product fits.
"""

from __future__ import annotations

import json
import os
import struct
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
def reference_root() -> Path:
    """The reference checkout: argv[1], else $CS_DMRI_REFERENCE."""
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CS_DMRI_REFERENCE")
    if not root:
        sys.exit("usage: python tests/golden/make_golden.py <cs_dmri checkout> (or set CS_DMRI_REFERENCE)")
    return Path(root)


def decode_bin(raw: bytes) -> dict:
    magic, version, m, n, positive, alpha, amax, obj = struct.unpack_from("<IIIIB7xddd", raw, 0)
    assert magic == 0x434C4153 and version == 1, "not a CLAS v1 fixture"
    off = 48
    design = np.frombuffer(raw, "<f8", m * n, off).reshape(m, n)
    off += 8 * m * n
    signal = np.frombuffer(raw, "<f8", m, off)
    off += 8 * m
    coef = np.frombuffer(raw, "<f8", n, off)
    assert off + 8 * n == len(raw)
    return dict(design=design.copy(), signal=signal.copy(), coef=coef.copy(), alpha=alpha, alpha_max=amax,
                objective=obj, positive=bool(positive))


def lasso_fixtures(reference: Path) -> None:
    src = reference / "tests" / "data" / "lasso_fixtures"
    names = json.loads((src / "manifest.json").read_text())
    arrays = {}
    for fname in names:
        fx = decode_bin((src / fname).read_bytes())
        key = fname[:-4]
        for k, v in fx.items():
            arrays[f"{key}__{k}"] = np.asarray(v)
    arrays["__names__"] = np.array([f[:-4] for f in names])
    np.savez_compressed(HERE / "lasso_fixtures.npz", **arrays)
    print(f"wrote {len(names)} reference LASSO fixtures")


def shore_lasso() -> None:
    from sklearn.linear_model import Lasso

    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    from cs_dmri_b200.phantom import BIG_DELTA, SMALL_DELTA, gradient_table, signals

    bvals, bvecs = gradient_table(1)
    M = O.design_matrix(bvals, bvecs, order=4, zeta=700.0, big_delta=BIG_DELTA, small_delta=SMALL_DELTA)
    S = signals(1, np.arange(6), bvals, bvecs).astype(np.float64)
    out = {"design": M, "signals": S}
    for alpha in (0.5, 2.0):
        coefs, objs = [], []
        for s in S:
            mdl = Lasso(alpha=alpha, fit_intercept=False, tol=1e-12, max_iter=2_000_000)
            mdl.fit(M, s)
            c = mdl.coef_.astype(np.float64)
            r = M @ c - s
            coefs.append(c)
            objs.append(0.5 / len(s) * r @ r + alpha * np.abs(c).sum())
        out[f"coef_a{alpha}"] = np.array(coefs)
        out[f"obj_a{alpha}"] = np.array(objs)
    np.savez_compressed(HERE / "shore_lasso.npz", **out)
    print("wrote SHORE sklearn golds")


if __name__ == "__main__":
    lasso_fixtures(reference_root())
    shore_lasso()
