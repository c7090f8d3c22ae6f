"""Minimal NIfTI-1 reading and writing for the coefficient files.

The reference writes coefficient volumes with the `nifti` crate
(src/io/coeffs.rs:92-150) and, from Python, with nibabel
(python/cs_dmri/shore.py:249-289).  Neither is available here, so this module
reads and writes the single-file NIfTI-1 format directly: a 348-byte header,
a 4-byte extension flag, then the voxel data with x varying fastest; ``.gz``
paths are gzip-compressed.  Writing covers float32 images with an affine
(stored as both sform and qform, code 1 = scanner); reading accepts the
common numeric types and returns the array in (x, y, z, ...) order.
"""

from __future__ import annotations

import gzip
import struct
from pathlib import Path

import numpy as np

__all__ = ["write", "read", "NiftiImage"]

_DTYPES = {2: np.uint8, 4: np.int16, 8: np.int32, 16: np.float32, 64: np.float64, 256: np.int8, 512: np.uint16,
           768: np.uint32}


class NiftiImage:
    """Array (x, y, z, ...) with its 4 x 4 voxel-to-world affine."""

    def __init__(self, data: np.ndarray, affine: np.ndarray, header: dict | None = None):
        self.data = data
        self.affine = affine
        self.header = header or {}


def _quaternion(R: np.ndarray):
    """qform quaternion (b, c, d) and qfac of a rotation-with-reflection."""
    qfac = 1.0
    if np.linalg.det(R) < 0:
        R = R.copy()
        R[:, 2] = -R[:, 2]
        qfac = -1.0
    # closest proper rotation, then the standard matrix -> quaternion
    u, _, vt = np.linalg.svd(R)
    R = u @ vt
    a = 1.0 + R[0, 0] + R[1, 1] + R[2, 2]
    if a > 0.5:
        a = 0.5 * np.sqrt(a)
        b = 0.25 * (R[2, 1] - R[1, 2]) / a
        c = 0.25 * (R[0, 2] - R[2, 0]) / a
        d = 0.25 * (R[1, 0] - R[0, 1]) / a
    else:
        xd, yd, zd = 1.0 + R[0, 0] - (R[1, 1] + R[2, 2]), 1.0 + R[1, 1] - (R[0, 0] + R[2, 2]), \
            1.0 + R[2, 2] - (R[0, 0] + R[1, 1])
        if xd > 1.0:
            b = 0.5 * np.sqrt(xd)
            c = 0.25 * (R[0, 1] + R[1, 0]) / b
            d = 0.25 * (R[0, 2] + R[2, 0]) / b
            a = 0.25 * (R[2, 1] - R[1, 2]) / b
        elif yd > 1.0:
            c = 0.5 * np.sqrt(yd)
            b = 0.25 * (R[0, 1] + R[1, 0]) / c
            d = 0.25 * (R[1, 2] + R[2, 1]) / c
            a = 0.25 * (R[0, 2] - R[2, 0]) / c
        else:
            d = 0.5 * np.sqrt(zd)
            b = 0.25 * (R[0, 2] + R[2, 0]) / d
            c = 0.25 * (R[1, 2] + R[2, 1]) / d
            a = 0.25 * (R[1, 0] - R[0, 1]) / d
        if a < 0:
            b, c, d = -b, -c, -d
    return float(b), float(c), float(d), qfac


def write(path, data: np.ndarray, affine: np.ndarray) -> None:
    """Write ``data`` ((x, y, z) or (x, y, z, t), any real dtype, stored as
    float32) with ``affine`` to a .nii or .nii.gz file."""
    arr = np.asarray(data, dtype=np.float32)
    if arr.ndim not in (3, 4):
        raise ValueError(f"NIfTI data must be 3-D or 4-D, got {arr.ndim}-D")
    A = np.asarray(affine, dtype=np.float64)
    if A.shape != (4, 4):
        raise ValueError("affine must be 4 x 4")
    zooms = np.sqrt((A[:3, :3] ** 2).sum(0))
    R = A[:3, :3] / np.where(zooms > 0, zooms, 1.0)
    qb, qc, qd, qfac = _quaternion(R)
    dim = [arr.ndim] + list(arr.shape) + [1] * (7 - arr.ndim)
    pixdim = [qfac] + list(zooms) + [1.0] * 4
    h = bytearray(348)
    struct.pack_into("<i", h, 0, 348)                        # sizeof_hdr
    struct.pack_into("<8h", h, 40, *dim)                      # dim
    struct.pack_into("<h", h, 70, 16)                         # datatype FLOAT32
    struct.pack_into("<h", h, 72, 32)                         # bitpix
    struct.pack_into("<8f", h, 76, *pixdim)                   # pixdim
    struct.pack_into("<f", h, 108, 352.0)                     # vox_offset
    struct.pack_into("<f", h, 112, 0.0)                       # scl_slope (0: unused)
    struct.pack_into("<f", h, 116, 0.0)                       # scl_inter
    struct.pack_into("<B", h, 123, 10)                        # xyzt_units: mm, s
    struct.pack_into("<h", h, 252, 1)                         # qform_code
    struct.pack_into("<h", h, 254, 1)                         # sform_code
    struct.pack_into("<3f", h, 256, qb, qc, qd)               # quatern_b/c/d
    struct.pack_into("<3f", h, 268, *A[:3, 3])                # qoffset_x/y/z
    struct.pack_into("<4f", h, 280, *A[0])                    # srow_x
    struct.pack_into("<4f", h, 296, *A[1])                    # srow_y
    struct.pack_into("<4f", h, 312, *A[2])                    # srow_z
    h[344:348] = b"n+1\x00"                                   # magic
    payload = bytes(h) + b"\x00\x00\x00\x00" + arr.tobytes(order="F")
    path = Path(path)
    if str(path).endswith(".gz"):
        with gzip.open(path, "wb", compresslevel=1) as f:
            f.write(payload)
    else:
        path.write_bytes(payload)


def read(path) -> NiftiImage:
    """Read a single-file NIfTI-1 image (.nii / .nii.gz)."""
    path = Path(path)
    raw = gzip.open(path, "rb").read() if str(path).endswith(".gz") else path.read_bytes()
    if len(raw) < 352:
        raise ValueError(f"{path}: not a NIfTI-1 file")
    end = "<" if struct.unpack_from("<i", raw, 0)[0] == 348 else ">"
    if struct.unpack_from(end + "i", raw, 0)[0] != 348 or raw[344:347] != b"n+1":
        raise ValueError(f"{path}: not a single-file NIfTI-1 image")
    dim = struct.unpack_from(end + "8h", raw, 40)
    datatype = struct.unpack_from(end + "h", raw, 70)[0]
    if datatype not in _DTYPES:
        raise ValueError(f"{path}: unsupported NIfTI datatype {datatype}")
    pixdim = struct.unpack_from(end + "8f", raw, 76)
    vox_offset = int(struct.unpack_from(end + "f", raw, 108)[0])
    slope, inter = struct.unpack_from(end + "2f", raw, 112)
    sform_code = struct.unpack_from(end + "h", raw, 254)[0]
    shape = tuple(dim[1:1 + dim[0]])
    dt = np.dtype(_DTYPES[datatype]).newbyteorder(end)
    n = int(np.prod(shape))
    data = np.frombuffer(raw, dtype=dt, count=n, offset=vox_offset).reshape(shape, order="F")
    data = np.asarray(data, dtype=dt.newbyteorder("="))
    if slope not in (0.0, 1.0) or inter != 0.0:
        data = data * (slope if slope != 0.0 else 1.0) + inter
    if sform_code > 0:
        A = np.eye(4)
        for r, off in enumerate((280, 296, 312)):
            A[r] = struct.unpack_from(end + "4f", raw, off)
    else:
        qb, qc, qd = struct.unpack_from(end + "3f", raw, 256)
        qx, qy, qz = struct.unpack_from(end + "3f", raw, 268)
        qa = np.sqrt(max(1.0 - (qb * qb + qc * qc + qd * qd), 0.0))
        R = np.array([[qa * qa + qb * qb - qc * qc - qd * qd, 2 * (qb * qc - qa * qd), 2 * (qb * qd + qa * qc)],
                      [2 * (qb * qc + qa * qd), qa * qa + qc * qc - qb * qb - qd * qd, 2 * (qc * qd - qa * qb)],
                      [2 * (qb * qd - qa * qc), 2 * (qc * qd + qa * qb), qa * qa + qd * qd - qb * qb - qc * qc]])
        qfac = -1.0 if pixdim[0] < 0 else 1.0
        A = np.eye(4)
        A[:3, :3] = R * np.array([pixdim[1], pixdim[2], pixdim[3] * qfac])
        A[:3, 3] = (qx, qy, qz)
    return NiftiImage(data, A, {"dim": dim, "pixdim": pixdim, "datatype": datatype, "sform_code": sform_code})
