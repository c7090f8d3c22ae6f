"""Coefficient files: the NIfTI-1 reader/writer and ShoreFit.save / load
(python/cs_dmri/shore.py:249-292, src/io/coeffs.rs:92-170).  CPU only: the fit
arrays are synthetic."""

import json
import struct

import numpy as np
import pytest


def affine_of(rot_deg=20.0, zooms=(2.0, 2.5, 3.0), flip=False):
    t = np.deg2rad(rot_deg)
    R = np.array([[np.cos(t), -np.sin(t), 0.0], [np.sin(t), np.cos(t), 0.0], [0.0, 0.0, 1.0]])
    if flip:
        R[:, 0] = -R[:, 0]
    A = np.eye(4)
    A[:3, :3] = R * np.array(zooms)
    A[:3, 3] = (-90.0, 12.5, 40.0)
    return A


@pytest.mark.parametrize("suffix", [".nii", ".nii.gz"])
@pytest.mark.parametrize("flip", [False, True])
def test_nifti_round_trip(tmp_path, suffix, flip):
    from cs_dmri_b200 import nifti
    rng = np.random.default_rng(0)
    data = rng.normal(size=(5, 4, 3, 7)).astype(np.float32)
    A = affine_of(flip=flip)
    p = tmp_path / f"x{suffix}"
    nifti.write(p, data, A)
    img = nifti.read(p)
    np.testing.assert_array_equal(img.data, data)
    np.testing.assert_allclose(img.affine, A, atol=1e-5)
    assert img.header["datatype"] == 16 and img.header["dim"][:5] == (4, 5, 4, 3, 7)
    np.testing.assert_allclose(img.header["pixdim"][1:4], (2.0, 2.5, 3.0), rtol=1e-6)


def test_nifti_x_fastest_on_disk(tmp_path):
    """Voxel (1, 0, 0) follows voxel (0, 0, 0) in the file (NIfTI order)."""
    from cs_dmri_b200 import nifti
    data = np.zeros((3, 2, 2), np.float32)
    data[1, 0, 0] = 7.0
    p = tmp_path / "x.nii"
    nifti.write(p, data, np.eye(4))
    raw = p.read_bytes()
    assert struct.unpack_from("<f", raw, 352 + 4)[0] == 7.0


@pytest.mark.parametrize("flip,atol", [(False, 1e-5), (True, 5e-3)])
def test_nifti_qform_only(tmp_path, flip, atol):
    """A file whose sform_code is 0 is read through its quaternion.  The
    quaternion is stored in float32, so a rotation close to 180 degrees (what
    a reflected affine becomes) keeps only about 3 digits, as in any NIfTI
    reader; that is why the writer also stores the sform."""
    from cs_dmri_b200 import nifti
    A = affine_of(35.0, flip=flip)
    p = tmp_path / "q.nii"
    nifti.write(p, np.ones((2, 2, 2), np.float32), A)
    raw = bytearray(p.read_bytes())
    struct.pack_into("<h", raw, 254, 0)
    p.write_bytes(bytes(raw))
    np.testing.assert_allclose(nifti.read(p).affine, A, atol=atol)


def test_shore_fit_save_load(tmp_path):
    from cs_dmri_b200.shore import ShoreFit
    rng = np.random.default_rng(1)
    coef = rng.normal(size=(4, 3, 2, 72)).astype(np.float32)
    coef[0, 0, 0] = 0.0
    sidecar = {"basis": {"name": "shore", "radial_order": 6, "zeta": 700.0}, "bvec_frame": "image-axis",
               "n_coefficients": 72, "big_delta_seconds": 0.0431, "small_delta_seconds": 0.0107}
    arrays = {"coefficients": coef, "sidecar": sidecar, "r2": rng.random((4, 3, 2)).astype(np.float32),
              "alpha": np.full((4, 3, 2), 0.01, np.float32)}
    A = affine_of()
    fit = ShoreFit(arrays, affine=A)
    out = tmp_path / "sub-01_shore.nii.gz"
    fit.save(out)
    for name in ("sub-01_shore.json", "sub-01_shore_r2.nii.gz", "sub-01_shore_alpha.nii.gz",
                 "sub-01_shore_sparsity.nii.gz"):
        assert (tmp_path / name).exists(), name
    assert not (tmp_path / "sub-01_shore_bic.nii.gz").exists()
    assert json.loads((tmp_path / "sub-01_shore.json").read_text()) == sidecar
    with pytest.raises(FileExistsError):
        fit.save(out)
    fit.save(out, overwrite=True)
    back = ShoreFit.load(out)
    np.testing.assert_array_equal(back.coefficients, coef)
    np.testing.assert_array_equal(back.r2, arrays["r2"])
    np.testing.assert_allclose(back.affine, A, atol=1e-5)
    assert back.radial_order == 6 and back.frame == "image" and back.sidecar == sidecar
    assert not back.mask[0, 0, 0] and back.mask.sum() == 23
    with pytest.raises(ValueError, match="affine"):
        ShoreFit(arrays).save(tmp_path / "y.nii.gz")
