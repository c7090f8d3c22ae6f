"""B200-native 3D-SHORE fit with the interface of cs_dmri's SHORE path.

``ShoreModel(gtab).fit(data, mask)`` and ``shore_fit(...)`` mirror
``cs_dmri.ShoreModel`` and ``cs_dmri._cs_dmri.shore_fit``; every per-voxel
computation runs in libcsdshore.so (hand-written CUDA for sm_100a) behind the
C ABI declared in include/csd_shore.h.
"""

from ._core import (affine_rotation, design_matrix, shore_fit, shore_fit_device, shore_microstructure,
                    shore_odf_peaks, shore_odf_sh, shore_predict)
from .gradients import GradientTable, as_gradient_table, read_bvals_bvecs
from .shore import ShoreFit, ShoreModel

__all__ = ["ShoreModel", "ShoreFit", "GradientTable", "as_gradient_table", "read_bvals_bvecs",
           "shore_fit", "shore_fit_device", "design_matrix", "affine_rotation", "shore_predict",
           "shore_odf_sh", "shore_odf_peaks", "shore_microstructure"]
__version__ = "0.1.0"
