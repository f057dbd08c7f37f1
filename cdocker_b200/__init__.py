"""cdocker_b200 -- B200-native FFT translational-rotational docking search.

Python face of libcdock_b200.so. The search itself runs in hand-written sm_100a kernels
behind the C-ABI (include/cdock_b200.h); this package only marshals arrays:

    rec = Receptor(grids, spacing)            # K resident receptor spectra
    minE, idx = rec.search(coor, charge, eps, slot, quats)

Host helpers keep the reference's semantics bit for bit (quaternion sampling and filtering,
vdW slot assignment, grid file I/O).
"""
from ._lib import CdkError, CDK_FORM_FP32, CDK_FORM_BF16X3, CDK_FORM_FP16X2, lib, last_error  # noqa: F401
from .api import (  # noqa: F401
    Receptor,
    fill_ligand_grid,
    filter_quaternions,
    quaternion_uniform_sampling,
    read_grids,
    synth_receptor_grids,
    vdw_slots,
    write_grids,
)

__all__ = [
    "Receptor",
    "CdkError",
    "fill_ligand_grid",
    "filter_quaternions",
    "quaternion_uniform_sampling",
    "read_grids",
    "synth_receptor_grids",
    "vdw_slots",
    "write_grids",
]
