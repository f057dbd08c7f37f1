"""Diverse-conformer selection on the GPU (the centre picking of
src/GeneDiverseConformations.cpp:84-111), through the C-ABI.

cluster_conformers() returns the indices of the centre conformers in selection order: energy
order, first centre the lowest, a new centre whenever the superposition RMSD to every centre so
far is above the cut-off, stopping when the count equals max_centers (tested after each
candidate from the second on, as the reference does). pair_rmsd() returns the RMSD matrix the
selection compares.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _prep(coords, atom_mask):
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    if coords.ndim != 3 or coords.shape[2] != 3:
        raise ValueError("coords must be [n_conf][n_atoms][3]")
    mask = None
    mptr = None
    if atom_mask is not None:
        mask = np.ascontiguousarray(atom_mask, dtype=np.uint8)
        if mask.shape != (coords.shape[1],):
            raise ValueError("atom_mask must have one entry per atom")
        mptr = mask.ctypes.data_as(C.c_void_p)
    return coords, mask, mptr


def cluster_conformers(coords, energies, cutoff: float = 1.5, max_centers: int = 100,
                       atom_mask=None) -> np.ndarray:
    coords, mask, mptr = _prep(coords, atom_mask)
    energies = np.ascontiguousarray(energies, dtype=np.float64)
    n_conf, n_atoms = coords.shape[:2]
    if energies.shape != (n_conf,):
        raise ValueError("energies must have one entry per conformer")
    centers = np.empty(max(n_conf, 1), np.int32)
    count = C.c_int(0)
    _lib.check(_lib.lib().cdk_cluster_conformers(
        n_conf, n_atoms, coords.ctypes.data_as(_dp), energies.ctypes.data_as(_dp), mptr,
        float(cutoff), int(max_centers), centers.ctypes.data_as(_ip), C.byref(count)))
    return centers[:count.value].copy()


def pair_rmsd(coords, atom_mask=None) -> np.ndarray:
    coords, mask, mptr = _prep(coords, atom_mask)
    n_conf, n_atoms = coords.shape[:2]
    out = np.empty((n_conf, n_conf), np.float64)
    _lib.check(_lib.lib().cdk_pair_rmsd(n_conf, n_atoms, coords.ctypes.data_as(_dp), mptr,
                                        out.ctypes.data_as(_dp)))
    return out
