"""Top-k poses after a search: ranking, coordinates and the reference's output files.

The reference ranks each conformer's rotations with sort_index (std::sort, strict <;
include/GeneDiverseConformations.h:9-20), rebuilds the nLowest poses
(src/TranRotaConfSearchNoMini.cu:467-487), writes each as conformer_<c>_<rank>.pdb and appends
`file,conformer,rank,energy` to energy.txt (:489-502). OpenMM minimisation of those poses stays
on the reference side.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L


def sort_index(values) -> np.ndarray:
    """Indices ordered by value, ascending, through cdk_sort_index: the reference's std::sort
    with strict < (include/GeneDiverseConformations.h:9-20), so equal energies rank in the same
    order as in the reference driver."""
    v = np.ascontiguousarray(values, np.float32).reshape(-1)
    out = np.empty(v.shape[0], np.int64)
    L.check(L.lib().cdk_sort_index(v.ctypes.data_as(C.POINTER(C.c_float)), v.shape[0],
                                   out.ctypes.data_as(C.POINTER(C.c_long))))
    return out


def pose_coordinates(coor, quat, grid_min, spacing, idx) -> np.ndarray:
    """[nAtom, 3] double coordinates of one pose (cdk_pose_coordinates)."""
    c = np.ascontiguousarray(coor, np.float32).reshape(-1, 3)
    q = np.ascontiguousarray(quat, np.float32).reshape(4)
    g = np.ascontiguousarray(grid_min, np.float64).reshape(3)
    i = np.ascontiguousarray(idx, np.int32).reshape(3)
    out = np.empty((c.shape[0], 3), np.float64)
    L.check(L.lib().cdk_pose_coordinates(
        c.shape[0], c.ctypes.data_as(C.POINTER(C.c_float)), q.ctypes.data_as(C.POINTER(C.c_float)),
        g.ctypes.data_as(C.POINTER(C.c_double)), float(spacing),
        i.ctypes.data_as(C.POINTER(C.c_int)), out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


def write_pdb(path: str, xyz: np.ndarray, elements=None) -> None:
    with open(path, "w") as f:
        for a, (x, y, z) in enumerate(np.asarray(xyz)):
            el = (elements[a] if elements is not None else "C")[:2]
            f.write(f"HETATM{a + 1:5d} {el:<4s} LIG A   1    {x:8.3f}{y:8.3f}{z:8.3f}"
                    f"  1.00  0.00          {el:>2s}\n")
        f.write("END\n")


def export_top(out_dir: str, conformer: int, coor, quats, minE, idx, grid_min, spacing,
               n_lowest: int, energy_file=None):
    """Writes the n_lowest poses of one conformer; returns [(file, rank, energy)]."""
    os.makedirs(out_dir, exist_ok=True)
    order = sort_index(minE)
    rows = []
    for rank in range(min(n_lowest, len(order))):
        r = int(order[rank])
        if not np.isfinite(minE[r]):
            break
        xyz = pose_coordinates(coor, quats[r], grid_min, spacing, idx[r])
        name = f"conformer_{conformer}_{rank}.pdb"
        write_pdb(os.path.join(out_dir, name), xyz)
        rows.append((name, rank, float(minE[r])))
        if energy_file is not None:
            energy_file.write(f"{name},{conformer},{rank},{float(minE[r]):g}\n")
    return rows


def rescore_top(receptor, coor, charge, eps, slot, quats, minE, idx, k: int = 8,
                batch: int = 1000):
    """FP64 re-score of the k lowest-energy rotations of every batch of `batch` consecutive
    rotations (direct trilinear grid-energy sum on the GPU, cdk_rescore_fp64).
    Returns (indices [n_batches, k] into the rotation list, energies [n_batches, k] float64)."""
    coor = np.ascontiguousarray(coor, np.float32)
    if coor.ndim == 2:
        coor = coor[None]
    q = np.ascontiguousarray(quats, np.float32).reshape(-1, 4)
    n_q = q.shape[0] // coor.shape[0]
    n = q.shape[0]
    tops, confs, qs, ts = [], [], [], []
    for b0 in range(0, n, batch):
        order = sort_index(minE[b0:b0 + batch])[:k] + b0
        tops.append(order)
        for r in order:
            confs.append(r // n_q)
            qs.append(q[r])
            ts.append(idx[r])
    e = receptor.rescore_fp64(coor, charge, eps, slot, np.asarray(confs, np.int32),
                              np.asarray(qs, np.float32), np.asarray(ts, np.int32))
    kk = min(k, batch)
    return np.asarray(tops).reshape(-1, kk), e.reshape(-1, kk)
