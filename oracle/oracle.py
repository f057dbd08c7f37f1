"""Oracle loaders and the FP64 FFT form -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import
this module, and only as the checker. It loads:
  * libcdk_oracle.so          the CPU restatement (oracle/cdk_oracle.cpp)
  * _ref/libcdk_ref.so        the reference's own host helpers compiled from their sources
  * _ref/libcdk_ref_cufft.so  the reference cuFFT path (needs a GPU to run)
and provides fft64_search(), a float64 numpy form of the same correlation computed through
rfftn / irfftn over the full grid (the reference's E = C2R(sum_k conj(F L_k) F P_k) / N,
src/kernel.cu:5-30 and src/TranRotaConfSearchNoMini.cu:415-464) -- an oracle independent of
both the direct sum and the GPU kernels.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "libcdk_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcdk_ref.so")
REF_CUFFT_LIB = os.path.join(HERE, "_ref", "libcdk_ref_cufft.so")

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)


def build(ref: bool | None = None) -> None:
    """Builds libcdk_oracle.so, and the reference libraries when the reference tree exists."""
    targets = ["oracle"]
    if ref is None:
        ref = os.path.isdir("/root/reference/src")
    if ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _pf(a):
    return a.ctypes.data_as(_fp)


def _pi(a):
    return a.ctypes.data_as(_ip)


_orc = None
_ref = None
_refcufft = None


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build(ref=False)
        L = C.CDLL(ORACLE_LIB)
        L.orc_search_direct.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _fp,
                                        C.c_int, C.c_int, _fp, _fp, _fp, _ip, C.c_int, _fp,
                                        C.c_int, C.c_int, C.c_int, _fp, _ip, _dp]
        L.orc_search_direct.restype = None
        L.orc_sample_quaternions.argtypes = [C.c_ulonglong, C.c_int, C.c_int, _fp]
        L.orc_filter_quaternions.argtypes = [_fp, C.c_int, C.c_int, _fp, C.c_float, C.c_float,
                                             C.c_float, C.c_int, _fp]
        L.orc_filter_quaternions.restype = C.c_int
        L.orc_vdw_slots.argtypes = [C.c_int, _fp, C.c_int, _fp, _ip, _ip]
        L.orc_vdw_slots.restype = C.c_int
        L.orc_fill_ligand_grid.argtypes = [C.c_int, C.c_int, _fp, _fp, _fp, _fp, _ip, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_float, _fp]
        L.orc_rotate_bbox.argtypes = [C.c_int, _fp, C.c_int, _fp, _fp, _fp, _fp]
        L.orc_rotate.argtypes = [_fp, _fp, _fp]
        L.orc_srand.argtypes = [C.c_uint]
        L.orc_window.argtypes = [C.c_int, C.c_float, C.c_float]
        L.orc_window.restype = C.c_int
        L.orc_energy_map.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _fp, C.c_int,
                                     _fp, _fp, _fp, _ip, _fp, _ip, _dp, C.c_long]
        L.orc_sort_index.argtypes = [C.c_int, _fp, _lp]
        L.orc_pair_rmsd.argtypes = [C.c_int, C.c_int, _dp, C.c_void_p, _dp]
        L.orc_pair_rmsd.restype = None
        L.orc_cluster_conformers.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_void_p, C.c_double,
                                             C.c_int, _ip]
        L.orc_cluster_conformers.restype = C.c_int
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(REF_LIB)
        L.ref_quaternion_uniform_sampling.argtypes = [C.c_ulonglong, C.c_int, C.c_int, _fp]
        L.ref_filter_quaternions.argtypes = [_fp, C.c_int, C.c_int, _fp, C.c_float, C.c_float,
                                             C.c_float, C.c_int, _fp]
        L.ref_filter_quaternions.restype = C.c_int
        L.ref_vdw_slots.argtypes = [C.c_int, _fp, C.c_int, _fp, _ip, _ip]
        L.ref_vdw_slots.restype = C.c_int
        L.ref_fill_ligand_grid.argtypes = [C.c_int, C.c_int, _fp, _fp, _fp, _fp, _fp, C.c_int,
                                           _fp, C.c_int, C.c_int, C.c_int, C.c_float, _fp]
        L.ref_min_max_coors.argtypes = [C.c_int, C.c_int, _fp, _fp, _fp]
        L.ref_rotate.argtypes = [_fp, _fp, _fp]
        L.ref_srand.argtypes = [C.c_uint]
        L.ref_read_grids.argtypes = [C.c_char_p, _ip, _fp, _fp, C.c_long, _fp, C.c_long]
        L.ref_read_grids.restype = C.c_int
        _ref = L
    return _ref


def refcufft() -> C.CDLL:
    global _refcufft
    if _refcufft is None:
        L = C.CDLL(REF_CUFFT_LIB)
        L.refcufft_search.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _fp, _fp,
                                      C.c_int, _fp, _fp, _fp, _fp, C.c_int, _fp, C.c_int, _fp,
                                      _ip, _dp]
        L.refcufft_search.restype = C.c_int
        _refcufft = L
    return _refcufft


# ------------------------------------------------------------------ restatement wrappers
def search_direct(grids, spacing, coor, charge, eps, slot, quats, prec=1, dense=0, nthreads=0):
    """cpuNaive-style direct correlation per rotation (oracle/cdk_oracle.cpp).
    grids [K,n,n,n]; coor [nConf,nAtom,3]; quats [nConf,nQ,4].
    Returns (minE float32, idx int32 [.,3], minE64 float64)."""
    g = _f32(grids)
    K, X, Y, Z = g.shape
    c = _f32(coor)
    if c.ndim == 2:
        c = c[None]
    nconf, na = c.shape[:2]
    q = _f32(quats).reshape(nconf, -1, 4)
    nq = q.shape[1]
    minE = np.empty(nconf * nq, np.float32)
    idx = np.empty((nconf * nq, 3), np.int32)
    m64 = np.empty(nconf * nq, np.float64)
    orc().orc_search_direct(X, Y, Z, float(spacing), K, _pf(g), na, nconf, _pf(c),
                            _pf(_f32(charge)), _pf(_f32(eps)), _pi(_i32(slot)), nq, _pf(q),
                            int(prec), int(dense), int(nthreads), _pf(minE), _pi(idx),
                            m64.ctypes.data_as(_dp))
    return minE, idx, m64


def energy_map(grids, spacing, coor, charge, eps, slot, quat, cap=10_000_000):
    """Double-precision energy over one rotation's whole window: [W0, W1, W2]."""
    g = _f32(grids)
    K, X, Y, Z = g.shape
    c = _f32(coor).reshape(-1, 3)
    w = np.zeros(3, np.int32)
    q = _f32(quat).reshape(4)
    # first call sizes the window
    out = np.empty(int(cap), np.float64)
    orc().orc_energy_map(X, Y, Z, float(spacing), K, _pf(g), c.shape[0], _pf(c),
                         _pf(_f32(charge)), _pf(_f32(eps)), _pi(_i32(slot)), _pf(q), _pi(w),
                         out.ctypes.data_as(_dp), int(cap))
    if w[0] <= 0 or w[1] <= 0 or w[2] <= 0:
        return np.zeros((0, 0, 0))
    return out[: w[0] * w[1] * w[2]].reshape(w[0], w[1], w[2]).copy()


def sample_quaternions(seed, nconf, nq):
    out = np.empty((nconf, nq, 4), np.float32)
    orc().orc_sample_quaternions(seed, nconf, nq, _pf(out))
    return out


def filter_quaternions(coor, quats, glen, max_n):
    c = _f32(coor).reshape(-1, 3)
    q = _f32(quats).reshape(-1, 4)
    out = np.empty_like(q)
    n = orc().orc_filter_quaternions(_pf(c), c.shape[0], q.shape[0], _pf(q), float(glen[0]),
                                     float(glen[1]), float(glen[2]), int(max_n), _pf(out))
    return out[:n].copy()


def vdw_slots(radii, grid_radii):
    r = _f32(radii)
    g = _f32(grid_radii)
    used = np.empty(g.shape[0], np.int32)
    slot = np.empty(r.shape[0], np.int32)
    n = orc().orc_vdw_slots(r.shape[0], _pf(r), g.shape[0], _pf(g), _pi(used), _pi(slot))
    return used[:n].copy(), slot


def rotate_bbox(coor, quats):
    c = _f32(coor).reshape(-1, 3)
    q = _f32(quats).reshape(-1, 4)
    rot = np.empty((q.shape[0], c.shape[0], 3), np.float32)
    mn = np.empty((q.shape[0], 3), np.float32)
    ln = np.empty((q.shape[0], 3), np.float32)
    orc().orc_rotate_bbox(c.shape[0], _pf(c), q.shape[0], _pf(q), _pf(rot), _pf(mn), _pf(ln))
    return rot, mn, ln


def fill_ligand_grid(rot, mn, charge, eps, slot, n_used, dims, spacing):
    r = _f32(rot)
    nq, na = r.shape[:2]
    out = np.zeros((nq, n_used + 1) + tuple(dims), np.float32)
    orc().orc_fill_ligand_grid(nq, na, _pf(r), _pf(_f32(mn)), _pf(_f32(charge)), _pf(_f32(eps)),
                               _pi(_i32(slot)), int(n_used), dims[0], dims[1], dims[2],
                               float(spacing), _pf(out))
    return out


# ------------------------------------------------------------------ FP64 FFT form
def fft64_search(grids, spacing, coor, charge, eps, slot, quats):
    """Float64 FFT correlation on the full grid, window min and first argmin per rotation."""
    g = np.asarray(grids, np.float64)
    K, X, Y, Z = g.shape
    Pf = np.fft.rfftn(g, axes=(1, 2, 3))
    c = _f32(coor)
    if c.ndim == 2:
        c = c[None]
    q = _f32(quats).reshape(c.shape[0], -1, 4)
    nq = q.shape[1]
    minE = np.full(c.shape[0] * nq, np.inf)
    idx = np.full((c.shape[0] * nq, 3), -1, np.int32)
    for ci in range(c.shape[0]):
        rot, mn, ln = rotate_bbox(c[ci], q[ci])
        lig = fill_ligand_grid(rot, mn, charge, eps, slot, K - 1, (X, Y, Z), spacing)
        for i in range(nq):
            r = ci * nq + i
            W = [d - int(np.float32(ln[i, a]) / np.float32(spacing)) - 2
                 for a, d in enumerate((X, Y, Z))]
            if min(W) <= 0:
                continue
            Lf = np.fft.rfftn(lig[i].astype(np.float64), axes=(1, 2, 3))
            S = (np.conj(Lf) * Pf).sum(axis=0)
            e = np.fft.irfftn(S, s=(X, Y, Z), axes=(0, 1, 2))[: W[0], : W[1], : W[2]]
            flat = int(np.argmin(e))
            minE[r] = e.reshape(-1)[flat]
            idx[r] = np.unravel_index(flat, e.shape)
    return minE, idx


def _mask_ptr(mask):
    if mask is None:
        return None, None
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    return m, m.ctypes.data_as(C.c_void_p)


def pair_rmsd(coor, mask=None):
    """All-pairs superposition RMSD (reference i, target j), the clustering's recipe."""
    coor = np.ascontiguousarray(coor, dtype=np.float64)
    nconf, natom = coor.shape[:2]
    out = np.empty((nconf, nconf), np.float64)
    m, mp = _mask_ptr(mask)
    orc().orc_pair_rmsd(nconf, natom, coor.ctypes.data_as(_dp), mp, out.ctypes.data_as(_dp))
    return out


def cluster_conformers(coor, energy, cutoff=1.5, max_num=100, mask=None):
    """Greedy leader clustering of src/GeneDiverseConformations.cpp:84-111; centre indices."""
    coor = np.ascontiguousarray(coor, dtype=np.float64)
    energy = np.ascontiguousarray(energy, dtype=np.float64)
    nconf, natom = coor.shape[:2]
    out = np.empty(max(nconf, 1), np.int32)
    m, mp = _mask_ptr(mask)
    n = orc().orc_cluster_conformers(nconf, natom, coor.ctypes.data_as(_dp),
                                     energy.ctypes.data_as(_dp), mp, cutoff, max_num,
                                     out.ctypes.data_as(_ip))
    return out[:n].copy()


def kabsch_rmsd(a, b):
    """Independent form of the superposition RMSD (SVD of the correlation, numpy)."""
    a = a - a.mean(axis=0)
    b = b - b.mean(axis=0)
    h = a.T @ b
    u, s, vt = np.linalg.svd(h)
    d = np.sign(np.linalg.det(h)) or 1.0
    lam = s[0] + s[1] + d * s[2]
    e = ((a * a).sum() + (b * b).sum() - 2.0 * lam) / len(a)
    return float(np.sqrt(max(e, 0.0)))
