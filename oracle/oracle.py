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


def build(ref: bool = True) -> None:
    """Builds libcdk_oracle.so and, with ref, the reference libraries through build_ref.sh
    (which does nothing where no reference checkout exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref:
        subprocess.run(["sh", os.path.join(HERE, "build_ref.sh")], check=True)


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
        L.orc_synth_receptor_grids.argtypes = [C.c_int, C.c_float, _fp, C.c_int, _fp, _fp, _fp,
                                               _fp, C.c_int, _fp, C.c_float, C.c_float, C.c_float,
                                               _fp]
        L.orc_synth_receptor_grids.restype = None
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
        L.ref_sort_index.argtypes = [C.c_int, _fp, _lp]
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
        L.refcufft_kernels.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _fp, _fp, _fp, _fp]
        L.refcufft_kernels.restype = C.c_int
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


# ------------------------------------------------------------------ inputs without the product
def synth_receptor_grids(n, spacing, origin, xyz, radius, sqrt_eps, charge, probe_radii,
                         vdw_cap=3.0, elec_cap=40.0, cutoff=12.0):
    """Receptor potential grids [len(probe_radii)+1, n, n, n] (orc_synth_receptor_grids)."""
    p = _f32(probe_radii)
    xyz = _f32(xyz).reshape(-1, 3)
    out = np.empty((p.shape[0] + 1, n, n, n), np.float32)
    orc().orc_synth_receptor_grids(n, float(spacing), _pf(_f32(origin)), xyz.shape[0], _pf(xyz),
                                   _pf(_f32(radius)), _pf(_f32(sqrt_eps)), _pf(_f32(charge)),
                                   p.shape[0], _pf(p), float(vdw_cap), float(elec_cap),
                                   float(cutoff), _pf(out))
    return out


def reference_inputs(name, seed=0, n_conf=None, n_q=None, n_atoms=None, ligand_radius=None):
    """The benchmark workload built without the product library, for the reference arm: the
    same seeds and shapes as cdocker_b200.synth.make_workload (its numpy ligand and conformer
    generators are imported; they load no library), receptor grids from
    orc_synth_receptor_grids, quaternion sampling and vdW slots from the reference's own helpers
    (oracle/_ref) -- or their restatements here when _ref is absent -- and the filter check
    from the restatement.
    Returns a dict with grids [K,n,n,n], all_grids, coor, charge, eps, radii, slot, quats,
    spacing, length, grid_radii."""
    from cdocker_b200 import synth as S  # numpy only: make_ligand, make_conformers, constants
    n, n_rec, box, n_lig, lig_r, conf_default, q_default = S.CONFIGS[name]
    n_lig = n_lig if n_atoms is None else n_atoms
    lig_r = lig_r if ligand_radius is None else ligand_radius
    n_conf = conf_default if n_conf is None else n_conf
    n_q = q_default if n_q is None else n_q
    spacing = 0.5
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(0.0, box, size=(n_rec, 3)).astype(np.float32)
    radius = rng.uniform(1.5, 2.0, n_rec).astype(np.float32)
    sqrt_eps = np.sqrt(rng.uniform(0.05, 0.2, n_rec)).astype(np.float32)
    charge_r = rng.normal(0.0, 0.3, n_rec).astype(np.float32)
    mid = np.full(3, box / 2, np.float32)
    length = np.full(3, (n - 1) * spacing, np.float32)
    origin = (mid - length / 2).astype(np.float32)
    all_grids = synth_receptor_grids(n, spacing, origin, xyz, radius, sqrt_eps, charge_r,
                                     S.PROBE_RADII)
    lxyz, radii, eps, charge = S.make_ligand(n_lig, lig_r, seed + 1)
    coor = S.make_conformers(lxyz, n_conf, seed + 2)
    use_ref = ref_available()
    g = _f32(S.PROBE_RADII)
    r = _f32(radii)
    used = np.empty(g.shape[0], np.int32)
    slot = np.empty(r.shape[0], np.int32)
    if use_ref:
        nu = ref().ref_vdw_slots(r.shape[0], _pf(r), g.shape[0], _pf(g), _pi(used), _pi(slot))
        quats = np.empty((n_conf, n_q, 4), np.float32)
        ref().ref_quaternion_uniform_sampling(seed + 3, n_conf, n_q, _pf(quats))
    else:
        nu = orc().orc_vdw_slots(r.shape[0], _pf(r), g.shape[0], _pf(g), _pi(used), _pi(slot))
        quats = sample_quaternions(seed + 3, n_conf, n_q)
    used = used[:nu].copy()
    for c in range(n_conf):
        qc = _f32(quats[c])
        out = np.empty_like(qc)
        cc = _f32(coor[c])
        # the restated filter (pinned bit-exact to the reference's in tests): the reference's
        # own prints its count to stdout, which would interleave with the bench's JSON line
        kept = orc().orc_filter_quaternions(_pf(cc), cc.shape[0], n_q, _pf(qc), float(length[0]),
                                            float(length[1]), float(length[2]), n_q, _pf(out))
        if kept != n_q:
            raise RuntimeError(f"conformer {c}: only {kept} of {n_q} rotations fit")
    grids = np.ascontiguousarray(np.concatenate([all_grids[used], all_grids[-1:]], axis=0))
    return {"grids": grids, "all_grids": all_grids, "coor": coor, "charge": charge, "eps": eps,
            "radii": radii, "slot": slot, "used": used, "quats": quats, "spacing": spacing,
            "length": length, "grid_radii": S.PROBE_RADII.copy(), "n": n,
            "source": "oracle/_ref (reference helpers)" if use_ref else "oracle restatement"}
