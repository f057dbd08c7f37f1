"""Array-level API over the C-ABI.

Each function names the reference code whose semantics it keeps; the work happens in
libcdock_b200.so (GPU kernels for the search, host C++ for the bit-exact helpers).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _pf(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def _pi(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def quaternion_uniform_sampling(seed: int, n_conf: int, n_q: int) -> np.ndarray:
    """[n_conf, n_q, 4] Shoemake quaternions from one std::mt19937_64(seed), drawn in turn
    (src/QuaternionUniformSampling.cpp:5-24)."""
    out = np.empty((n_conf, n_q, 4), np.float32)
    L.check(L.lib().cdk_quaternion_uniform_sampling(C.c_uint64(seed), n_conf, n_q, _pf(out)))
    return out


def filter_quaternions(coor, quats, grid_len, max_n: int) -> np.ndarray:
    """FilterQuaternions (src/FilterQuaternions.cpp:11-83). Uses the process-wide rand()."""
    c = _f32(coor).reshape(-1, 3)
    q = _f32(quats).reshape(-1, 4)
    out = np.empty_like(q)
    cnt = C.c_int(0)
    L.check(L.lib().cdk_filter_quaternions(_pf(c), c.shape[0], q.shape[0], _pf(q),
                                           float(grid_len[0]), float(grid_len[1]),
                                           float(grid_len[2]), int(max_n), _pf(out),
                                           C.byref(cnt)))
    return out[: cnt.value].copy()


def vdw_slots(radii, grid_radii):
    """GetIdxOfAtomsForVdwRadius (src/GetIdxOfAtomsForVdwRadius.cpp:4-35).
    Returns (used grid indices, per-atom slot among the used grids)."""
    r = _f32(radii)
    g = _f32(grid_radii)
    used = np.empty(g.shape[0], np.int32)
    slot = np.empty(r.shape[0], np.int32)
    n = C.c_int(0)
    L.check(L.lib().cdk_vdw_slots(r.shape[0], _pf(r), g.shape[0], _pf(g), _pi(used), _pi(slot),
                                  C.byref(n)))
    return used[: n.value].copy(), slot


def fill_ligand_grid(coors, mincoors, charge, eps, slot, n_vdw_used: int, dims, spacing: float):
    """FillLigandGrid on the GPU (src/FillLigandGrid.cpp:7-120), bit-exact.
    coors [nQ, nAtom, 3] rotated; mincoors [nQ, 3]. Returns [nQ, K, x, y, z]."""
    c = _f32(coors)
    nq, na = c.shape[0], c.shape[1]
    m = _f32(mincoors)
    q = _f32(charge)
    e = _f32(eps)
    s = _i32(slot)
    x, y, z = dims
    out = np.empty((nq, n_vdw_used + 1, x, y, z), np.float32)
    L.check(L.lib().cdk_fill_ligand_grid(nq, na, _pf(c), _pf(m), _pf(q), _pf(e), _pi(s),
                                         n_vdw_used, x, y, z, float(spacing), _pf(out)))
    return out


def read_grids(path: str) -> dict:
    """ReadGrids (src/ReadGrids.cpp:6-68)."""
    hi = np.zeros(4, np.int32)
    hf = np.zeros(8, np.float32)
    lib = L.lib()
    L.check(lib.cdk_read_grids(path.encode(), _pi(hi), _pf(hf), None, 0, None, 0))
    ng, x, y, z = (int(v) for v in hi)
    radii = np.zeros(max(ng - 1, 0), np.float32)
    values = np.zeros((ng, x, y, z), np.float32)
    L.check(lib.cdk_read_grids(path.encode(), _pi(hi), _pf(hf), _pf(radii), radii.size,
                               _pf(values), values.size))
    return {"num_grids": ng, "dims": (x, y, z), "mid": hf[0:3].copy(), "len": hf[3:6].copy(),
            "spacing": float(hf[6]), "restraint_k": float(hf[7]), "radii": radii,
            "values": values}


def write_grids(path: str, values, radii, mid, length, spacing: float, restraint_k: float = 0.0):
    v = _f32(values)
    ng, x, y, z = v.shape
    r = _f32(radii)
    L.check(L.lib().cdk_write_grids(path.encode(), ng, x, y, z, _pf(_f32(mid)), _pf(_f32(length)),
                                    float(spacing), float(restraint_k), _pf(r), _pf(v)))


def synth_receptor_grids(n, spacing, origin, xyz, radius, sqrt_eps, charge, probe_radii,
                         vdw_cap=3.0, elec_cap=40.0, cutoff=12.0, device=None) -> np.ndarray:
    """Receptor potential grids [len(probe_radii)+1, n, n, n]: soft-core capped LJ per probe
    radius, then the eps(r)=4r Coulomb grid. device=None computes on the host (multithreaded);
    an int computes on that CUDA device, bit-identical to the host result."""
    p = _f32(probe_radii)
    xyz = _f32(xyz).reshape(-1, 3)
    out = np.empty((p.shape[0] + 1, n, n, n), np.float32)
    head = () if device is None else (int(device),)
    fn = L.lib().cdk_synth_receptor_grids if device is None else L.lib().cdk_receptor_grids_gpu
    L.check(fn(
        *head, n, float(spacing), _pf(_f32(origin)), xyz.shape[0], _pf(xyz), _pf(_f32(radius)),
        _pf(_f32(sqrt_eps)), _pf(_f32(charge)), p.shape[0], _pf(p), float(vdw_cap),
        float(elec_cap), float(cutoff), _pf(out)))
    return out


class Receptor:
    """A receptor grid set with its K spectra resident on one GPU (one cdk_ctx).

    grids: [K, n, n, n] float32, K-1 vdW grids (used ones, ascending) then the elec grid --
    the reference's usedGridValues (src/TranRotaConfSearchNoMini.cu:135-146).
    """

    def __init__(self, grids, spacing: float, device: int = 0, wave_rotations: int = 0,
                 max_atoms: int = 256, col_tile: int = 0, form: int = L.CDK_FORM_FP32,
                 use_graphs: int = 0, profile: bool = False, fft_planes: bool = False,
                 autotune: bool = False, tc_mma_sync: bool = False, tc_build: bool = False,
                 group_rotations: bool = True, tc_stream_tiles: bool = False,
                 tc_hankel: bool = False,
                 tc_cols: int = 0, top_k: int = 0, tie_break: bool = True,
                 yz_block_stages: bool = False, yz_octets: bool = False, tc_ksteps: int = 0,
                 tc_thread_copies: bool = False, tc_tiled_rows: bool = False):
        g = _f32(grids)
        if g.ndim != 4:
            raise ValueError("grids must be [K, n, n, n]")
        self.K, self.n = g.shape[0], g.shape[1]
        self.spacing = float(spacing)
        lib = L.lib()
        opts = L.CdkOpts()
        lib.cdk_opts_default(C.byref(opts))
        opts.device = device
        opts.form = form
        opts.wave_rotations = wave_rotations
        opts.max_atoms = max_atoms
        opts.col_tile = col_tile
        opts.use_graphs = use_graphs
        opts.reserved[0] = 1 if profile else 0
        opts.reserved[1] = ((1 if fft_planes else 0) | (2 if yz_block_stages else 0) |
                            (4 if yz_octets else 0))
        opts.reserved[2] = 1 if autotune else 0
        opts.reserved[3] = (1 if tc_mma_sync else 2 if tc_build else 3 if tc_stream_tiles
                            else 4 if tc_hankel else 0)
        opts.reserved[5] = ((tc_cols & 3) | ((tc_ksteps & 7) << 2) |
                            (32 if tc_thread_copies else 0) | (64 if tc_tiled_rows else 0))
        opts.reserved[6] = top_k
        opts.reserved[7] = 0 if tie_break else 1
        opts.reserved[4] = 0 if group_rotations else 1
        h = C.c_void_p()
        L.check(lib.cdk_ctx_create(g.shape[1], g.shape[2], g.shape[3], self.spacing, self.K,
                                   _pf(g), C.byref(opts), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().cdk_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def search(self, coor, charge, eps, slot, quats, stream: int = 0):
        """Host-buffer search (cdk_search). coor [nConf, nAtom, 3]; quats [nConf, nQ, 4].
        Returns minE [nConf*nQ] float32 and idx [nConf*nQ, 3] int32."""
        c = _f32(coor)
        if c.ndim == 2:
            c = c[None]
        nconf, na = c.shape[0], c.shape[1]
        q = _f32(quats).reshape(nconf, -1, 4)
        nq = q.shape[1]
        minE = np.empty(nconf * nq, np.float32)
        idx = np.empty((nconf * nq, 3), np.int32)
        L.check(L.lib().cdk_search(self._h, na, nconf, _pf(c), _pf(_f32(charge)), _pf(_f32(eps)),
                                   _pi(_i32(slot)), nq, _pf(q), _pf(minE), _pi(idx),
                                   C.c_void_p(stream)))
        return minE, idx

    def search_device(self, n_atom, n_conf, d_coor, d_charge, d_eps, d_slot, n_q, d_quats,
                      d_minE, d_idx, stream: int = 0):
        """Device-pointer search (cdk_search_device); pointers as ints (e.g. tensor.data_ptr())."""
        L.check(L.lib().cdk_search_device(self._h, n_atom, n_conf, C.c_void_p(d_coor),
                                          C.c_void_p(d_charge), C.c_void_p(d_eps),
                                          C.c_void_p(d_slot), n_q, C.c_void_p(d_quats),
                                          C.c_void_p(d_minE), C.c_void_p(d_idx),
                                          C.c_void_p(stream)))

    def rescore_fp64(self, coor, charge, eps, slot, rot_conf, quats, tidx):
        """FP64 direct grid-energy sum of poses (cdk_rescore_fp64)."""
        c = _f32(coor)
        if c.ndim == 2:
            c = c[None]
        rc = _i32(rot_conf)
        q = _f32(quats).reshape(-1, 4)
        t = _i32(tidx).reshape(-1, 3)
        out = np.empty(rc.shape[0], np.float64)
        L.check(L.lib().cdk_rescore_fp64(self._h, c.shape[1], c.shape[0], _pf(c),
                                         _pf(_f32(charge)), _pf(_f32(eps)), _pi(_i32(slot)),
                                         rc.shape[0], _pi(rc), _pf(q), _pi(t),
                                         out.ctypes.data_as(_dp), None))
        return out

    def stats(self) -> dict:
        out = np.zeros(21, np.float64)
        L.check(L.lib().cdk_ctx_stats(self._h, out.ctypes.data_as(_dp), 21))
        names = ["prep", "spread_yz", "xpass", "yz_inv_argmin", "finalize"]
        return {"launches": int(out[0]), "waves": int(out[1]), "rotations": int(out[2]),
                "device_ms": float(out[3]), "box": int(out[4]), "wave_rotations": int(out[5]),
                "planes_spread": int(out[6]), "planes_window": int(out[7]),
                "kernel_ms": {k: float(v) for k, v in zip(names, out[8:13])},
                "col_tile": int(out[13]), "rotations_per_cta": int(out[14]),
                "graph_state": int(out[15]),
                "xpass_kind": ["fp32_radix", "mma_sync", "tcgen05_build",
                               "tcgen05_streamed", "unused",
                               "tcgen05_streamed_fp16", "tcgen05_hankel",
                               "tcgen05_hankel_fp16"][int(out[16])],
                "tensor_steps": int(out[17]), "mma_units": int(out[18]),
                "near_ties_rescored": int(out[19]), "near_ties_changed": int(out[20])}

    def top_poses(self):
        """The FP64 re-scores of each wave's lowest poses from the last search
        (cdk_ctx_top_poses): rot [m], minE [m], idx [m, 3], e64 [m]; m = waves x k."""
        cnt = C.c_int(0)
        L.check(L.lib().cdk_ctx_top_poses(self._h, 0, None, None, None, None, C.byref(cnt)))
        m = cnt.value
        rot = np.empty(m, np.int32)
        e = np.empty(m, np.float32)
        idx = np.empty((m, 3), np.int32)
        e64 = np.empty(m, np.float64)
        if m:
            L.check(L.lib().cdk_ctx_top_poses(self._h, m, _pi(rot), _pf(e), _pi(idx),
                                              e64.ctypes.data_as(_dp), C.byref(cnt)))
        return rot, e, idx, e64
