"""Serving: continuous batching of docking requests over one resident receptor.

Thin wrapper of the C-ABI server (cdk_server_*, cdocker_b200/csrc/server.cu) plus a Poisson
load generator. Requests are admitted by free device arena, packed across requests into
shared waves, and their latency (submit -> results) is recorded per request.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .api import Receptor, _f32, _i32, _pf, _pi


@dataclass
class Ticket:
    id: int
    n_rot: int
    t_submit: float


class Server:
    def __init__(self, receptor: Receptor, arena_bytes: int = 1 << 30, wave_rotations: int = 1024,
                 max_box: int = 0, max_atoms: int = 128, max_conformers: int = 1 << 16,
                 max_waiting: int = 4096, inject_fault_wave: int = -1):
        lib = L.lib()
        o = L.CdkServerOpts()
        lib.cdk_server_opts_default(C.byref(o))
        o.arena_bytes = arena_bytes
        o.wave_rotations = wave_rotations
        o.max_box = max_box
        o.max_atoms = max_atoms
        o.max_conformers = max_conformers
        o.max_waiting = max_waiting
        # test switch: the host sets the device-wait fault word of this wave (0-based)
        o.reserved[0] = inject_fault_wave + 1 if inject_fault_wave >= 0 else 0
        h = C.c_void_p()
        L.check(lib.cdk_server_create(receptor.handle, C.byref(o), C.byref(h)))
        self._h = h
        self.receptor = receptor

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().cdk_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, coor, charge, eps, slot, quats) -> Ticket:
        c = _f32(coor)
        if c.ndim == 2:
            c = c[None]
        q = _f32(quats).reshape(c.shape[0], -1, 4)
        t = C.c_uint64(0)
        L.check(L.lib().cdk_server_submit(self._h, c.shape[1], c.shape[0], _pf(c),
                                          _pf(_f32(charge)), _pf(_f32(eps)), _pi(_i32(slot)),
                                          q.shape[1], _pf(q), C.byref(t)))
        return Ticket(int(t.value), c.shape[0] * q.shape[1], time.perf_counter())

    def poll(self, ticket: Ticket, wait_ms: int = -1):
        """(minE, idx, timing_ms[queue, run, total]) when done, None while running."""
        e = np.empty(ticket.n_rot, np.float32)
        i = np.empty((ticket.n_rot, 3), np.int32)
        tm = np.zeros(3, np.float64)
        rc = L.lib().cdk_server_poll(self._h, C.c_uint64(ticket.id), int(wait_ms), _pf(e), _pi(i),
                                     tm.ctypes.data_as(C.POINTER(C.c_double)))
        if rc == L.CDK_ERR_BUSY:
            return None
        L.check(rc)
        return e, i, tm

    def stats(self) -> dict:
        out = np.zeros(9, np.float64)
        L.check(L.lib().cdk_server_stats(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), 9))
        return {"waves": int(out[0]), "rotations": int(out[1]), "launches": int(out[2]),
                "completed": int(out[3]), "p50_ms": float(out[4]), "p99_ms": float(out[5]),
                "waiting": int(out[6]), "in_flight": int(out[7]), "tc_waves": int(out[8])}


def poisson_arrivals(rate_hz: float, duration_s: float, seed: int) -> np.ndarray:
    """Arrival times (s) of a Poisson process of the given rate over [0, duration)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            return np.asarray(out)
        out.append(t)


def make_requests(n_req: int, seed: int, spacing: float, grid_len, probe_radii, atoms=(10, 80),
                  confs=(10, 200), rots=(500, 5000), max_rot_total=None):
    """Seeded request mix: ligand size U(atoms), conformers U(confs), rotations per request
    U(rots) split over its conformers; every rotation passes the reference filter."""
    from . import synth
    from .api import filter_quaternions, quaternion_uniform_sampling, vdw_slots
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n_req):
        na = int(rng.integers(atoms[0], atoms[1] + 1))
        nconf = int(rng.integers(confs[0], confs[1] + 1))
        nrot = int(rng.integers(rots[0], rots[1] + 1))
        nq = max(1, nrot // nconf)
        radius = 4.0 * (na / 24) ** (1 / 3)
        xyz, radii, eps, charge = synth.make_ligand(na, radius, seed * 1000 + k)
        coor = synth.make_conformers(xyz, nconf, seed * 1000 + k + 500)
        used, slot = vdw_slots(radii, probe_radii)
        slot_full = used[slot].astype(np.int32)  # index among all probe grids
        q = quaternion_uniform_sampling(seed * 1000 + k + 900, nconf, nq)
        for c in range(nconf):
            kept = filter_quaternions(coor[c], q[c], grid_len, nq)
            assert kept.shape[0] == nq
        reqs.append({"coor": coor, "charge": charge, "eps": eps, "slot": slot,
                     "slot_full": slot_full, "quats": q,
                     "atoms": na, "conformers": nconf, "rotations": nconf * nq})
    return reqs


def run_load(server: Server, requests, arrivals) -> dict:
    """Submits requests at the given arrival times (s, relative to start) and waits for all;
    returns throughput and latency percentiles measured on the host clock."""
    t0 = time.perf_counter()
    tickets = []
    for req, at in zip(requests, arrivals):
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        tickets.append((server.submit(req["coor"], req["charge"], req["eps"], req["slot_full"],
                                      req["quats"]), req))
    lat, rots = [], 0
    for t, req in tickets:
        res = server.poll(t, -1)
        lat.append(res[2][2])
        rots += t.n_rot
    wall = time.perf_counter() - t0
    lat = np.sort(np.asarray(lat))
    return {"requests": len(tickets), "rotations": rots, "wall_s": wall,
            "rotations_per_s": rots / wall, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat[-1])}
