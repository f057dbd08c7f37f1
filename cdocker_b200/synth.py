"""Seeded synthetic docking workloads (no public dataset is involved in this path).

Seed policy: seed s for the receptor, s+1 the ligand, s+2 the conformers, s+3 the quaternion
generator (std::mt19937_64, as the reference draws them).

Receptor: atoms uniform in a cube of side `box`; radius U(1.5, 2.0) A, epsilon
U(0.05, 0.2) kcal/mol, charge N(0, 0.3). Grids: n^3 at spacing h centred on the cube,
xlen = (n-1) h; 8 soft-core capped LJ vdW grids at probe radii linspace(1.2, 2.2, 8) (cap
+3 kcal/mol) and one Coulomb grid with eps(r) = 4r (cap +-40).
Ligand: atoms uniform in a ball of radius `lig_radius`; radius class U{0..7} (the atom radius
is that probe radius, so each class maps to one vdW grid), epsilon U(0.02, 0.2), charges
N(0, 0.3) shifted to sum to zero. Conformers: the ligand with every atom moved by
U(-0.5, 0.5) A per axis.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import api

PROBE_RADII = np.linspace(1.2, 2.2, 8).astype(np.float32)


@dataclass
class Workload:
    name: str
    n: int
    spacing: float
    mid: np.ndarray
    length: np.ndarray
    grid_radii: np.ndarray      # [8]
    all_grids: np.ndarray       # [9, n, n, n] (8 vdW + elec)
    coor: np.ndarray            # [nConf, nAtom, 3]
    charge: np.ndarray          # [nAtom]
    eps: np.ndarray             # [nAtom]
    radii: np.ndarray           # [nAtom]
    used_idx: np.ndarray        # used vdW grid indices
    slot: np.ndarray            # [nAtom] slot among the used grids
    grids: np.ndarray           # [K, n, n, n] used vdW grids then elec
    quats: np.ndarray           # [nConf, nQ, 4] (all pass the filter)
    meta: dict = field(default_factory=dict)

    @property
    def K(self) -> int:
        return self.grids.shape[0]

    @property
    def n_rot(self) -> int:
        return self.quats.shape[0] * self.quats.shape[1]


CONFIGS = {
    # name: (n, receptor atoms, box A, ligand atoms, ligand radius A, conformers, rotations)
    "c0_32": (32, 400, 16.0, 24, 4.0, 1, 500),
    "c1_64": (64, 2500, 32.0, 40, 4.0 * (40 / 24) ** (1 / 3), 100, 1000),
    "c3_96": (96, 6000, 48.0, 40, 4.0 * (40 / 24) ** (1 / 3), 10, 500),
    "c4_128": (128, 12000, 64.0, 60, 4.0 * (60 / 24) ** (1 / 3), 500, 2000),
}


def make_receptor(n: int, n_atoms: int, box: float, seed: int, spacing: float = 0.5):
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(0.0, box, size=(n_atoms, 3)).astype(np.float32)
    radius = rng.uniform(1.5, 2.0, n_atoms).astype(np.float32)
    sqrt_eps = np.sqrt(rng.uniform(0.05, 0.2, n_atoms)).astype(np.float32)
    charge = rng.normal(0.0, 0.3, n_atoms).astype(np.float32)
    mid = np.full(3, box / 2, np.float32)
    length = np.full(3, (n - 1) * spacing, np.float32)
    origin = (mid - length / 2).astype(np.float32)
    grids = api.synth_receptor_grids(n, spacing, origin, xyz, radius, sqrt_eps, charge,
                                     PROBE_RADII)
    return grids, mid, length


def make_ligand(n_atoms: int, radius: float, seed: int):
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < n_atoms:
        p = rng.uniform(-radius, radius, 3)
        if np.dot(p, p) <= radius * radius:
            pts.append(p)
    xyz = np.asarray(pts, np.float32)
    cls = rng.integers(0, 8, n_atoms)
    radii = PROBE_RADII[cls].astype(np.float32)
    eps = rng.uniform(0.02, 0.2, n_atoms).astype(np.float32)
    charge = rng.normal(0.0, 0.3, n_atoms)
    charge = (charge - charge.mean()).astype(np.float32)
    return xyz, radii, eps, charge


def make_conformers(base: np.ndarray, n_conf: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = rng.uniform(-0.5, 0.5, size=(n_conf,) + base.shape)
    return (base[None].astype(np.float64) + d).astype(np.float32)


def make_workload(name: str = "c0_32", seed: int = 0, n_conf: int | None = None,
                  n_q: int | None = None, grids_cache: dict | None = None,
                  n_atoms: int | None = None, ligand_radius: float | None = None) -> Workload:
    n, n_rec, box, n_lig, lig_r, conf_default, q_default = CONFIGS[name]
    n_lig = n_lig if n_atoms is None else n_atoms
    lig_r = lig_r if ligand_radius is None else ligand_radius
    n_conf = conf_default if n_conf is None else n_conf
    n_q = q_default if n_q is None else n_q
    spacing = 0.5
    key = (name, seed)
    if grids_cache is not None and key in grids_cache:
        all_grids, mid, length = grids_cache[key]
    else:
        all_grids, mid, length = make_receptor(n, n_rec, box, seed, spacing)
        if grids_cache is not None:
            grids_cache[key] = (all_grids, mid, length)
    xyz, radii, eps, charge = make_ligand(n_lig, lig_r, seed + 1)
    coor = make_conformers(xyz, n_conf, seed + 2)
    used_idx, slot = api.vdw_slots(radii, PROBE_RADII)
    grids = np.concatenate([all_grids[used_idx], all_grids[-1:]], axis=0)
    quats = api.quaternion_uniform_sampling(seed + 3, n_conf, n_q)
    # every rotation of every conformer must pass the reference filter for a uniform batch
    for c in range(n_conf):
        kept = api.filter_quaternions(coor[c], quats[c], length, n_q)
        if kept.shape[0] != n_q:
            raise RuntimeError(f"conformer {c}: only {kept.shape[0]} of {n_q} rotations fit")
    return Workload(name=name, n=n, spacing=spacing, mid=mid, length=length,
                    grid_radii=PROBE_RADII.copy(), all_grids=all_grids, coor=coor,
                    charge=charge, eps=eps, radii=radii, used_idx=used_idx, slot=slot,
                    grids=np.ascontiguousarray(grids), quats=quats,
                    meta={"seed": seed, "receptor_atoms": n_rec, "box": box,
                          "ligand_atoms": n_lig, "ligand_radius": lig_r})


def conformer_ensemble(seed: int, n_atoms: int = 40, n_conf: int = 1000, n_rotors: int = 6,
                       bond: float = 1.5):
    """Random-rotor conformers of one chain ligand, like the 1000 random conformers the
    reference draws before clustering (src/GeneDiverseConformations.cpp:30-47): a chain with
    tetrahedral bond angles; per conformer every rotor bond is set to a uniform angle in
    (-pi, pi) (the atoms past the bond turn about it), then the whole conformer gets a random
    rigid rotation and translation, so that only superposition sees the shape. Energies are a
    seeded smooth function of the shape (compact conformers lower) plus noise.
    Returns coords [n_conf][n_atoms][3] float64 and energies [n_conf] float64."""
    rng = np.random.default_rng(seed)
    # chain with 109.5 degree bond angles and random dihedrals
    pts = [np.zeros(3), np.array([bond, 0.0, 0.0])]
    ang = np.deg2rad(109.5)
    prev = np.array([0.0, 1.0, 0.0])
    for _ in range(n_atoms - 2):
        u = pts[-1] - pts[-2]
        u /= np.linalg.norm(u)
        w = np.cross(u, prev)
        if np.linalg.norm(w) < 1e-6:
            w = np.cross(u, [0.0, 0.0, 1.0])
        w /= np.linalg.norm(w)
        v = np.cross(w, u)
        phi = rng.uniform(-np.pi, np.pi)
        d = -np.cos(ang) * u + np.sin(ang) * (np.cos(phi) * v + np.sin(phi) * w)
        prev = u
        pts.append(pts[-1] + bond * d)
    base = np.array(pts)
    rotors = np.sort(rng.choice(np.arange(1, n_atoms - 2), size=min(n_rotors, n_atoms - 3),
                                replace=False))

    def axis_rot(axis, t):
        axis = axis / np.linalg.norm(axis)
        K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
        return np.eye(3) + np.sin(t) * K + (1 - np.cos(t)) * (K @ K)

    out = np.empty((n_conf, n_atoms, 3))
    energy = np.empty(n_conf)
    for c in range(n_conf):
        x = base.copy()
        for r in rotors:
            R = axis_rot(x[r + 1] - x[r], rng.uniform(-np.pi, np.pi))
            x[r + 1:] = (x[r + 1:] - x[r + 1]) @ R.T + x[r + 1]
        rg = np.sqrt(((x - x.mean(0)) ** 2).sum(1).mean())
        energy[c] = 5.0 * rg + rng.normal(0.0, 1.0)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w_, a_, b_, c_ = q
        Rr = np.array([[1 - 2 * (b_ * b_ + c_ * c_), 2 * (a_ * b_ - c_ * w_), 2 * (a_ * c_ + b_ * w_)],
                       [2 * (a_ * b_ + c_ * w_), 1 - 2 * (a_ * a_ + c_ * c_), 2 * (b_ * c_ - a_ * w_)],
                       [2 * (a_ * c_ - b_ * w_), 2 * (b_ * c_ + a_ * w_), 1 - 2 * (a_ * a_ + b_ * b_)]])
        out[c] = x @ Rr.T + rng.uniform(-10, 10, size=3)
    return out, energy
