"""Generates tests/golden/c0_32_seed0.npz from the reference's own helpers.

Run in a checkout where the reference tree is present (oracle/_ref built):
    python tests/golden/make_golden.py
Inputs are the seeded config-0 workload (32^3 grids, K=9, 24-atom ligand, 500 rotations).
  quats, filtered  -- QuaternionUniformSampling(seed 3) and FilterQuaternions (grid length
                      7.9 A so that some rotations are rejected, cap 320 so the
                      std::random_shuffle branch runs, rand() state from srand(1)),
                      both from oracle/_ref (the reference's code)
  used_idx, slot   -- GetIdxOfAtomsForVdwRadius from oracle/_ref
  fill4            -- FillLigandGrid of the first 4 rotations from oracle/_ref
  minE64, idx64    -- the oracle's FP64 direct correlation (cpuNaive's algorithm) over all 500
  minE32, idx32    -- the same with cpuNaive's float accumulation
  fft64_minE/_idx  -- the float64 FFT form for the first 50 rotations
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cdocker_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    assert O.ref_available(), "build oracle/_ref first (make -C oracle ref)"
    R = O.ref()
    w = synth.make_workload("c0_32", seed=0)
    quats = np.empty((1, 500, 4), np.float32)
    R.ref_quaternion_uniform_sampling(3, 1, 500, O._pf(quats))
    flen = np.full(3, 7.9, np.float32)
    fmax = 320
    out = np.empty((500, 4), np.float32)
    R.ref_srand(1)
    n = R.ref_filter_quaternions(O._pf(np.ascontiguousarray(w.coor[0])), w.coor.shape[1], 500,
                                 O._pf(np.ascontiguousarray(quats[0])), 7.9, 7.9, 7.9, fmax,
                                 O._pf(out))
    filtered = out[:n].copy()
    used = np.empty(8, np.int32)
    slot = np.empty(w.coor.shape[1], np.int32)
    nu = R.ref_vdw_slots(w.coor.shape[1], O._pf(O._f32(w.radii)), 8,
                         O._pf(O._f32(w.grid_radii)), O._pi(used), O._pi(slot))
    used = used[:nu].copy()
    rot, mn, _ = O.rotate_bbox(w.coor[0], quats[0, :4])
    fill4 = np.zeros((4, nu + 1, 32, 32, 32), np.float32)
    R.ref_fill_ligand_grid(4, rot.shape[1], O._pf(rot), O._pf(mn), O._pf(O._f32(w.charge)),
                           O._pf(O._f32(w.eps)), O._pf(O._f32(w.radii)), 8,
                           O._pf(O._f32(w.grid_radii)), 32, 32, 32, 0.5, O._pf(fill4))
    _, idx64, m64 = O.search_direct(w.grids, 0.5, w.coor, w.charge, w.eps, slot, quats, prec=1)
    m32, idx32, _ = O.search_direct(w.grids, 0.5, w.coor, w.charge, w.eps, slot, quats, prec=0)
    f64, fi = O.fft64_search(w.grids, 0.5, w.coor, w.charge, w.eps, slot, quats[:, :50])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c0_32_seed0.npz")
    np.savez_compressed(path, quats=quats, filter_len=flen, filter_max=np.int32(fmax),
                        filtered=filtered, used_idx=used, slot=slot, fill4=fill4, minE64=m64,
                        idx64=idx64, minE32=m32, idx32=idx32, fft64_minE=f64, fft64_idx=fi)
    print(path, "filtered", n, "used", nu, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
