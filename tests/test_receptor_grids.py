"""Receptor potential grids: the host generator against a brute-force numpy restatement, and
the GPU generator (cdk_receptor_grids_gpu) bit-identical to the host one.

The reference reads these grids from CHARMM-written files (src/ReadGrids.cpp:6-68); the
generator sits upstream of that reader, so its definition is the host function's formula.
"""
import ctypes as C

import numpy as np
import pytest

from cdocker_b200 import _lib as L
from cdocker_b200 import api, synth


def _brute(n, spacing, origin, xyz, radius, sqrt_eps, charge, probe, vdw_cap, elec_cap, cutoff):
    """All atoms per grid point (no cell list), float64."""
    h = float(np.float32(spacing))  # the C-ABI takes the spacing as float
    ax = [float(origin[d]) + np.arange(n, dtype=np.float64) * h for d in range(3)]
    P = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3)
    d2 = ((P[:, None, :] - xyz[None].astype(np.float64)) ** 2).sum(-1)
    inside = d2 <= float(cutoff) ** 2
    out = []
    for p in probe.astype(np.float64):
        rmin = radius.astype(np.float64) + p
        dd2 = np.maximum(d2, 0.25 * rmin * rmin)
        s6 = (rmin * rmin / dd2) ** 3
        e = np.where(inside, sqrt_eps.astype(np.float64) * (s6 * s6 - 2.0 * s6), 0.0).sum(1)
        out.append(np.minimum(e, vdw_cap))
    el = np.where(inside, 332.0716 * charge.astype(np.float64) / (4.0 * np.maximum(d2, 0.25)),
                  0.0).sum(1)
    out.append(np.clip(el, -elec_cap, elec_cap))
    return np.stack(out).reshape(len(probe) + 1, n, n, n).astype(np.float32)


def _receptor(n_atoms, box, seed):
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(0.0, box, size=(n_atoms, 3)).astype(np.float32)
    radius = rng.uniform(1.5, 2.0, n_atoms).astype(np.float32)
    sqrt_eps = np.sqrt(rng.uniform(0.05, 0.2, n_atoms)).astype(np.float32)
    charge = rng.normal(0.0, 0.3, n_atoms).astype(np.float32)
    return xyz, radius, sqrt_eps, charge


@pytest.mark.parametrize("cutoff", [4.0, 12.0])
def test_host_grids_match_brute_force(cutoff):
    n, h = 10, 0.7
    xyz, rad, se, q = _receptor(60, 8.0, seed=3)
    origin = np.array([-0.5, 0.25, 0.0], np.float32)
    probe = synth.PROBE_RADII[:3]
    got = api.synth_receptor_grids(n, h, origin, xyz, rad, se, q, probe, 3.0, 40.0, cutoff)
    ref = _brute(n, h, origin, xyz, rad, se, q, probe, 3.0, 40.0, cutoff)
    np.testing.assert_allclose(got, ref, rtol=2e-6, atol=2e-6)


def test_gpu_grids_invalid_arguments():
    f = np.zeros(3, np.float32)
    pf = f.ctypes.data_as(C.POINTER(C.c_float))
    lib = L.lib()
    # 16 vdW probes exceed the kernel's accumulator count
    assert lib.cdk_receptor_grids_gpu(0, 8, 0.5, pf, 1, pf, pf, pf, pf, 16, pf, 3.0, 40.0, 12.0,
                                      pf) == L.CDK_ERR_INVALID
    assert lib.cdk_receptor_grids_gpu(0, 8, 0.5, pf, 1, pf, pf, pf, pf, 1, pf, 3.0, 40.0, 0.0,
                                      pf) == L.CDK_ERR_INVALID
    assert lib.cdk_receptor_grids_gpu(-1, 8, 0.5, pf, 1, pf, pf, pf, pf, 1, pf, 3.0, 40.0, 12.0,
                                      pf) == L.CDK_ERR_INVALID


GPU_CASES = [
    # n, receptor atoms, box, spacing, cutoff, probes
    (32, 400, 16.0, 0.5, 12.0, 8),
    (33, 300, 14.0, 0.45, 5.0, 3),     # ragged point count, several cells per axis
    (64, 2500, 32.0, 0.5, 12.0, 8),
    (20, 0, 10.0, 0.5, 12.0, 2),       # no receptor atoms: all zeros
    (24, 150, 40.0, 0.5, 6.0, 15),     # receptor wider than the grid, 15 probes
]


@pytest.mark.gpu
@pytest.mark.parametrize("n,na,box,h,cut,nv", GPU_CASES)
def test_gpu_grids_bit_identical_to_host(n, na, box, h, cut, nv):
    xyz, rad, se, q = _receptor(na, box, seed=n + na)
    probe = np.linspace(1.0, 2.4, nv).astype(np.float32)
    mid = np.full(3, box / 2, np.float32)
    origin = (mid - (n - 1) * h / 2).astype(np.float32)
    host = api.synth_receptor_grids(n, h, origin, xyz, rad, se, q, probe, 3.0, 40.0, cut)
    dev = api.synth_receptor_grids(n, h, origin, xyz, rad, se, q, probe, 3.0, 40.0, cut, device=0)
    assert dev.shape == (nv + 1, n, n, n)
    assert np.array_equal(dev.view(np.uint32), host.view(np.uint32))
    if na == 0:
        assert not dev.any()
