"""Pins the oracle against the reference's own code (CPU, no GPU).

The reference ships no tests or golden vectors for this path, so the oracle restatement
(oracle/cdk_oracle.cpp) is checked two ways: against the reference's helpers compiled from
their sources (oracle/_ref/libcdk_ref.so, when present) and against the committed fixtures
under tests/golden/ (generated by tests/golden/make_golden.py from those same helpers). The
product's host helpers (libcdock_b200.so) are held to the same bit-exact bar.
"""
import os

import numpy as np
import pytest

from cdocker_b200 import api
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "c0_32_seed0.npz")
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@needs_ref
@pytest.mark.parametrize("seed", [0, 3, 12345, 2**63 + 7])
def test_quaternion_sampling_bitexact(seed):
    R = O.ref()
    a = np.empty((3, 257, 4), np.float32)
    R.ref_quaternion_uniform_sampling(seed, 3, 257, O._pf(a))
    assert np.array_equal(_bits(a), _bits(O.sample_quaternions(seed, 3, 257)))
    assert np.array_equal(_bits(a), _bits(api.quaternion_uniform_sampling(seed, 3, 257)))


@needs_ref
def test_rotate_and_bbox_bitexact(c0):
    R = O.ref()
    q = c0.quats[0, :64]
    rot, mn, ln = O.rotate_bbox(c0.coor[0], q)
    rr = np.empty_like(rot)
    for i in range(q.shape[0]):
        for a in range(c0.coor.shape[1]):
            R.ref_rotate(O._pf(np.ascontiguousarray(q[i])), O._pf(np.ascontiguousarray(c0.coor[0, a])),
                         O._pf(rr[i, a]))
    assert np.array_equal(_bits(rot), _bits(rr))
    rmn = np.empty((q.shape[0], 3), np.float32)
    rmx = np.empty((q.shape[0], 3), np.float32)
    R.ref_min_max_coors(q.shape[0], rot.shape[1], O._pf(rr), O._pf(rmn), O._pf(rmx))
    assert np.array_equal(_bits(mn), _bits(rmn))
    assert np.array_equal(_bits(ln), _bits(rmx - rmn))


@needs_ref
@pytest.mark.parametrize("max_n", [500, 320, 1])
def test_filter_bitexact_including_shuffle(c0, max_n):
    """Kept set and order, with the std::random_shuffle cap; every run starts from srand(1)."""
    R = O.ref()
    # a grid length that rejects part of the rotations so both branches matter
    glen = np.full(3, 7.9, np.float32)
    q = c0.quats[0]
    out = np.empty_like(q)
    R.ref_srand(1)
    n = R.ref_filter_quaternions(O._pf(np.ascontiguousarray(c0.coor[0])), c0.coor.shape[1], q.shape[0],
                                 O._pf(q), 7.9, 7.9, 7.9, max_n, O._pf(out))
    ref = out[:n]
    O.orc().orc_srand(1)
    mine = O.filter_quaternions(c0.coor[0], q, glen, max_n)
    R.ref_srand(1)
    prod = api.filter_quaternions(c0.coor[0], q, glen, max_n)
    assert np.array_equal(_bits(ref), _bits(mine))
    assert np.array_equal(_bits(ref), _bits(prod))


@needs_ref
def test_vdw_slots_bitexact_with_ties():
    R = O.ref()
    g = np.linspace(1.2, 2.2, 8).astype(np.float32)
    rng = np.random.default_rng(5)
    radii = rng.uniform(1.0, 2.5, 200).astype(np.float32)
    # exact midpoints between neighbouring probe radii: the first minimum must win
    radii[:7] = ((g[:-1].astype(np.float64) + g[1:]) / 2).astype(np.float32)
    radii[7:10] = g[[0, 3, 7]]
    used = np.empty(8, np.int32)
    slot = np.empty(200, np.int32)
    n = R.ref_vdw_slots(200, O._pf(radii), 8, O._pf(g), O._pi(used), O._pi(slot))
    u2, s2 = O.vdw_slots(radii, g)
    u3, s3 = api.vdw_slots(radii, g)
    assert np.array_equal(used[:n], u2) and np.array_equal(slot, s2)
    assert np.array_equal(used[:n], u3) and np.array_equal(slot, s3)


@needs_ref
def test_fill_bitexact_vs_reference(c0):
    R = O.ref()
    rot, mn, _ = O.rotate_bbox(c0.coor[0], c0.quats[0, :3])
    mine = O.fill_ligand_grid(rot, mn, c0.charge, c0.eps, c0.slot, c0.K - 1, (32, 32, 32), 0.5)
    ref = np.zeros_like(mine)
    R.ref_fill_ligand_grid(3, rot.shape[1], O._pf(rot), O._pf(mn), O._pf(O._f32(c0.charge)),
                           O._pf(O._f32(c0.eps)), O._pf(O._f32(c0.radii)), 8,
                           O._pf(O._f32(c0.grid_radii)), 32, 32, 32, 0.5, O._pf(ref))
    assert np.array_equal(_bits(mine), _bits(ref))


def test_golden_quaternions_and_filter(gold, c0):
    assert np.array_equal(_bits(O.sample_quaternions(3, 1, 500)), _bits(gold["quats"]))
    assert np.array_equal(_bits(api.quaternion_uniform_sampling(3, 1, 500)), _bits(gold["quats"]))
    O.orc().orc_srand(1)
    kept = O.filter_quaternions(c0.coor[0], gold["quats"][0], gold["filter_len"], int(gold["filter_max"]))
    assert np.array_equal(_bits(kept), _bits(gold["filtered"]))


def test_golden_slots_and_fill(gold, c0):
    used, slot = O.vdw_slots(c0.radii, c0.grid_radii)
    assert np.array_equal(used, gold["used_idx"]) and np.array_equal(slot, gold["slot"])
    rot, mn, _ = O.rotate_bbox(c0.coor[0], gold["quats"][0, :4])
    fill = O.fill_ligand_grid(rot, mn, c0.charge, c0.eps, slot, len(used), (32, 32, 32), 0.5)
    assert np.array_equal(_bits(fill), _bits(gold["fill4"]))


def test_golden_search_fp64_and_fp32(gold, c0):
    q = gold["quats"][:, :60]
    m32, i32, m64 = O.search_direct(c0.grids, 0.5, c0.coor, c0.charge, c0.eps, c0.slot, q, prec=1)
    np.testing.assert_allclose(m64, gold["minE64"][:60], rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(i32, gold["idx64"][:60])
    f32, fi, _ = O.search_direct(c0.grids, 0.5, c0.coor, c0.charge, c0.eps, c0.slot, q, prec=0)
    assert np.array_equal(_bits(f32), _bits(gold["minE32"][:60]))
    np.testing.assert_array_equal(fi, gold["idx32"][:60])


def test_direct_equals_fft64(c0):
    """Two independent FP64 forms of the correlation agree (direct sum vs rfftn/irfftn)."""
    q = c0.quats[:, :12]
    _, i1, m1 = O.search_direct(c0.grids, 0.5, c0.coor, c0.charge, c0.eps, c0.slot, q, prec=1)
    m2, i2 = O.fft64_search(c0.grids, 0.5, c0.coor, c0.charge, c0.eps, c0.slot, q)
    np.testing.assert_allclose(m1, m2, rtol=1e-10, atol=1e-9)
    np.testing.assert_array_equal(i1, i2)


def test_dense_equals_sparse_direct(c0):
    """Skipping zero box cells adds the same nonzero terms in the same order: bit-identical."""
    q = c0.quats[:, :3]
    a = O.search_direct(c0.grids, 0.5, c0.coor, c0.charge, c0.eps, c0.slot, q, prec=0, dense=1)
    b = O.search_direct(c0.grids, 0.5, c0.coor, c0.charge, c0.eps, c0.slot, q, prec=0, dense=0)
    assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])


def test_window_rule_and_empty_window(c0):
    L = O.orc()
    assert L.orc_window(32, np.float32(7.99), np.float32(0.5)) == 32 - 15 - 2
    assert L.orc_window(32, np.float32(8.0), np.float32(0.5)) == 32 - 16 - 2
    big = c0.coor[0] * 4.0
    m, i, _ = O.search_direct(c0.grids, 0.5, big, c0.charge, c0.eps, c0.slot, c0.quats[:, :4])
    assert np.all(np.isinf(m)) and np.all(i == -1)
