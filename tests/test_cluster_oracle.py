"""The conformer-selection oracle (oracle/cdk_oracle.cpp, restating
src/GeneDiverseConformations.cpp:84-111) pinned against an independent numpy form.

OBAlign (OpenBabel) is absent, so the reference's own RMSD cannot run here; the pin is an SVD
(Kabsch) evaluation of the same minimum RMSD and a pure-Python restatement of the greedy loop.
"""
import numpy as np
import pytest

from cdocker_b200 import synth
from oracle import oracle as O


def greedy_py(coords, energy, cutoff, max_num):
    """The reference loop with the SVD RMSD (candidate = reference, centre = target)."""
    idx = sorted(range(len(energy)), key=lambda i: energy[i])  # ties: none in these inputs
    centers = [idx[0]]
    margin = np.inf
    for i in range(1, len(idx)):
        new = True
        for c in centers:
            r = O.kabsch_rmsd(coords[idx[i]], coords[c])
            margin = min(margin, abs(r - cutoff))
            if r <= cutoff:
                new = False
                break
        if new:
            centers.append(idx[i])
        if len(centers) == max_num:
            break
    return np.array(centers), margin


@pytest.mark.parametrize("n_rotors", [2, 4])
def test_pair_rmsd_matches_svd(n_rotors):
    x, _ = synth.conformer_ensemble(3, n_atoms=24, n_conf=48, n_rotors=n_rotors)
    R = O.pair_rmsd(x)
    K = np.array([[O.kabsch_rmsd(x[i], x[j]) for j in range(48)] for i in range(48)])
    big = K > 0.5
    assert big.sum() > 100
    np.testing.assert_allclose(R[big], K[big], rtol=1e-11)
    # the identity pairs: rounding noise of (Ga + Gb - 2 lambda) only
    assert np.abs(np.diag(R)).max() < 1e-5
    # invariant under a rigid motion of the target
    th = 0.7
    Rz = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    y = x @ Rz.T + np.array([3.0, -2.0, 5.0])
    R2 = O.pair_rmsd(np.concatenate([x[:8], y[:8]]))
    np.testing.assert_allclose(R2[:8, 8:][big[:8, :8]], R[:8, :8][big[:8, :8]], rtol=1e-11)


@pytest.mark.parametrize("seed,n_rotors,max_num", [(1, 2, 1000), (2, 3, 1000), (3, 4, 10),
                                                   (4, 3, 1), (5, 2, 0)])
def test_cluster_matches_python_loop(seed, n_rotors, max_num):
    x, e = synth.conformer_ensemble(seed, n_atoms=24, n_conf=120, n_rotors=n_rotors)
    want, margin = greedy_py(x, e, 1.5, max_num)
    assert margin > 1e-9  # no decision within rounding of the cut-off
    got = O.cluster_conformers(x, e, 1.5, max_num)
    np.testing.assert_array_equal(got, want)


def test_cluster_limit_quirk():
    # a limit of 1 stops only when the second conformer joins the first centre
    x, e = synth.conformer_ensemble(7, n_atoms=24, n_conf=60, n_rotors=4)
    full = O.cluster_conformers(x, e, 1.5, 0)
    one = O.cluster_conformers(x, e, 1.5, 1)
    order = np.argsort(e, kind="stable")
    second_is_centre = O.kabsch_rmsd(x[order[1]], x[order[0]]) > 1.5
    if second_is_centre:
        np.testing.assert_array_equal(one, full)
    else:
        assert list(one) == [order[0]]
    # a limit reached from below is honoured
    assert len(full) >= 3
    np.testing.assert_array_equal(O.cluster_conformers(x, e, 1.5, 3), full[:3])


def test_cluster_mask_and_identical():
    x, e = synth.conformer_ensemble(8, n_atoms=24, n_conf=40, n_rotors=3)
    mask = np.zeros(24, np.uint8)
    mask[::2] = 1
    want, margin = greedy_py(x[:, ::2], e, 1.5, 1000)
    assert margin > 1e-9
    np.testing.assert_array_equal(O.cluster_conformers(x, e, 1.5, 1000, mask=mask), want)
    # identical conformers collapse to the lowest-energy one
    same = np.repeat(x[:1], 5, axis=0)
    assert list(O.cluster_conformers(same, np.arange(5.0)[::-1].copy(), 1.5, 100)) == [4]
