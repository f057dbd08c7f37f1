"""GPU conformer selection (cdk_cluster_conformers / cdk_pair_rmsd) against the oracle:
bit-identical RMSDs and identical centre lists (src/GeneDiverseConformations.cpp:84-111)."""
import numpy as np
import pytest

from cdocker_b200 import _lib, conformers, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_conf,n_atoms,n_rotors", [(1, 5, 1), (37, 24, 3), (300, 40, 4),
                                                     (100, 70, 5)])
def test_pair_rmsd_bit_exact(n_conf, n_atoms, n_rotors):
    x, _ = synth.conformer_ensemble(11, n_atoms=n_atoms, n_conf=n_conf, n_rotors=n_rotors)
    got = conformers.pair_rmsd(x)
    want = O.pair_rmsd(x)
    assert np.array_equal(got, want), np.abs(got - want).max()


def test_pair_rmsd_mask_bit_exact():
    x, _ = synth.conformer_ensemble(12, n_atoms=33, n_conf=65, n_rotors=3)
    mask = (np.arange(33) % 3 != 1).astype(np.uint8)
    assert np.array_equal(conformers.pair_rmsd(x, mask), O.pair_rmsd(x, mask))


@pytest.mark.parametrize("seed,n_conf,n_rotors,max_num", [
    (1, 1000, 6, 100),   # the reference's shape: 1000 random-rotor conformers, 100 centres
    (2, 1000, 3, 1000),
    (3, 333, 2, 0),      # no limit
    (4, 200, 4, 1),      # the limit-1 quirk
    (5, 1, 3, 100),      # one conformer
    (6, 2049, 3, 64),    # rows spanning many 32-bit words
])
def test_cluster_matches_oracle(seed, n_conf, n_rotors, max_num):
    x, e = synth.conformer_ensemble(seed, n_atoms=40, n_conf=n_conf, n_rotors=n_rotors)
    got = conformers.cluster_conformers(x, e, 1.5, max_num)
    want = O.cluster_conformers(x, e, 1.5, max_num)
    np.testing.assert_array_equal(got, want)


def test_cluster_ties_mask_and_errors():
    x, e = synth.conformer_ensemble(9, n_atoms=30, n_conf=150, n_rotors=3)
    e = np.round(e)  # many equal energies: std::sort's (unstable) order must match
    mask = (np.arange(30) < 20).astype(np.uint8)
    np.testing.assert_array_equal(conformers.cluster_conformers(x, e, 1.5, 50, mask),
                                  O.cluster_conformers(x, e, 1.5, 50, mask))
    same = np.repeat(x[:1], 7, axis=0)
    assert list(conformers.cluster_conformers(same, np.zeros(7), 1.5, 100)) == \
        list(O.cluster_conformers(same, np.zeros(7), 1.5, 100))
    bad = e.copy()
    bad[3] = np.nan
    with pytest.raises(_lib.CdkError):
        conformers.cluster_conformers(x, bad)
    with pytest.raises(_lib.CdkError):
        conformers.cluster_conformers(x, e, atom_mask=np.zeros(30, np.uint8))
