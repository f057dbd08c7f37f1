"""Pose ranking and reconstruction (src/TranRotaConfSearchNoMini.cu:467-510) on the host:
sort_index against the reference's own template (include/GeneDiverseConformations.h:9-20,
compiled from the header into oracle/_ref), cdk_pose_coordinates against its definition, and
the PDB + energy.txt export."""
import os

import numpy as np
import pytest

from cdocker_b200 import poses, synth
from cdocker_b200.shard import top_k
from oracle import oracle as O


def _ref_sort_index(v):
    out = np.empty(v.shape[0], np.int64)
    O.ref().ref_sort_index(v.shape[0], O._pf(v), out.ctypes.data_as(O._lp))
    return out


@pytest.mark.parametrize("n,levels", [(17, 0), (500, 7), (5000, 40), (20000, 3)])
def test_sort_index_matches_reference_std_sort(n, levels):
    """Equal values come out in std::sort's order (not a stable one): many ties included."""
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(n)
    v = rng.normal(size=n).astype(np.float32)
    if levels:
        v = np.round(v * levels).astype(np.float32)  # heavy ties
    got = poses.sort_index(v)
    want = _ref_sort_index(v)
    assert np.array_equal(got, want)
    assert np.array_equal(top_k(v, 10), want[:10])
    if levels:
        # the order differs from a stable sort on these inputs: the test is not vacuous
        assert not np.array_equal(want, np.argsort(v, kind="stable")) or n < 40


def test_pose_coordinates_definition():
    """pose = rotated float coordinates widened to double + (gridMin - mincoor + idx*spacing),
    idx*spacing a float product (src/TranRotaConfSearchNoMini.cu:473-487)."""
    w = synth.make_workload("c0_32", seed=6, n_conf=1, n_q=20)
    grid_min = (w.mid - w.length / np.float32(2)).astype(np.float32).astype(np.float64)
    for r in range(20):
        idx = np.array([r % 7, (3 * r) % 11, (5 * r) % 5], np.int32)
        got = poses.pose_coordinates(w.coor[0], w.quats[0, r], grid_min, w.spacing, idx)
        rot, mn, _ = O.rotate_bbox(w.coor[0], w.quats[0, r][None])
        step = (idx.astype(np.float32) * np.float32(w.spacing)).astype(np.float64)
        want = rot[0].astype(np.float64) + (grid_min - mn[0].astype(np.float64) + step)
        assert np.array_equal(got, want)


def test_export_top_files(tmp_path):
    """conformer_<c>_<rank>.pdb per pose and `file,conformer,rank,energy` lines, lowest first;
    a rotation without a window (+inf) is never exported."""
    w = synth.make_workload("c0_32", seed=7, n_conf=1, n_q=12)
    rng = np.random.default_rng(1)
    minE = rng.normal(size=12).astype(np.float32)
    minE[4] = np.inf
    idx = rng.integers(0, 8, size=(12, 3)).astype(np.int32)
    grid_min = (w.mid - w.length / np.float32(2)).astype(np.float64)
    path = os.path.join(tmp_path, "energy.txt")
    with open(path, "w") as ef:
        rows = poses.export_top(str(tmp_path), 3, w.coor[0], w.quats[0], minE, idx, grid_min,
                                w.spacing, 20, energy_file=ef)
    order = poses.sort_index(minE)
    assert [r[0] for r in rows] == [f"conformer_3_{k}.pdb" for k in range(11)]
    assert [r[2] for r in rows] == [float(minE[i]) for i in order[:11]]
    lines = open(path).read().splitlines()
    assert lines[0] == f"conformer_3_0.pdb,3,0,{float(minE[order[0]]):g}"
    pdb = open(os.path.join(tmp_path, "conformer_3_0.pdb")).read().splitlines()
    atoms = [ln for ln in pdb if ln.startswith("HETATM")]
    assert len(atoms) == w.coor.shape[1] and pdb[-1] == "END"
    xyz = poses.pose_coordinates(w.coor[0], w.quats[0, order[0]], grid_min, w.spacing, idx[order[0]])
    first = [float(atoms[0][30:38]), float(atoms[0][38:46]), float(atoms[0][46:54])]
    assert np.allclose(first, xyz[0], atol=5e-4)
