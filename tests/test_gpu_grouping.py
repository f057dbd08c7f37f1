"""Rotation grouping of the tensor-core x pass: the search sorts its rotation list so
that rotations whose channels reach the same 8-plane chunks of the ligand box share 128-rotation
tiles. Chunks a rotation does not touch add exact zeros, so grouping must change no result --
checked bit for bit against the ungrouped order -- while the tiles issue fewer K-steps."""
import numpy as np
import pytest

from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, Receptor, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", [CDK_FORM_FP16X2, CDK_FORM_BF16X3])
def test_grouping_changes_no_result(form, grids_cache):
    # 2,400 rotations: three 1,024-rotation segments of the counting sort, several waves
    w = synth.make_workload("c1_64", seed=11, n_conf=6, n_q=400, grids_cache=grids_cache)
    out = {}
    for grouped in (True, False):
        with Receptor(w.grids, w.spacing, form=form, wave_rotations=700,
                      group_rotations=grouped) as rec:
            e, i = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
            st = rec.stats()
        assert st["xpass_kind"].startswith("tcgen05_")
        out[grouped] = (e, i, st["tensor_steps"])
    (eg, ig, sg), (eu, iu, su) = out[True], out[False]
    assert np.array_equal(eg.view(np.uint32), eu.view(np.uint32))
    assert np.array_equal(ig, iu)
    assert np.isfinite(eg).all()
    # the point of the sort: fewer tensor-core K-steps for the same rotations
    assert sg < su


def test_grouping_with_a_ragged_tail(grids_cache):
    """A rotation count that is neither a multiple of the tile nor of the sort segment, and a
    quaternion set with duplicates (equal keys across segments keep their order)."""
    w = synth.make_workload("c1_64", seed=12, n_conf=3, n_q=389, grids_cache=grids_cache)
    q = w.quats.copy()
    q[:, 100:150] = q[:, 0:50]
    res = []
    for grouped in (True, False):
        with Receptor(w.grids, w.spacing, form=CDK_FORM_FP16X2, group_rotations=grouped) as rec:
            res.append(rec.search(w.coor, w.charge, w.eps, w.slot, q))
    assert np.array_equal(res[0][0].view(np.uint32), res[1][0].view(np.uint32))
    assert np.array_equal(res[0][1], res[1][1])
