"""Tensor-core forms (CDK_FORM_BF16X3, CDK_FORM_FP16X2): the x pass as a split-BF16 (or
split-FP16 operator x FP16 ligand) circulant contraction on the tensor cores. Bar: per-rotation
minimum energy within 1e-3 relative of the FP64 oracle (floor 1 kcal/mol), best translation
identical except at near-ties of that tolerance; FP64 re-score of the top poses."""
import numpy as np
import pytest

from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, Receptor, synth
from cdocker_b200.poses import rescore_top
from oracle import oracle as O
from tests.parity import check_search, rel_err

pytestmark = pytest.mark.gpu

TOL_TC = 1e-3


@pytest.mark.parametrize("form", [CDK_FORM_BF16X3, CDK_FORM_FP16X2])
@pytest.mark.parametrize("name,nconf,nq", [("c0_32", 1, 500), ("c1_64", 4, 25), ("c4_128", 1, 4)])
def test_tc_form_vs_fp64(name, nconf, nq, form, grids_cache):
    """Both tensor-core forms against FP64; the split-FP16 form runs its own kernel at 64^3 and
    the split-BF16 kernels at the other grid sizes."""
    w = synth.make_workload(name, seed=5, n_conf=nconf, n_q=nq, grids_cache=grids_cache)
    with Receptor(w.grids, w.spacing, form=form) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        if form == CDK_FORM_FP16X2 and name == "c1_64":
            assert rec.stats()["xpass_kind"] == "tcgen05_streamed_fp16"
    _, ridx, r64 = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot, w.quats,
                                   prec=1)
    qq = w.quats.reshape(-1, 4)
    st = check_search(minE, idx, r64, ridx,
                      lambda r: O.energy_map(w.grids, w.spacing, w.coor[r // nq], w.charge, w.eps,
                                             w.slot, qq[r]), rel_tol=TOL_TC)
    assert st["max_rel"] <= TOL_TC


def test_tc_and_fp32_forms_agree(c0):
    w = c0
    q = w.quats[:, :200]
    with Receptor(w.grids, w.spacing) as r32, Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3) as rtc:
        e32, i32 = r32.search(w.coor, w.charge, w.eps, w.slot, q)
        etc, itc = rtc.search(w.coor, w.charge, w.eps, w.slot, q)
    assert rel_err(etc, e32).max() <= TOL_TC
    assert np.mean(np.all(itc == i32, axis=1)) >= 0.98


def test_fp64_rescore_of_top_poses(c0):
    w = c0
    q = w.quats[:, :100]
    with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, q)
        top, e64 = rescore_top(rec, w.coor, w.charge, w.eps, w.slot, q, minE, idx, k=8,
                               batch=100)
    assert top.shape == (1, 8) and e64.shape == (1, 8)
    qq = q.reshape(-1, 4)
    for j, r in enumerate(top[0]):
        emap = O.energy_map(w.grids, w.spacing, w.coor[0], w.charge, w.eps, w.slot, qq[r])
        ref = emap[tuple(idx[r])]
        assert abs(e64[0, j] - ref) <= 1e-7 * max(1.0, abs(ref))


@pytest.mark.parametrize("wave", [0, 200])
def test_tensor_core_variants_agree(grids_cache, wave):
    """tcgen05 with streamed operands (default at 64^3: both operands in shared memory; or the
    ligand in tensor memory), tcgen05 with in-kernel operand builds and mma.sync apply the
    same split-BF16 operator; ragged waves (200 rotations: a partial 128-rotation tile)
    included."""
    w = synth.make_workload("c1_64", seed=8, n_conf=2, n_q=150, grids_cache=grids_cache)
    out = {}
    for name, kw in [("streamed", {}), ("streamed_tmem", {"tc_tmem_ligand": True}),
                     ("build", {"tc_build": True}), ("mma_sync", {"tc_mma_sync": True})]:
        with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3, wave_rotations=wave, **kw) as r:
            out[name] = r.search(w.coor, w.charge, w.eps, w.slot, w.quats)
            kind = r.stats()["xpass_kind"]
        assert kind == {"streamed": "tcgen05_streamed", "streamed_tmem": "tcgen05_streamed_tmem",
                        "build": "tcgen05_build", "mma_sync": "mma_sync"}[name]
    es, is_ = out["streamed"]
    # the two streamed kernels run the same MMAs in the same order: bit-identical
    assert np.array_equal(es, out["streamed_tmem"][0]) and np.array_equal(is_, out["streamed_tmem"][1])
    for other in ("build", "mma_sync"):
        eo, io = out[other]
        assert rel_err(es, eo).max() <= 1e-5
        assert np.mean(np.all(is_ == io, axis=1)) >= 0.99


def test_streamed_falls_back_for_large_ligands(grids_cache):
    """Ligands above 96 atoms take the FFT plane path, which writes no split rows: the context
    picks the in-kernel-build tcgen05 x pass for them and stays correct."""
    w = synth.make_workload("c1_64", seed=9, n_conf=1, n_q=20, grids_cache=grids_cache,
                            n_atoms=110)
    with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3) as rtc, \
            Receptor(w.grids, w.spacing) as r32:
        etc, itc = rtc.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        assert rtc.stats()["xpass_kind"] != "tcgen05_streamed"
        e32, i32 = r32.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    assert rel_err(etc, e32).max() <= TOL_TC


@pytest.mark.parametrize("form", [CDK_FORM_BF16X3, CDK_FORM_FP16X2])
@pytest.mark.parametrize("n_atoms,radius,n_q,wave", [(6, 1.2, 40, 0),    # box 7 planes: one K-step, 6-stage ring
                                                     (60, 6.8, 12, 0),   # box 30 planes: 4-column shape
                                                     (40, 4.7, 37, 29)])  # ragged waves (not multiples of 8)
def test_streamed_shapes_vs_fp64(grids_cache, n_atoms, radius, n_q, wave, form):
    """The streamed tensor-core x pass of both forms across ligand boxes (1 to 4 K-steps, both
    CTA shapes) and ragged waves, against the FP64 oracle."""
    w = synth.make_workload("c1_64", seed=31, n_conf=1, n_q=n_q, grids_cache=grids_cache,
                            n_atoms=n_atoms, ligand_radius=radius)
    with Receptor(w.grids, w.spacing, form=form, wave_rotations=wave) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        assert rec.stats()["xpass_kind"] == ("tcgen05_streamed_fp16" if form == CDK_FORM_FP16X2
                                             else "tcgen05_streamed")
    _, ridx, r64 = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot, w.quats,
                                   prec=1)
    qq = w.quats.reshape(-1, 4)
    st = check_search(minE, idx, r64, ridx,
                      lambda r: O.energy_map(w.grids, w.spacing, w.coor[0], w.charge, w.eps,
                                             w.slot, qq[r]), rel_tol=TOL_TC)
    assert st["max_rel"] <= TOL_TC


def test_fp16_form_rejects_ligands_outside_its_range(grids_cache):
    """The split-FP16 form bounds every scaled ligand value by the channel's sum of |charge| or
    sqrt-epsilon (prep kernel); ligands whose bound leaves the FP16 range are refused with
    CDK_ERR_UNSUPPORTED instead of overflowing, while the split-BF16 form searches them."""
    from cdocker_b200 import _lib as L
    w = synth.make_workload("c1_64", seed=14, n_conf=1, n_q=8, grids_cache=grids_cache)
    big = (w.charge * 1e4).astype(np.float32)
    with Receptor(w.grids, w.spacing, form=CDK_FORM_FP16X2) as rec:
        with pytest.raises(L.CdkError) as e:
            rec.search(w.coor, big, w.eps, w.slot, w.quats)
        assert e.value.code == L.CDK_ERR_UNSUPPORTED
        # the context stays usable for ligands inside the range
        minE, _ = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        assert np.all(np.isfinite(minE))
    with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3) as rec:
        minE, _ = rec.search(w.coor, big, w.eps, w.slot, w.quats)
        assert np.all(np.isfinite(minE))
