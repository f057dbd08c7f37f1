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


HANKEL = {CDK_FORM_BF16X3: "tcgen05_hankel", CDK_FORM_FP16X2: "tcgen05_hankel_fp16"}


def auto_kind(n, form):
    """The automatic tensor-core x pass: the Hankel kernel over tiled ligand rows at every n and
    in both forms (streamed operator tiles only on request)."""
    return HANKEL[form]


@pytest.mark.parametrize("form", [CDK_FORM_BF16X3, CDK_FORM_FP16X2])
@pytest.mark.parametrize("name,nconf,nq", [("c0_32", 1, 500), ("c1_64", 4, 25), ("c3_96", 2, 32),
                                           ("c4_128", 2, 32)])
def test_tc_form_vs_fp64(name, nconf, nq, form, grids_cache):
    """Both tensor-core forms against FP64 at every grid size, every rotation checked (64 at
    96^3 and at 128^3), with the automatic x pass and, at 64^3, the Hankel kernel as well."""
    w = synth.make_workload(name, seed=5, n_conf=nconf, n_q=nq, grids_cache=grids_cache)
    for hankel in ((False, True) if w.n == 64 else (False,)):
        with Receptor(w.grids, w.spacing, form=form, tc_hankel=hankel) as rec:
            minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
            assert rec.stats()["xpass_kind"] == (HANKEL[form] if hankel else auto_kind(w.n, form))
        _check_fp64(w, nq, minE, idx)


def _check_fp64(w, nq, minE, idx):
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
    """tcgen05 with the resident Hankel operator (the default; one and two columns per CTA),
    tcgen05 with streamed operator tiles, tcgen05 with in-kernel operand builds and mma.sync
    apply the same split-BF16 operator; ragged waves (200 rotations: a partial 128-rotation
    tile) included."""
    w = synth.make_workload("c1_64", seed=8, n_conf=2, n_q=150, grids_cache=grids_cache)
    out = {}
    kinds = {"hankel": "tcgen05_hankel", "hankel_1col": "tcgen05_hankel",
             "hankel_2col": "tcgen05_hankel", "stream_tiles": "tcgen05_streamed",
             "build": "tcgen05_build", "mma_sync": "mma_sync"}
    for name, kw in [("hankel", {"tc_hankel": True}), ("hankel_1col", {"tc_hankel": True, "tc_cols": 1}),
                     ("hankel_2col", {"tc_hankel": True, "tc_cols": 2}),
                     ("stream_tiles", {"tc_stream_tiles": True}), ("build", {"tc_build": True}),
                     ("mma_sync", {"tc_mma_sync": True})]:
        with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3, wave_rotations=wave, **kw) as r:
            out[name] = r.search(w.coor, w.charge, w.eps, w.slot, w.quats)
            st = r.stats()
        assert st["xpass_kind"] == kinds[name]
        if name.startswith("hankel_"):
            assert st["col_tile"] == int(name[-4])
    es, is_ = out["hankel"]
    # one or two columns per CTA: the same MMAs per column, bit-identical
    for v in ("hankel_1col", "hankel_2col"):
        assert np.array_equal(es, out[v][0]) and np.array_equal(is_, out[v][1])
    for other in ("stream_tiles", "build", "mma_sync"):
        eo, io = out[other]
        assert rel_err(es, eo).max() <= 1e-5
        assert np.mean(np.all(is_ == io, axis=1)) >= 0.99


@pytest.mark.parametrize("form", [CDK_FORM_FP16X2, CDK_FORM_BF16X3])
@pytest.mark.parametrize("name,n_conf,n_q,wave,cols", [("c1_64", 2, 150, 200, 1),
                                                       ("c1_64", 3, 111, 0, 2),
                                                       ("c3_96", 1, 130, 0, 1),
                                                       ("c4_128", 1, 70, 45, 1)])
def test_tiled_rows_match_thread_copies(grids_cache, form, name, n_conf, n_q, wave, cols):
    """The Hankel x pass loads its ligand rows either as 128-rotation row sets that the plane
    kernel writes column by column (one tensor copy per K-step and column gathers the 128 rows
    and applies the tensor cores' 32- or 64-byte swizzle; the default) or rotation by rotation
    with per-thread copies from the untiled rows. The MMAs see the same operands either way, so
    results are bit-identical: ragged waves (partial tiles), one and two columns per CTA, chunks
    of a tile's plan that a rotation does not touch (zeros written by the plane kernel,
    zero-filled by the copies), 64^3, 96^3 and 128^3."""
    w = synth.make_workload(name, seed=17, n_conf=n_conf, n_q=n_q, grids_cache=grids_cache)
    out = {}
    for thread_copies in (False, True):
        with Receptor(w.grids, w.spacing, form=form, wave_rotations=wave, tc_hankel=True,
                      tc_cols=cols, tc_thread_copies=thread_copies,
                      tc_tiled_rows=not thread_copies) as rec:
            out[thread_copies] = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
            st = rec.stats()
        assert st["xpass_kind"] == HANKEL[form] and st["col_tile"] == cols
    (et, it), (ec, ic) = out[False], out[True]
    assert np.isfinite(et).all()
    assert np.array_equal(et.view(np.uint32), ec.view(np.uint32))
    assert np.array_equal(it, ic)


def test_streamed_falls_back_for_large_ligands(grids_cache):
    """Ligands above 96 atoms take the FFT plane path, which writes no split rows: a split-BF16
    context picks the in-kernel-build tcgen05 x pass for them and stays correct; a split-FP16
    context refuses them with CDK_ERR_UNSUPPORTED instead of switching form silently."""
    w = synth.make_workload("c1_64", seed=9, n_conf=1, n_q=20, grids_cache=grids_cache,
                            n_atoms=110)
    with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3) as rtc, \
            Receptor(w.grids, w.spacing) as r32:
        etc, itc = rtc.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        assert rtc.stats()["xpass_kind"] == "tcgen05_build"
        e32, i32 = r32.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    assert rel_err(etc, e32).max() <= TOL_TC
    from cdocker_b200 import _lib as L
    with Receptor(w.grids, w.spacing, form=CDK_FORM_FP16X2) as r16:
        with pytest.raises(L.CdkError) as e:
            r16.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        assert e.value.code == L.CDK_ERR_UNSUPPORTED


@pytest.mark.parametrize("form", [CDK_FORM_BF16X3, CDK_FORM_FP16X2])
@pytest.mark.parametrize("hankel", [False, True])
@pytest.mark.parametrize("name,n_atoms,radius,n_q,wave",
                         [("c1_64", 6, 1.2, 40, 0),     # box 7 planes: one K-step
                          ("c1_64", 60, 6.8, 12, 0),    # box 30 planes: four K-steps
                          ("c1_64", 40, 4.7, 37, 29),   # ragged waves (not multiples of 8)
                          ("c4_128", 6, 1.2, 20, 0),    # 128^3: one K-step, windows near n
                          ("c4_128", 60, 6.8, 12, 5),   # 128^3: four K-steps, 5-rotation waves
                          ("c3_96", 30, 4.4, 21, 0)])   # 96^3
def test_streamed_shapes_vs_fp64(grids_cache, name, n_atoms, radius, n_q, wave, form, hankel):
    """The tensor-core x passes of both forms across ligand boxes (1 to 4 K-steps), grid sizes
    and ragged waves, against the FP64 oracle (the automatic choice, and the Hankel kernel)."""
    w = synth.make_workload(name, seed=31, n_conf=1, n_q=n_q, grids_cache=grids_cache,
                            n_atoms=n_atoms, ligand_radius=radius)
    if hankel and w.n != 64:
        pytest.skip("the automatic choice is the Hankel kernel at this size")
    with Receptor(w.grids, w.spacing, form=form, wave_rotations=wave, tc_hankel=hankel) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        assert rec.stats()["xpass_kind"] == (HANKEL[form] if hankel else auto_kind(w.n, form))
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


@pytest.mark.parametrize("form", [CDK_FORM_FP16X2, CDK_FORM_BF16X3])
def test_fp64_near_tie_break(grids_cache, form):
    """The precision forms re-score a rotation's two best translations in FP64 when they lie
    within the near-tie tolerance and keep the lower: against the same search without the tie
    break, every changed translation is at least as low in FP64, and agreement with the FP64
    oracle's argmin does not drop."""
    w = synth.make_workload("c1_64", seed=41, n_conf=3, n_q=200, grids_cache=grids_cache)
    res = {}
    for tb in (True, False):
        with Receptor(w.grids, w.spacing, form=form, tie_break=tb) as rec:
            e, i = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
            st = rec.stats()
            res[tb] = (e, i, st)
    (e1, i1, st1), (e0, i0, st0) = res[True], res[False]
    assert st1["near_ties_rescored"] >= st1["near_ties_changed"] >= 0
    assert st0["near_ties_rescored"] == 0
    changed = np.nonzero(np.any(i1 != i0, axis=1))[0]
    assert changed.size == st1["near_ties_changed"]
    qq = w.quats.reshape(-1, 4)
    if changed.size:
        with Receptor(w.grids, w.spacing, form=form) as rec:
            rc = (changed // 200).astype(np.int32)
            f1 = rec.rescore_fp64(w.coor, w.charge, w.eps, w.slot, rc, qq[changed], i1[changed])
            f0 = rec.rescore_fp64(w.coor, w.charge, w.eps, w.slot, rc, qq[changed], i0[changed])
        assert np.all(f1 <= f0)
    sel = np.arange(0, 600, 5)
    _, ridx, r64 = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot, w.quats,
                                   prec=1)
    agree1 = np.mean(np.all(i1[sel] == ridx[sel], axis=1))
    agree0 = np.mean(np.all(i0[sel] == ridx[sel], axis=1))
    assert agree1 >= agree0
    assert rel_err(e1, r64).max() <= TOL_TC


def test_top_poses_rescored_per_wave(grids_cache):
    """Per wave, the k lowest-energy poses with their FP64 re-score (cdk_ctx_top_poses): the
    rotations are the k smallest minima of their wave, the FP64 energies equal the oracle's
    double energy map at those poses."""
    w = synth.make_workload("c1_64", seed=42, n_conf=1, n_q=250, grids_cache=grids_cache)
    k = 8
    # with the grouping sort the waves hold rotations from anywhere in the list: every wave's
    # k lowest still include each of the search's k lowest that it holds
    with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3, wave_rotations=100, top_k=k) as rec:
        e, i = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        rot, te, tidx, e64 = rec.top_poses()
    assert rot.shape[0] == 3 * k and len(set(rot.tolist())) == 3 * k
    assert set(np.argsort(e, kind="stable")[:k].tolist()) <= set(rot.tolist())
    assert np.array_equal(te, e[rot]) and np.array_equal(tidx, i[rot])
    # in the given order (no grouping) wave w holds rotations [100 w, 100 w + 100)
    with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3, wave_rotations=100, top_k=k,
                  group_rotations=False) as rec:
        e, i = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        rot, te, tidx, e64 = rec.top_poses()
        st = rec.stats()
    assert st["waves"] == 3 and rot.shape[0] == 3 * k
    qq = w.quats.reshape(-1, 4)
    for wv in range(3):
        lo, hi = 100 * wv, min(250, 100 * (wv + 1))
        want = np.sort(e[lo:hi])[:k]
        got = rot[wv * k:(wv + 1) * k]
        assert np.all((got >= lo) & (got < hi))
        assert np.array_equal(np.sort(e[got]), want)
        assert np.array_equal(te[wv * k:(wv + 1) * k], e[got])
        assert np.array_equal(tidx[wv * k:(wv + 1) * k], i[got])
    for j in range(0, 3 * k, 5):
        r = int(rot[j])
        emap = O.energy_map(w.grids, w.spacing, w.coor[0], w.charge, w.eps, w.slot, qq[r])
        ref = emap[tuple(tidx[j])]
        # the oracle's map sums FillLigandGrid's float-rounded cells; the re-score sums the
        # exact trilinear weights in double: they agree to the float grid's rounding
        assert abs(e64[j] - ref) <= 1e-7 * max(1.0, abs(ref))
