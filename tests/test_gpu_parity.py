"""GPU parity of the FP32 search against the oracle, through the C-ABI (cdk_search)."""
import numpy as np
import pytest

from cdocker_b200 import Receptor, synth, fill_ligand_grid
from oracle import oracle as O
from tests.parity import check_search

pytestmark = pytest.mark.gpu


def _emap(w, conf_of, quat_of):
    def f(r):
        return O.energy_map(w.grids, w.spacing, w.coor[conf_of(r)], w.charge, w.eps, w.slot,
                            quat_of(r))
    return f


def test_c0_full_vs_fp64_direct(c0):
    """Config 0 (32^3, K=9, 24 atoms, 500 rotations): every rotation vs the FP64 oracle."""
    w = c0
    with Receptor(w.grids, w.spacing) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    _, ridx, r64 = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot, w.quats,
                                   prec=1)
    q = w.quats.reshape(-1, 4)
    st = check_search(minE, idx, r64, ridx, _emap(w, lambda r: 0, lambda r: q[r]))
    assert st["n"] == 500


def test_c0_vs_fp32_cpunaive(c0):
    """Same inputs vs cpuNaive's float accumulation (src/cpuNaive.cpp:194-216)."""
    w = c0
    q = w.quats[:, :100]
    with Receptor(w.grids, w.spacing) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, q)
    r32, ridx, _ = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot, q, prec=0)
    qq = q.reshape(-1, 4)
    check_search(minE, idx, r32, ridx, _emap(w, lambda r: 0, lambda r: qq[r]))


@pytest.mark.parametrize("name,nconf,nq", [("c1_64", 3, 16), ("c3_96", 1, 6), ("c4_128", 1, 4)])
def test_larger_grids_vs_fp64(name, nconf, nq, grids_cache):
    w = synth.make_workload(name, seed=1, n_conf=nconf, n_q=nq, grids_cache=grids_cache)
    with Receptor(w.grids, w.spacing) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    _, ridx, r64 = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot, w.quats,
                                   prec=1)
    qq = w.quats.reshape(-1, 4)
    check_search(minE, idx, r64, ridx, _emap(w, lambda r: r // nq, lambda r: qq[r]))


def test_waves_and_tiles_agree(c0):
    """Different wave sizes and column tiles give identical results (work split only)."""
    w = c0
    q = w.quats[:, :64]
    outs = []
    for wave, ct in [(0, 0), (7, 8), (64, 8), (13, 16)]:
        with Receptor(w.grids, w.spacing, wave_rotations=wave, col_tile=ct) as rec:
            outs.append(rec.search(w.coor, w.charge, w.eps, w.slot, q))
    for m, i in outs[1:]:
        # the channel sum runs in the same order whatever the split: bit-identical
        np.testing.assert_array_equal(i, outs[0][1])
        np.testing.assert_array_equal(m, outs[0][0])


def test_fill_bitexact_vs_reference(c0):
    """cdk_fill_ligand_grid == the reference's FillLigandGrid, bit for bit."""
    w = c0
    rot, mn, ln = O.rotate_bbox(w.coor[0], w.quats[0, :4])
    gpu = fill_ligand_grid(rot, mn, w.charge, w.eps, w.slot, w.K - 1, (w.n,) * 3, w.spacing)
    if O.ref_available():
        R = O.ref()
        ref = np.zeros_like(gpu)
        R.ref_fill_ligand_grid(4, rot.shape[1], O._pf(rot), O._pf(mn), O._pf(O._f32(w.charge)),
                               O._pf(O._f32(w.eps)), O._pf(O._f32(w.radii)), 8,
                               O._pf(O._f32(w.grid_radii)), w.n, w.n, w.n, w.spacing, O._pf(ref))
    else:
        ref = O.fill_ligand_grid(rot, mn, w.charge, w.eps, w.slot, w.K - 1, (w.n,) * 3, w.spacing)
    assert np.array_equal(gpu.view(np.uint32), ref.view(np.uint32))


def test_empty_window_and_zero_rotations(c0):
    """A ligand longer than the grid leaves the window empty: +inf and -1 (the reference
    leaves INFINITY and unset indices); nQ = 0 is a no-op."""
    w = c0
    big = w.coor[0] * 4.0  # ~32 A across on a 15.5 A grid
    with Receptor(w.grids, w.spacing) as rec:
        minE, idx = rec.search(big, w.charge, w.eps, w.slot, w.quats[:, :5])
        assert np.all(np.isinf(minE)) and np.all(idx == -1)
        m0, i0 = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats[:, :0])
        assert m0.size == 0


def test_invalid_slot_rejected(c0):
    from cdocker_b200 import CdkError
    w = c0
    bad = w.slot.copy()
    bad[0] = w.K - 1  # the elec channel is not a vdW slot
    with Receptor(w.grids, w.spacing) as rec:
        with pytest.raises(CdkError):
            rec.search(w.coor, w.charge, w.eps, bad, w.quats[:, :3])


def test_rescore_fp64_matches_oracle_map(c0):
    w = c0
    q = w.quats[0, :8]
    with Receptor(w.grids, w.spacing) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, q[None])
        e64 = rec.rescore_fp64(w.coor, w.charge, w.eps, w.slot, np.zeros(8, np.int32), q, idx)
    for r in range(8):
        emap = O.energy_map(w.grids, w.spacing, w.coor[0], w.charge, w.eps, w.slot, q[r])
        ref = emap[tuple(idx[r])]
        # the oracle map sums the float-rounded ligand grid; the re-score keeps the trilinear
        # weights in double, so the two differ by float rounding of the weights (~1e-8)
        assert abs(e64[r] - ref) <= 1e-7 * max(1.0, abs(ref))
        assert abs(e64[r] - minE[r]) <= 1e-4 * max(1.0, abs(ref))


def test_direct_planes_match_fft_planes(grids_cache):
    """The direct separable plane spectrum and the spread + radix-FFT planes agree."""
    w = synth.make_workload("c1_64", seed=6, n_conf=2, n_q=32, grids_cache=grids_cache)
    with Receptor(w.grids, w.spacing) as rd, Receptor(w.grids, w.spacing, fft_planes=True) as rf:
        e1, i1 = rd.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        e2, i2 = rf.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    from tests.parity import rel_err
    assert rel_err(e1, e2).max() <= 1e-5
    assert np.mean(np.all(i1 == i2, axis=1)) >= 0.98


def _device_search(rec, w, torch, reps):
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev)
         for k, v in (("coor", w.coor), ("charge", w.charge), ("eps", w.eps), ("slot", w.slot),
                      ("quats", w.quats))}
    out = []
    for _ in range(reps):
        e = torch.empty(w.n_rot, device=dev)
        i = torch.empty(w.n_rot, 3, dtype=torch.int32, device=dev)
        # same output buffers every time for the graph key: reuse the first pair
        if out:
            e, i = out[0][2], out[0][3]
        rec.search_device(w.coor.shape[1], w.coor.shape[0], t["coor"].data_ptr(),
                          t["charge"].data_ptr(), t["eps"].data_ptr(), t["slot"].data_ptr(),
                          w.quats.shape[1], t["quats"].data_ptr(), e.data_ptr(), i.data_ptr(), 0)
        torch.cuda.synchronize()
        out.append((e.cpu().numpy().copy(), i.cpu().numpy().copy(), e, i))
    return out


def test_graph_replay_matches(c0):
    import torch
    w = c0
    with Receptor(w.grids, w.spacing) as plain:
        ref = _device_search(plain, w, torch, 1)[0]
    with Receptor(w.grids, w.spacing, use_graphs=1, wave_rotations=100) as rec:
        outs = _device_search(rec, w, torch, 4)
        assert rec.stats()["graph_state"] == 2
    for e, i, _, _ in outs:
        np.testing.assert_array_equal(e, ref[0])
        np.testing.assert_array_equal(i, ref[1])


def test_autotune_same_results(c0):
    w = c0
    q = w.quats[:, :200]
    with Receptor(w.grids, w.spacing) as plain:
        e0, i0 = plain.search(w.coor, w.charge, w.eps, w.slot, q)
    with Receptor(w.grids, w.spacing, autotune=True) as rec:
        e1, i1 = rec.search(w.coor, w.charge, w.eps, w.slot, q)
        st = rec.stats()
    np.testing.assert_array_equal(e0, e1)
    np.testing.assert_array_equal(i0, i1)
    assert st["col_tile"] in (8, 16) and st["rotations_per_cta"] in (16, 32, 64)


@pytest.mark.parametrize("form", [0, 2])
@pytest.mark.parametrize("name,nq", [("c0_32", 60), ("c1_64", 120), ("c3_96", 24), ("c4_128", 12)])
def test_yz_octet_kernel_matches_block_stages(grids_cache, form, name, nq):
    """The inverse (y,z) transform runs warp-local line transforms (octets of lanes); the
    block-stage kernel runs the same radix stages, twiddles and packing, so the minima and
    translations agree (bit for bit where the compiler keeps the same operation order)."""
    w = synth.make_workload(name, seed=3, n_conf=2, n_q=nq, grids_cache=grids_cache)
    out = []
    for kw in ({"yz_octets": True}, {"yz_block_stages": True}):
        with Receptor(w.grids, w.spacing, form=form, **kw) as rec:
            out.append(rec.search(w.coor, w.charge, w.eps, w.slot, w.quats))
    (e0, i0), (e1, i1) = out
    assert np.abs(e0.astype(np.float64) - e1).max() <= 1e-6 * np.abs(e1).max()
    assert np.mean(np.all(i0 == i1, axis=1)) >= 0.99


def test_graph_replay_tensor_core_form(grids_cache):
    """The split-FP16 search (rotation grouping, tile plans, the Hankel x pass, the FP64
    near-tie break and the per-wave top-pose re-score) captured into one CUDA graph and replayed:
    the same results as the plain search every time."""
    import torch
    w = synth.make_workload("c1_64", seed=12, n_conf=2, n_q=150, grids_cache=grids_cache)
    with Receptor(w.grids, w.spacing, form=2) as plain:
        ref = _device_search(plain, w, torch, 1)[0]
    with Receptor(w.grids, w.spacing, form=2, use_graphs=1, wave_rotations=128,
                  profile=True) as rec:
        outs = _device_search(rec, w, torch, 4)
        st = rec.stats()
        assert st["graph_state"] == 2
        # the per-kernel events are recorded inside the graph too
        assert st["kernel_ms"]["xpass"] > 0 and st["kernel_ms"]["yz_inv_argmin"] > 0
        outs += _device_search(rec, w, torch, 1)  # and leave no error behind
    for e, i, _, _ in outs:
        np.testing.assert_array_equal(e, ref[0])
        np.testing.assert_array_equal(i, ref[1])


@pytest.mark.parametrize("form", [1, 2])
def test_autotune_tensor_core_same_results(grids_cache, form):
    """The autotuner times the Hankel x pass under one and two columns per CTA and several ring
    depths on the first wave and keeps the fastest; every candidate computes the same numbers."""
    w = synth.make_workload("c1_64", seed=13, n_conf=2, n_q=200, grids_cache=grids_cache)
    with Receptor(w.grids, w.spacing, form=form, tc_hankel=True) as plain:
        e0, i0 = plain.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    with Receptor(w.grids, w.spacing, form=form, autotune=True, tc_hankel=True) as rec:
        e1, i1 = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
        st = rec.stats()
        e2, i2 = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    np.testing.assert_array_equal(e0, e1)
    np.testing.assert_array_equal(i0, i1)
    np.testing.assert_array_equal(e1, e2)
    assert st["xpass_kind"].startswith("tcgen05_hankel") and st["col_tile"] in (1, 2)
