"""Serving (cdk_server_*): requests packed into shared waves give the same results as each
request searched alone, admission waits for arena space, and latency stats are reported."""
import numpy as np
import pytest

from cdocker_b200 import CDK_FORM_BF16X3, CDK_FORM_FP16X2, Receptor, synth
from cdocker_b200.serving import Server, make_requests, poisson_arrivals, run_load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def receptor_c1(grids_cache):
    w = synth.make_workload("c1_64", seed=4, n_conf=1, n_q=1, grids_cache=grids_cache)
    # all 8 vdW grids + elec: requests map atoms to any probe radius
    rec = Receptor(w.all_grids, w.spacing, max_atoms=128)
    yield w, rec
    rec.close()


def _reqs(w, n, seed, **kw):
    return make_requests(n, seed, w.spacing, w.length, synth.PROBE_RADII, **kw)


def test_mixed_requests_match_alone(receptor_c1):
    w, rec = receptor_c1
    reqs = _reqs(w, 4, seed=11, atoms=(10, 60), confs=(2, 6), rots=(100, 400))
    alone = []
    for r in reqs:
        slot = r["slot_full"]
        alone.append(rec.search(r["coor"], r["charge"], r["eps"], slot, r["quats"]))
    with Server(rec, arena_bytes=64 << 20, wave_rotations=256, max_atoms=128) as srv:
        tickets = [srv.submit(r["coor"], r["charge"], r["eps"], _full_slot(r), r["quats"])
                   for r in reqs]
        outs = [srv.poll(t, -1) for t in tickets]
        st = srv.stats()
    for (e, i, tm), (ae, ai) in zip(outs, alone):
        assert np.array_equal(e, ae) and np.array_equal(i, ai)
        assert tm[2] >= tm[1] >= 0
    assert st["completed"] == 4 and st["rotations"] == sum(r["rotations"] for r in reqs)
    # waves were shared across requests: fewer waves than requests' own wave counts
    assert st["waves"] < sum((r["rotations"] + 255) // 256 for r in reqs)


def test_admission_waits_for_arena(receptor_c1):
    w, rec = receptor_c1
    reqs = _reqs(w, 6, seed=12, atoms=(20, 40), confs=(4, 8), rots=(2000, 3000))
    # an arena that holds about two requests at a time
    with Server(rec, arena_bytes=160 << 10, wave_rotations=512, max_atoms=128) as srv:
        tickets = [srv.submit(r["coor"], r["charge"], r["eps"], _full_slot(r), r["quats"])
                   for r in reqs]
        outs = [srv.poll(t, -1) for t in tickets]
    for (e, i, tm), r in zip(outs, reqs):
        ae, ai = rec.search(r["coor"], r["charge"], r["eps"], _full_slot(r), r["quats"])
        assert np.array_equal(e, ae) and np.array_equal(i, ai)
    assert max(tm[0] for _, _, tm in outs) > 0.0  # somebody queued


def test_poisson_load_reports_latency(receptor_c1):
    w, rec = receptor_c1
    reqs = _reqs(w, 12, seed=13, atoms=(10, 80), confs=(10, 40), rots=(500, 1500))
    arr = poisson_arrivals(40.0, 10.0, seed=1)[:12]
    with Server(rec, arena_bytes=256 << 20, wave_rotations=1024, max_atoms=128) as srv:
        res = run_load(srv, reqs[: len(arr)], arr)
    assert res["requests"] == len(arr) and res["p99_ms"] >= res["p50_ms"] > 0


@pytest.mark.parametrize("form", [CDK_FORM_BF16X3, CDK_FORM_FP16X2])
def test_precision_form_server_runs_tensor_core_waves(grids_cache, form):
    """A precision-form receptor serves its waves on the streamed tensor-core x pass; each
    rotation's column of the contraction is independent of the other rotations in its tile, so
    shared waves reproduce each request searched alone."""
    w = synth.make_workload("c1_64", seed=4, n_conf=1, n_q=1, grids_cache=grids_cache)
    with Receptor(w.all_grids, w.spacing, max_atoms=96, form=form) as rec:
        reqs = _reqs(w, 4, seed=21, atoms=(10, 60), confs=(2, 6), rots=(100, 400))
        alone = [rec.search(r["coor"], r["charge"], r["eps"], _full_slot(r), r["quats"])
                 for r in reqs]
        with Server(rec, arena_bytes=64 << 20, wave_rotations=256, max_atoms=96) as srv:
            tickets = [srv.submit(r["coor"], r["charge"], r["eps"], _full_slot(r), r["quats"])
                       for r in reqs]
            outs = [srv.poll(t, -1) for t in tickets]
            st = srv.stats()
    assert st["tc_waves"] == st["waves"] > 0
    for (e, i, _), (ae, ai) in zip(outs, alone):
        assert np.array_equal(e, ae) and np.array_equal(i, ai)


def _full_slot(req):
    """Slots against the full 8-grid receptor: the atom's probe-radius class."""
    return req["slot_full"]
