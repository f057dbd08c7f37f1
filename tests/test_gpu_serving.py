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
    """A precision-form receptor serves its waves on the tensor-core x pass; each rotation's row
    of the contraction is independent of the other rotations in its tile, so shared waves
    reproduce each request searched alone."""
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


def _poll_status(srv, ticket):
    """(status code, minE, idx) of a finished request, whatever its status."""
    import ctypes as C

    from cdocker_b200 import _lib as L
    e = np.empty(ticket.n_rot, np.float32)
    i = np.empty((ticket.n_rot, 3), np.int32)
    tm = np.zeros(3, np.float64)
    rc = L.lib().cdk_server_poll(srv._h, C.c_uint64(ticket.id), -1,
                                 e.ctypes.data_as(C.POINTER(C.c_float)),
                                 i.ctypes.data_as(C.POINTER(C.c_int)),
                                 tm.ctypes.data_as(C.POINTER(C.c_double)))
    return rc, e, i


def test_fp16_range_failure_is_attributed_to_its_request(grids_cache):
    """Split-FP16 server: a request whose charges (x 1e4) would leave the FP16 range fails with
    CDK_ERR_UNSUPPORTED, a normal request submitted right after it -- in the same waves --
    succeeds with the results it gets alone, and the next request after both succeeds too
    (the status words are per wave, not sticky)."""
    from cdocker_b200 import _lib as L
    w = synth.make_workload("c1_64", seed=4, n_conf=1, n_q=1, grids_cache=grids_cache)
    with Receptor(w.all_grids, w.spacing, max_atoms=96, form=CDK_FORM_FP16X2) as rec:
        bad, good, later = _reqs(w, 3, seed=31, atoms=(20, 40), confs=(2, 4), rots=(100, 200))
        alone_good = rec.search(good["coor"], good["charge"], good["eps"], _full_slot(good),
                                good["quats"])
        alone_later = rec.search(later["coor"], later["charge"], later["eps"], _full_slot(later),
                                 later["quats"])
        with Server(rec, arena_bytes=64 << 20, wave_rotations=1024, max_atoms=96) as srv:
            tb = srv.submit(bad["coor"], bad["charge"] * 1e4, bad["eps"], _full_slot(bad),
                            bad["quats"])
            tg = srv.submit(good["coor"], good["charge"], good["eps"], _full_slot(good),
                            good["quats"])
            rc_b, eb, ib = _poll_status(srv, tb)
            rc_g, eg, ig = _poll_status(srv, tg)
            tl = srv.submit(later["coor"], later["charge"], later["eps"], _full_slot(later),
                            later["quats"])
            rc_l, el, il = _poll_status(srv, tl)
    assert rc_b == L.CDK_ERR_UNSUPPORTED
    assert np.all(ib[:, 0] == -3) and np.all(np.isnan(eb))
    assert rc_g == L.CDK_OK and rc_l == L.CDK_OK
    assert np.array_equal(eg, alone_good[0]) and np.array_equal(ig, alone_good[1])
    assert np.array_equal(el, alone_later[0]) and np.array_equal(il, alone_later[1])


def test_overflow_is_attributed_to_its_request(receptor_c1):
    """FP32 server: one rotation of a request has a non-unit quaternion (norm^2 = 2) whose
    stretched ligand leaves the planned box of every request in the wave: that request fails with CDK_ERR_OVERFLOW (the
    rotation reads NaN / -2, the others their normal results), the request sharing its wave
    succeeds, and a later request succeeds as well."""
    from cdocker_b200 import _lib as L
    w, rec = receptor_c1
    a, b, c = _reqs(w, 3, seed=32, atoms=(20, 30), confs=(2, 3), rots=(60, 120))
    qa = a["quats"].copy()
    qa[0, 3] = np.array([np.sqrt(2.0), 0.0, 0.0, 0.0], np.float32)
    alone_a = rec.search(a["coor"], a["charge"], a["eps"], _full_slot(a), a["quats"])
    alone_b = rec.search(b["coor"], b["charge"], b["eps"], _full_slot(b), b["quats"])
    with Server(rec, arena_bytes=64 << 20, wave_rotations=1024, max_atoms=128) as srv:
        ta = srv.submit(a["coor"], a["charge"], a["eps"], _full_slot(a), qa)
        tb = srv.submit(b["coor"], b["charge"], b["eps"], _full_slot(b), b["quats"])
        rc_a, ea, ia = _poll_status(srv, ta)
        rc_b, eb, ib = _poll_status(srv, tb)
        tc = srv.submit(c["coor"], c["charge"], c["eps"], _full_slot(c), c["quats"])
        rc_c, _, _ = _poll_status(srv, tc)
    assert rc_a == L.CDK_ERR_OVERFLOW and rc_b == L.CDK_OK and rc_c == L.CDK_OK
    assert np.isnan(ea[3]) and np.all(ia[3] == -2)
    keep = np.arange(ea.shape[0]) != 3
    assert np.array_equal(ea[keep], alone_a[0][keep]) and np.array_equal(ia[keep], alone_a[1][keep])
    assert np.array_equal(eb, alone_b[0]) and np.array_equal(ib, alone_b[1])


def test_injected_fault_fails_only_its_wave(receptor_c1):
    """Failure detection without a GPU fault: the host sets the device-wait fault word of the
    server's first wave after its kernels (the word a bounded tcgen05 wait sets when it gives
    up). The request in that wave fails with CDK_ERR_CUDA; the next request, in a later wave,
    succeeds with the results it gets alone."""
    from cdocker_b200 import _lib as L
    w, rec = receptor_c1
    a, b = _reqs(w, 2, seed=33, atoms=(20, 30), confs=(2, 3), rots=(60, 120))
    alone_b = rec.search(b["coor"], b["charge"], b["eps"], _full_slot(b), b["quats"])
    with Server(rec, arena_bytes=64 << 20, wave_rotations=1024, max_atoms=128,
                inject_fault_wave=0) as srv:
        ta = srv.submit(a["coor"], a["charge"], a["eps"], _full_slot(a), a["quats"])
        rc_a, _, _ = _poll_status(srv, ta)
        msg = L.last_error()
        tb = srv.submit(b["coor"], b["charge"], b["eps"], _full_slot(b), b["quats"])
        rc_b, eb, ib = _poll_status(srv, tb)
    assert rc_a == L.CDK_ERR_CUDA and "gave up" in msg
    assert rc_b == L.CDK_OK
    assert np.array_equal(eb, alone_b[0]) and np.array_equal(ib, alone_b[1])
