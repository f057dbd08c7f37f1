"""cdk_search_device_noalloc: the search entry point for callers that cannot allocate.

Callers that run the search from a real-time loop (cudaMalloc and cudaFree can synchronise
the whole device), or that own all device memory through a pool, cannot let the library call
cudaMalloc mid-search. This entry
point takes the same device buffers as cdk_search_device and carves its scratch from a fixed
64 MiB file-scope device array instead. The test calls it through the C-ABI twice in a row and
checks both results against cdk_search_device (the existing entry point) on the same inputs.
The file name sorts last so that a stop-at-first-failure run has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_inputs(w, torch, dev):
    t = {
        "coor": torch.from_numpy(np.ascontiguousarray(w.coor)).to(dev),
        "charge": torch.from_numpy(w.charge).to(dev),
        "eps": torch.from_numpy(w.eps).to(dev),
        "slot": torch.from_numpy(w.slot).to(dev),
        "quats": torch.from_numpy(np.ascontiguousarray(w.quats)).to(dev),
    }
    return t


def _call(fn, handle, w, t, e, i):
    from cdocker_b200 import _lib as L
    rc = fn(handle, w.coor.shape[1], w.coor.shape[0], C.c_void_p(t["coor"].data_ptr()),
            C.c_void_p(t["charge"].data_ptr()), C.c_void_p(t["eps"].data_ptr()),
            C.c_void_p(t["slot"].data_ptr()), w.quats.shape[1],
            C.c_void_p(t["quats"].data_ptr()), C.c_void_p(e.data_ptr()),
            C.c_void_p(i.data_ptr()), None)
    L.check(rc)


@pytest.mark.parametrize("name,nconf,nq", [("c0_32", 1, 200), ("c1_64", 2, 40)])
def test_noalloc_matches_search_device_twice(name, nconf, nq):
    import torch
    from cdocker_b200 import Receptor, synth
    from cdocker_b200 import _lib as L
    from tests.parity import rel_err

    w = synth.make_workload(name, seed=2, n_conf=nconf, n_q=nq)
    dev = torch.device("cuda", 0)
    t = _device_inputs(w, torch, dev)
    n_rot = w.n_rot
    lib = L.lib()
    with Receptor(w.grids, w.spacing) as rec:
        e_ref = torch.empty(n_rot, device=dev)
        i_ref = torch.empty(n_rot, 3, dtype=torch.int32, device=dev)
        _call(lib.cdk_search_device, rec.handle, w, t, e_ref, i_ref)
        torch.cuda.synchronize()
        ref_e, ref_i = e_ref.cpu().numpy(), i_ref.cpu().numpy()
        for _ in range(2):
            e = torch.full((n_rot,), float("nan"), device=dev)
            i = torch.full((n_rot, 3), -7, dtype=torch.int32, device=dev)
            _call(lib.cdk_search_device_noalloc, rec.handle, w, t, e, i)
            torch.cuda.synchronize()
            got_e, got_i = e.cpu().numpy(), i.cpu().numpy()
            assert np.all(np.isfinite(got_e))
            # same kernels on the same inputs: the FP32 tolerance of the parity tests
            assert rel_err(got_e, ref_e).max() <= 1e-4
            np.testing.assert_array_equal(got_i, ref_i)


def _status(fn, handle, w, t, e, i):
    return fn(handle, w.coor.shape[1], w.coor.shape[0], C.c_void_p(t["coor"].data_ptr()),
              C.c_void_p(t["charge"].data_ptr()), C.c_void_p(t["eps"].data_ptr()),
              C.c_void_p(t["slot"].data_ptr()), w.quats.shape[1],
              C.c_void_p(t["quats"].data_ptr()), C.c_void_p(e.data_ptr()),
              C.c_void_p(i.data_ptr()), None)


def test_noalloc_rejects_tensor_core_context():
    """The entry point runs the FP32 form only: a split-BF16 context is refused with
    CDK_ERR_UNSUPPORTED and a message, rather than searched in another form."""
    import torch
    from cdocker_b200 import CDK_FORM_BF16X3, Receptor, synth
    from cdocker_b200 import _lib as L

    w = synth.make_workload("c0_32", seed=2, n_conf=1, n_q=8)
    dev = torch.device("cuda", 0)
    t = _device_inputs(w, torch, dev)
    e = torch.empty(w.n_rot, device=dev)
    i = torch.empty(w.n_rot, 3, dtype=torch.int32, device=dev)
    with Receptor(w.grids, w.spacing, form=CDK_FORM_BF16X3) as rec:
        rc = _status(L.lib().cdk_search_device_noalloc, rec.handle, w, t, e, i)
        assert rc == L.CDK_ERR_UNSUPPORTED
        assert "FP32 form only" in L.last_error()


def test_noalloc_rejects_rotation_beyond_scratch():
    """A 128^3, K = 9 context and a ligand whose box spans the whole grid: one rotation needs
    more than the 64 MiB array, so the call is refused before any search kernel runs."""
    import torch
    from cdocker_b200 import Receptor
    from cdocker_b200 import _lib as L

    class W:
        pass

    w = W()
    rng = np.random.default_rng(5)
    grids = rng.normal(0.0, 1.0, size=(9, 128, 128, 128)).astype(np.float32)
    w.coor = np.array([[[0.0, 0.0, 0.0], [70.0, 0.0, 0.0]]], np.float32)
    w.charge = np.array([0.5, -0.5], np.float32)
    w.eps = np.array([0.1, 0.1], np.float32)
    w.slot = np.array([0, 1], np.int32)
    w.quats = np.array([[[1.0, 0.0, 0.0, 0.0]]], np.float32)
    dev = torch.device("cuda", 0)
    t = _device_inputs(w, torch, dev)
    e = torch.empty(1, device=dev)
    i = torch.empty(1, 3, dtype=torch.int32, device=dev)
    with Receptor(grids, 0.5) as rec:
        rc = _status(L.lib().cdk_search_device_noalloc, rec.handle, w, t, e, i)
        assert rc == L.CDK_ERR_UNSUPPORTED
        assert "exceeds the no-alloc scratch" in L.last_error()


def test_noalloc_overflow_count_matches_search_device():
    """The overflow counter kept in the static array: a non-unit quaternion (norm^2 = 1.5)
    stretches one rotation's ligand past the planned box (with a non-empty window), which
    k_prep flags; both entry points return CDK_ERR_OVERFLOW, twice in a row for this one."""
    import torch
    from cdocker_b200 import Receptor, synth
    from cdocker_b200 import _lib as L

    w = synth.make_workload("c0_32", seed=2, n_conf=1, n_q=16)
    w.quats = w.quats.copy()
    w.quats[0, 5] = np.array([np.sqrt(1.5), 0.0, 0.0, 0.0], np.float32)
    dev = torch.device("cuda", 0)
    t = _device_inputs(w, torch, dev)
    e = torch.empty(w.n_rot, device=dev)
    i = torch.empty(w.n_rot, 3, dtype=torch.int32, device=dev)
    with Receptor(w.grids, w.spacing) as rec:
        assert _status(L.lib().cdk_search_device, rec.handle, w, t, e, i) == L.CDK_ERR_OVERFLOW
        ref_e = e.cpu().numpy()
        for _ in range(2):
            e.fill_(float("nan"))
            rc = _status(L.lib().cdk_search_device_noalloc, rec.handle, w, t, e, i)
            assert rc == L.CDK_ERR_OVERFLOW
            assert "overflowed the planned ligand box" in L.last_error()
            got = e.cpu().numpy()
            ok = np.arange(w.n_rot) != 5
            np.testing.assert_array_equal(got[ok], ref_e[ok])
