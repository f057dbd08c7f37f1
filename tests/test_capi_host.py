"""CPU tests of the C-ABI library: it loads without a GPU, exports every declared symbol, its
host helpers keep the reference's semantics, and its GPU entry points fail with a status
(never a crash) when no GPU is present."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from cdocker_b200 import _lib as L
from cdocker_b200 import api, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(cdk_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert set(names) <= set(L.SIGNATURES), set(names) - set(L.SIGNATURES)


def test_version_and_defaults():
    lib = L.lib()
    assert b"sm_100a" in lib.cdk_version()
    o = L.CdkOpts()
    lib.cdk_opts_default(C.byref(o))
    assert o.max_atoms == 256 and o.form == L.CDK_FORM_FP32
    # every reserved switch off by default: no per-kernel events, direct planes, no autotune,
    # the streamed tensor-core x pass where it applies, rotations grouped (reserved[4] = 0)
    assert list(o.reserved) == [0] * 8


def test_invalid_arguments_return_status():
    lib = L.lib()
    h = C.c_void_p()
    g = np.zeros((2, 30, 30, 30), np.float32)
    rc = lib.cdk_ctx_create(30, 30, 30, 0.5, 2, g.ctypes.data_as(C.POINTER(C.c_float)), None,
                            C.byref(h))
    assert rc == L.CDK_ERR_UNSUPPORTED and "cubic" in L.last_error()
    g = np.zeros((17, 32, 32, 32), np.float32)
    rc = lib.cdk_ctx_create(32, 32, 32, 0.5, 17, g.ctypes.data_as(C.POINTER(C.c_float)), None,
                            C.byref(h))
    assert rc == L.CDK_ERR_UNSUPPORTED
    rc = lib.cdk_search(None, 1, 1, None, None, None, None, 1, None, None, None, None)
    assert rc == L.CDK_ERR_INVALID


def test_gpu_entry_points_fail_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = L.lib()
    h = C.c_void_p()
    g = np.zeros((2, 32, 32, 32), np.float32)
    rc = lib.cdk_ctx_create(32, 32, 32, 0.5, 2, g.ctypes.data_as(C.POINTER(C.c_float)), None,
                            C.byref(h))
    assert rc == L.CDK_ERR_CUDA and not h.value


def test_grid_file_roundtrip_and_reference_reader(tmp_path):
    rng = np.random.default_rng(0)
    vals = rng.normal(size=(3, 4, 5, 6)).astype(np.float32)
    radii = np.array([1.2, 1.6], np.float32)
    p = str(tmp_path / "g.txt")
    api.write_grids(p, vals, radii, [1, 2, 3], [1.5, 2.0, 2.5], 0.5, 10.0)
    d = api.read_grids(p)
    assert d["num_grids"] == 3 and d["dims"] == (4, 5, 6)
    np.testing.assert_array_equal(d["values"], vals)
    np.testing.assert_array_equal(d["radii"], radii)
    assert d["spacing"] == 0.5 and d["restraint_k"] == 10.0
    from oracle import oracle as O
    if O.ref_available():
        hi = np.zeros(4, np.int32)
        hf = np.zeros(8, np.float32)
        rr = np.zeros(2, np.float32)
        vv = np.zeros(vals.size, np.float32)
        assert O.ref().ref_read_grids(p.encode(), O._pi(hi), O._pf(hf), O._pf(rr), 2,
                                      O._pf(vv), vv.size) == 0
        np.testing.assert_array_equal(vv.reshape(vals.shape), vals)
        np.testing.assert_array_equal(hf, np.array([1, 2, 3, 1.5, 2, 2.5, 0.5, 10], np.float32))


def test_read_grids_errors(tmp_path):
    with pytest.raises(L.CdkError) as e:
        api.read_grids(str(tmp_path / "missing.txt"))
    assert e.value.code == L.CDK_ERR_IO
    p = tmp_path / "short.txt"
    p.write_text("a\nb\nc\n2 2 2 2 0 0 0 1 1 1 0.5 0\n1.5\ngrid 0\n0 0 0 1.0\n")
    with pytest.raises(L.CdkError):
        api.read_grids(str(p))


def test_synth_grids_deterministic_and_capped():
    a, mid, ln = synth.make_receptor(32, 200, 16.0, seed=7)
    b, _, _ = synth.make_receptor(32, 200, 16.0, seed=7)
    assert np.array_equal(a, b)
    assert a.shape == (9, 32, 32, 32)
    assert a[:8].max() <= 3.0 and np.abs(a[8]).max() <= 40.0
    assert np.all(np.isfinite(a))


def test_workload_shapes(c0):
    assert c0.K == len(c0.used_idx) + 1
    assert c0.quats.shape == (1, 500, 4)
    assert np.all((c0.slot >= 0) & (c0.slot < c0.K - 1))
    np.testing.assert_allclose(np.linalg.norm(c0.quats, axis=-1), 1.0, atol=1e-6)
