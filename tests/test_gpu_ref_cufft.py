"""Our search against the reference's own cuFFT path (oracle/_ref/libcdk_ref_cufft.so:
src/kernel.cu ConjMult/SumGrids + cuFFT + the reference host helpers, batch 50) on the same
seeded inputs."""
import os

import numpy as np
import pytest

from cdocker_b200 import Receptor
from oracle import oracle as O
from tests.parity import check_search

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(O.REF_CUFFT_LIB),
                                 reason="reference cuFFT path not built (oracle/_ref)")]


def _ref_cufft(w, quats):
    L = O.refcufft()
    q = np.ascontiguousarray(quats.reshape(-1, 4))
    n = q.shape[0]
    minE = np.empty(n, np.float32)
    idx = np.empty((n, 3), np.int32)
    times = np.zeros(6)
    rc = L.refcufft_search(w.n, w.n, w.n, w.spacing, 8, O._pf(O._f32(w.grid_radii)),
                           O._pf(O._f32(w.all_grids)), w.coor.shape[1],
                           O._pf(np.ascontiguousarray(w.coor[0])), O._pf(O._f32(w.charge)),
                           O._pf(O._f32(w.eps)), O._pf(O._f32(w.radii)), n, O._pf(q), 50,
                           O._pf(minE), O._pi(idx), times.ctypes.data_as(O._dp))
    assert rc == 0
    return minE, idx


def test_c0_ours_vs_reference_cufft_path(c0):
    w = c0
    ref_e, ref_i = _ref_cufft(w, w.quats[0])
    with Receptor(w.grids, w.spacing) as rec:
        minE, idx = rec.search(w.coor, w.charge, w.eps, w.slot, w.quats)
    q = w.quats.reshape(-1, 4)
    st = check_search(minE, idx, ref_e, ref_i,
                      lambda r: O.energy_map(w.grids, w.spacing, w.coor[0], w.charge, w.eps,
                                             w.slot, q[r]))
    assert st["n"] == 500


def test_reference_cufft_path_vs_fp64(c0):
    """The reference's own FP32 cuFFT path against the FP64 oracle: the error it carries."""
    w = c0
    ref_e, ref_i = _ref_cufft(w, w.quats[0, :100])
    _, oi, o64 = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot,
                                 w.quats[:, :100], prec=1)
    q = w.quats.reshape(-1, 4)
    check_search(ref_e, ref_i, o64, oi,
                 lambda r: O.energy_map(w.grids, w.spacing, w.coor[0], w.charge, w.eps, w.slot,
                                        q[r]))
