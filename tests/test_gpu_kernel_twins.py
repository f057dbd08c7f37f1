"""kernel.h twins: cdk_conj_mult / cdk_sum_grids against the reference's own ConjMult / SumGrids
(src/kernel.cu:5-30, compiled unmodified into oracle/_ref/libcdk_ref_cufft.so and launched with
the driver's launch shapes on padded buffers). Same inputs, the same float operations: the
results must agree bit for bit."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,K,Q", [(32, 4, 3), (64, 9, 2)])
def test_conj_mult_and_sum_grids_match_reference(n, K, Q):
    import os

    import torch
    from cdocker_b200 import _lib as L
    if not os.path.exists(O.REF_CUFFT_LIB):
        pytest.skip("reference cuFFT harness not built")
    odist, idist = n * n * (n // 2 + 1), n * n * n
    rng = np.random.default_rng(n + K)
    pot = rng.normal(0, 1, (K, odist, 2)).astype(np.float32)
    lig = rng.normal(0, 1, (Q, K, odist, 2)).astype(np.float32)
    ref_lig = np.empty_like(lig)
    ref_sum = np.empty((Q, odist, 2), np.float32)
    rc = O.refcufft().refcufft_kernels(odist, K, Q, idist, O._pf(pot), O._pf(lig), O._pf(ref_lig),
                                       O._pf(ref_sum))
    assert rc == 0
    dev = torch.device("cuda", 0)
    d_pot = torch.from_numpy(pot).to(dev)
    d_lig = torch.from_numpy(lig).to(dev)
    d_sum = torch.empty((Q, odist, 2), dtype=torch.float32, device=dev)
    lib = L.lib()
    L.check(lib.cdk_conj_mult(C.c_void_p(d_pot.data_ptr()), C.c_void_p(d_lig.data_ptr()), odist,
                              K, Q, None))
    L.check(lib.cdk_sum_grids(C.c_void_p(d_lig.data_ptr()), C.c_void_p(d_sum.data_ptr()), K,
                              odist, idist, Q, None))
    torch.cuda.synchronize()
    got_lig, got_sum = d_lig.cpu().numpy(), d_sum.cpu().numpy()
    assert np.array_equal(got_lig.view(np.uint32), ref_lig.view(np.uint32))
    assert np.array_equal(got_sum.view(np.uint32), ref_sum.view(np.uint32))


def test_twins_reject_bad_sizes():
    from cdocker_b200 import _lib as L
    lib = L.lib()
    assert lib.cdk_conj_mult(None, None, 16, 2, 1, None) == L.CDK_ERR_INVALID
    assert lib.cdk_sum_grids(None, None, 2, 16, 32, 1, None) == L.CDK_ERR_INVALID
