"""Multi-rank rotation sharding on CPU (gloo, world size 2): partition, gather, top-k.

The search itself needs a GPU; here each rank produces its shard's results with the oracle
(the stand-in for the per-rank GPU search) and the gather must rebuild exactly the
single-process answer.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cdocker_b200.shard import conformer_range, top_k


def test_conformer_ranges_cover_and_balance():
    for n in [0, 1, 5, 100, 101]:
        for world in [1, 2, 3, 8]:
            spans = [conformer_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        conformer_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from cdocker_b200 import synth
    from cdocker_b200.shard import conformer_range, gather_results
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = synth.make_workload("c0_32", seed=0, n_conf=5, n_q=6)
    b, e = conformer_range(5, rank, world)
    m32, idx, _ = O.search_direct(w.grids, w.spacing, w.coor[b:e], w.charge, w.eps, w.slot,
                                  w.quats[b:e], prec=1, nthreads=1)
    gm, gi = gather_results(m32, idx, 5, 6)
    np.save(os.path.join(out_dir, f"m{rank}.npy"), gm)
    np.save(os.path.join(out_dir, f"i{rank}.npy"), gi)
    dist.barrier()
    dist.destroy_process_group()


def test_gather_rebuilds_single_process_result(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    from cdocker_b200 import synth
    from oracle import oracle as O
    w = synth.make_workload("c0_32", seed=0, n_conf=5, n_q=6)
    m, i, _ = O.search_direct(w.grids, w.spacing, w.coor, w.charge, w.eps, w.slot, w.quats, prec=1)
    for r in range(world):
        gm = np.load(tmp_path / f"m{r}.npy")
        gi = np.load(tmp_path / f"i{r}.npy")
        np.testing.assert_array_equal(gm, m)
        np.testing.assert_array_equal(gi, i)
        np.testing.assert_array_equal(top_k(gm, 5), top_k(m, 5))
