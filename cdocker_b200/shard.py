"""Rotation sharding across ranks (one process per GPU).

Rotations (conformer x quaternion pairs) are independent, so a job is cut into contiguous
conformer ranges, one per rank; each rank keeps its own copy of the receptor spectra. The
only exchange is the final gather of (minE, idx) -- 16 bytes per rotation -- after which
every rank (or rank 0) can rank poses globally. No collective runs inside the search.
"""
from __future__ import annotations

import numpy as np


def conformer_range(n_conf: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced [begin, end) of conformers for `rank` (sizes differ by <= 1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(n_conf, world)
    begin = rank * base + min(rank, extra)
    end = begin + base + (1 if rank < extra else 0)
    return begin, end


def gather_results(minE: np.ndarray, idx: np.ndarray, n_conf: int, n_q: int, group=None):
    """All-gathers every rank's (minE, idx) shard into the global arrays, in conformer order.

    Uses torch.distributed (any backend: nccl on GPUs, gloo on CPU). Shards are padded to
    the largest one so that all ranks send equal-sized tensors.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b, e = conformer_range(n_conf, rank, world)
    assert minE.shape[0] == (e - b) * n_q
    biggest = max(conformer_range(n_conf, r, world)[1] - conformer_range(n_conf, r, world)[0]
                  for r in range(world)) * n_q
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    buf = torch.full((biggest, 4), float("nan"), dtype=torch.float64, device=dev)
    if minE.shape[0]:
        local = np.concatenate([minE.astype(np.float64)[:, None], idx.astype(np.float64)], axis=1)
        buf[: minE.shape[0]] = torch.from_numpy(local).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out_e = np.empty(n_conf * n_q, np.float32)
    out_i = np.empty((n_conf * n_q, 3), np.int32)
    for r in range(world):
        rb, re_ = conformer_range(n_conf, r, world)
        cnt = (re_ - rb) * n_q
        p = parts[r][:cnt].cpu().numpy()
        out_e[rb * n_q: re_ * n_q] = p[:, 0].astype(np.float32)
        out_i[rb * n_q: re_ * n_q] = p[:, 1:].astype(np.int32)
    return out_e, out_i


def top_k(minE: np.ndarray, k: int) -> np.ndarray:
    """Indices of the k lowest energies of the gathered job, ranked as the reference ranks a
    conformer's rotations (sort_index: std::sort with strict <,
    include/GeneDiverseConformations.h:9-20, through cdk_sort_index)."""
    from .poses import sort_index
    return sort_index(minE)[:k]
