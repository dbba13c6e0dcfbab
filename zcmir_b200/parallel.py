"""The sweep split across the ranks of a torch.distributed group, one process per GPU.

A sweep's candidate maps are independent. Rank r maps the candidates in slots ≡ r (mod N) of the
plane-size order (zcb_sweep's shard/nshard), so every rank gets candidates of every plane size.
A candidate's lane maxima are non-empty on its own rank only, so the ranks' outputs merge with
two small all-reduces: the sum of the scores and the minimum of the indices (3240 candidates ×
4 lanes ≈ 100 KB). Every rank then finishes the search from the merged lanes (zcb_search_lanes:
NMS, batched Gauss–Newton screen, finalists), and rank 0's pose is broadcast so that all ranks end
on the same pose. This is the sweep's only collective; single maps do not shard (each needs all
45 correlations of every shift) and run as independent replicas.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def _device(group):
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def merge_lanes(scores, index, group=None):
    """Every candidate's lane maxima from the ranks' shares (scores summed, indices minimised)."""
    dev = _device(group)
    s = torch.from_numpy(np.ascontiguousarray(scores, np.float32)).to(dev)
    i = torch.from_numpy(np.ascontiguousarray(index, np.uint32).astype(np.int64)).to(dev)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(i, op=dist.ReduceOp.MIN, group=group)
    return s.cpu().numpy(), i.cpu().numpy().astype(np.uint32)


def sharded_sweep(reg, group=None, n_peak=4, batch=0):
    """This rank's share of the sweep of `reg`'s images, merged over the group: (scores, index,
    this rank's info)."""
    rank, ws = dist.get_rank(group), dist.get_world_size(group)
    sw = reg.sweep(n_peak=n_peak, batch=batch, shard=rank, nshard=ws)
    sc, ix = merge_lanes(sw.scores, sw.index, group)
    return sc, ix, sw.info


def sharded_search(reg, group=None, batch=0):
    """search() with its sweep split across the group; every rank ends on rank 0's pose."""
    sc, ix, _ = sharded_sweep(reg, group, 4, batch)
    r = reg.search_lanes(sc, ix)
    H = torch.tensor(np.asarray(reg.pose, np.float64).reshape(9), device=_device(group))
    dist.broadcast(H, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    reg.pose = H.cpu().numpy().reshape(3, 3)
    return r
