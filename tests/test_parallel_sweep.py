"""The sweep split across ranks (zcmir_b200.parallel) on two CPU processes over gloo.

Each rank stands in a registrar whose sweep returns the float64 oracle's lane maxima for the
rank's shard (slots ≡ rank mod 2 of the plane-size order, the engine's rule); the merged lanes
must equal the unsharded oracle's exactly, and after sharded_search both ranks hold rank 0's
pose. The GPU side of the same split is checked in test_gpu_sweep.py."""
import os
import socket
import tempfile
import types

import numpy as np
import pytest
import torch.multiprocessing as mp

G, NT, NS = 32, 6, 2


def oracle_lanes(pa, pb, shard=0, nshard=1):
    from oracle import sweep_oracle as S

    gv = S.sweep_grid(n_theta=NT, n_sigma=NS, s_min=0.8, s_max=1.25)
    st = S.sweep_setup(pa["w"], pa["h"], pb["w"], pb["h"], np.eye(3), gv, G)
    nc = len(st["cands"])
    only = {st["perm"][s] for s in range(shard, nc, nshard)}
    r = S.sweep(pa, pb, np.eye(3), gv, G=G, only=only)
    sc = np.zeros((nc, 4), np.float32)
    ix = np.full((nc, 4), 0xFFFFFFFF, np.uint32)
    c2 = r["setup"]["cell"] ** 2
    for ci, top in r["raw"].items():
        for k, (v, t) in enumerate(top):
            sc[ci, k] = np.float32(v * c2)
            ix[ci, k] = t
    return sc, ix


def images():
    from oracle import smi_oracle as O
    from zcmir_b200 import synth

    m, f, _ = synth.pair_similarity(n=64, seed=9, deg=30.0, scale=1.0, shift=(2.0, -1.0))
    return O.prepare(m.astype(np.float32) / 65535), O.prepare(f.astype(np.float32) / 65535)


class OracleShardRegistrar:
    """Stands in for a Registrar: sweep(shard, nshard) gives the oracle's lanes for that shard;
    search_lanes records what it was given and moves the pose to a rank-dependent value."""

    def __init__(self, rank):
        self.rank = rank
        self.pa, self.pb = images()
        self.pose = np.eye(3)
        self.lanes = None

    def sweep(self, n_peak=4, batch=0, shard=0, nshard=1):
        sc, ix = oracle_lanes(self.pa, self.pb, shard, nshard)
        return types.SimpleNamespace(scores=sc, index=ix, info={"candidates": len(sc)})

    def search_lanes(self, sc, ix):
        self.lanes = (sc, ix)
        self.pose = np.diag([1.0 + self.rank, 1.0, 1.0])
        return types.SimpleNamespace(H=self.pose)


def _worker(rank, ws, port, out):
    import torch.distributed as dist

    from zcmir_b200 import parallel

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws)
    try:
        reg = OracleShardRegistrar(rank)
        sc, ix, _ = parallel.sharded_sweep(reg)
        parallel.sharded_search(reg)
        np.savez(os.path.join(out, f"r{rank}.npz"), sc=sc, ix=ix, lsc=reg.lanes[0], lix=reg.lanes[1], pose=reg.pose)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_sweep_merges_to_the_whole_sweep():
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_worker, args=(2, free_port(), out), nprocs=2, join=True)
        pa, pb = images()
        full_sc, full_ix = oracle_lanes(pa, pb)
        assert (full_sc > 0).sum() > 0
        for r in range(2):
            d = np.load(os.path.join(out, f"r{r}.npz"))
            np.testing.assert_array_equal(d["sc"], full_sc)
            np.testing.assert_array_equal(d["ix"], full_ix)
            np.testing.assert_array_equal(d["lsc"], full_sc)
            np.testing.assert_array_equal(d["pose"], np.eye(3))  # rank 0's pose on both
        # the shards split the candidates: each holds some, together all
        s0, _ = oracle_lanes(pa, pb, 0, 2)
        s1, _ = oracle_lanes(pa, pb, 1, 2)
        assert ((s0 != 0).any(axis=1) & (s1 != 0).any(axis=1)).sum() == 0
        np.testing.assert_array_equal(s0 + s1, full_sc)
