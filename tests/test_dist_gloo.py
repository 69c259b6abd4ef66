"""The multi-rank host logic (source sharding + bc reduction) on CPU with the
gloo backend, world_size 2; each rank's per-source work is the oracle here
(the GPU path of a rank is covered by the gpu tests)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bcg
import oracle
import shard

SPEC = "rmat:scale=9,ef=8,seed=13,pendant_frac=0.1,pendant_mean=4"


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, deterministic, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        offs, adj = bcg.generate(SPEC)
        n = len(offs) - 1
        src = bcg.sample_sources(n, 101, 4)
        mine = shard.shard_sources(src, rank, world, mode)
        part, _ = oracle.bc(offs, adj, mine)
        t = torch.from_numpy(part)
        shard.reduce_bc(t, deterministic=deterministic)
        if rank == 0:
            np.save(out_path, t.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode,deterministic", [("block", False), ("cyclic", True)])
def test_two_rank_sharded_bc(tmp_path, mode, deterministic):
    out = str(tmp_path / "bc.npy")
    mp.spawn(_worker, args=(2, _free_port(), mode, deterministic, out), nprocs=2, join=True)
    got = np.load(out)
    offs, adj = bcg.generate(SPEC)
    ref, _ = oracle.bc(offs, adj, bcg.sample_sources(len(offs) - 1, 101, 4))
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_shard_partition():
    s = np.arange(10, dtype=np.uint32)
    parts = [shard.shard_sources(s, r, 3) for r in range(3)]
    assert [len(p) for p in parts] == [4, 3, 3]
    assert np.array_equal(np.concatenate(parts), s)
    parts = [shard.shard_sources(s, r, 3, "cyclic") for r in range(3)]
    assert sorted(np.concatenate(parts).tolist()) == s.tolist()
    with pytest.raises(ValueError):
        shard.shard_sources(s, 3, 3)
