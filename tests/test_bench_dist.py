"""bench.py's multi-rank code path on CPU (gloo, world_size 2): the same
source sharding and rank-ordered bc reduction the GPU ranks use, with the
oracle standing in for each rank's engine run; and `bench.py --gpus 2`
starting its own two ranks (the CPU reference arm, so no GPU is needed)."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bcg
import bench
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SPEC = "rmat:scale=9,ef=8,seed=13,pendant_frac=0.1,pendant_mean=4"


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        offs, adj = bcg.generate(SPEC)
        n = len(offs) - 1
        outs = []
        for _ in range(2):
            mine = bench.rank_sources(bcg.sample_sources, n, 40, rank, world)
            part, _ = oracle.bc(offs, adj, mine)
            t = torch.from_numpy(part)
            bench.combine_bc(t)
            outs.append(t.numpy().copy())
        if rank == 0:
            np.save(out_path, np.stack(outs))
    finally:
        dist.destroy_process_group()


def test_bench_sharding_and_reduction(tmp_path):
    out = str(tmp_path / "bc.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    offs, adj = bcg.generate(SPEC)
    ref, _ = oracle.bc(offs, adj, bcg.sample_sources(len(offs) - 1, 80, 2))
    np.testing.assert_allclose(got[0], ref, rtol=1e-12, atol=1e-12)
    # the rank-ordered reduction gives the same bits every time
    assert np.array_equal(got[0].view(np.uint64), got[1].view(np.uint64))


def test_gpus_flag_starts_its_ranks():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0", "--sources", "64", "--graph", SPEC],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def test_cpu_baseline_reports_the_pruned_leg():
    """The bench line's cpu_baseline: the unpruned oracle on a bounded sample
    and, on the same sources, the tree-pruned oracle (the GPU arm's
    algorithm), each with a positive TEPS figure."""
    offs, adj = bcg.generate(SPEC)
    src = bcg.sample_sources(len(offs) - 1, 64, 2)
    cb = bench.cpu_baseline(offs, adj, src, budget_s=0.5)
    assert cb["kind"] == "port" and cb["value"] > 0 and cb["cores"] >= 1
    pr = cb["pruned"]
    assert pr["value"] > 0 and pr["unit"] == "TEPS" and "pendant trees folded" in pr["sample"]


def test_traffic_only_from_a_capture_of_the_same_kernel():
    """roofline.traffic comes from the committed ncu summary only when it was
    captured from the kernel instantiation that ran; otherwise null, with the
    reason in the note."""
    with open(os.path.join(ROOT, "profiles", "sweep_traffic.json")) as f:
        d = json.load(f)
    k = d["trees"]["kernel"]
    tps, note = bench.traffic_per_source("trees", k)
    assert tps == d["trees"]["dram_bytes_per_source"] and note
    tps, note = bench.traffic_per_source("trees", k.replace("false", "true"))
    assert tps is None and "no ncu capture" in note
    assert bench.traffic_per_source("no-such-mode", k) == (None, "")
