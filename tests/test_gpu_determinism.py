"""Bitwise reproducibility of the sweep kernel.

Every neighbour sum is formed in a fixed order (adjacency order within a
lane's run, lane order across a warp, round order within a tile, chunk order
across a hub's chunks), with no floating-point atomics in those sums (the one
FP64 atomic add, into bc, meets no other add in its sweep).  So the same run
twice gives the same bits, and one source's dependencies do not depend on
which other sources share its batch or which slot it sits in."""
import numpy as np
import pytest

import bcg
import oracle
from test_gpu_parity import assert_bc_close

pytestmark = pytest.mark.gpu

SPEC = "rmat:scale=20,ef=16,a=0.57,b=0.19,c=0.19,seed=2,pendant_frac=0.1,pendant_mean=4"


@pytest.fixture(scope="module")
def big():
    offs, adj = bcg.generate(SPEC)
    src = bcg.sample_sources(len(offs) - 1, 4096, 2)
    return offs, adj, src


@pytest.mark.parametrize("flags,width", [(bcg.PRUNE_TREES, 0), (bcg.PRUNE_DEGREE1, 3), (0, 6)])
def test_two_runs_bitwise_identical(big, flags, width):
    offs, adj, src = big
    sample = src[:240]
    with bcg.Graph(offs, adj, flags) as G:
        G.set_batch_width(width)
        G.run(sample)
        first = G.bc()
        G.reset()
        G.run(sample)
        second = G.bc()
    assert np.array_equal(first.view(np.uint64), second.view(np.uint64))


def test_small_graph_runs_bitwise_identical():
    """Hub chunks (vertices with more than 512 neighbours) meet through their
    per-chunk slots: a dense small graph, all sources, three times."""
    offs, adj = bcg.generate("rmat:scale=12,ef=32,a=0.57,b=0.19,c=0.19,seed=5")
    assert np.diff(offs).max() > 1024
    n = len(offs) - 1
    src = np.arange(n, dtype=np.uint32)
    outs = []
    with bcg.Graph(offs, adj) as G:
        for _ in range(3):
            G.reset()
            G.run(src)
            outs.append(G.bc())
    ref, _ = oracle.bc(offs, adj, src, nthreads=oracle.max_threads())
    assert_bc_close(outs[0], ref, "rmat12 ef32")
    for o in outs[1:]:
        assert np.array_equal(outs[0].view(np.uint64), o.view(np.uint64))


def test_source_independent_of_batch_mates(big):
    """The same root run in slot 0 of a width-3 batch and in slot 4 of a
    width-6 batch with other roots: depth, sigma and delta bit for bit."""
    offs, adj, src = big
    deg = np.diff(offs)
    cand = [int(s) for s in src if deg[s] > 2][:8]
    with bcg.Graph(offs, adj) as G:
        l3, s3, d3 = G.debug_batch([cand[0], cand[1], cand[2]], 3)
        l6, s6, d6 = G.debug_batch([cand[3], cand[4], cand[5], cand[6], cand[0], cand[7]], 6)
    assert np.array_equal(l3[0], l6[4])
    assert np.array_equal(s3[0], s6[4])
    assert np.array_equal(d3[0].view(np.uint64), d6[4].view(np.uint64))


@pytest.mark.parametrize("flags,width,ext", [(bcg.PRUNE_TREES, 6, False), (bcg.PRUNE_DEGREE1, 3, False),
                                             (0, 1, False), (bcg.PRUNE_TREES, 6, True)])
def test_child_marks_change_no_bit(big, tmp_path, monkeypatch, flags, width, ext):
    """Backward sweeps of small levels mark their parents, and the sweep of the
    level above reads the edges of marked vertices only: the run must mark and
    filter some levels, and give the same bits as a run without marks (bc, and
    one batch's delta read-out)."""
    offs, adj, src = big
    sample = src[:60]
    trace = tmp_path / "trace.csv"
    outs = []
    for ratio in ("8", "0"):
        monkeypatch.setenv("BCG_CHILD_MARK_RATIO", ratio)
        monkeypatch.setenv("BCG_TRACE_FILE", str(trace) if ratio == "8" else "")
        with bcg.Graph(offs, adj, flags) as G:
            G.set_batch_width(width)
            if ext:
                G.set_sigma_mode(bcg.SIGMA_EXTENDED)
            G.run(sample)
            anc, _ = G.pruning()
            deg_kept = np.zeros(len(anc), dtype=np.int64)
            kept = anc == np.arange(len(anc), dtype=anc.dtype)
            np.add.at(deg_kept, np.repeat(np.arange(len(anc)), np.diff(offs))[kept[adj]], 1)
            roots = [int(s) for s in sample if kept[s] and deg_kept[s] > 0][:width]
            _, _, dl = G.debug_batch(roots, width)
            outs.append((G.bc(), dl))
    flags_seen = set()
    for line in trace.read_text().splitlines():
        if line.startswith("#"):
            continue
        f = line.split(",")
        if int(f[1]) == 3:
            flags_seen.add(int(f[4]))
    assert 1 in flags_seen and 2 in flags_seen, flags_seen  # some level marked, some filtered
    assert np.array_equal(outs[0][0].view(np.uint64), outs[1][0].view(np.uint64))
    assert np.array_equal(outs[0][1].view(np.uint64), outs[1][1].view(np.uint64))
