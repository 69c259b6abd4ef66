"""GPU parity at the benchmark's full size (R-MAT scale 20 + pendant trees).

Per-vertex comparison against the oracle on a sample of the benchmark's
sources (the oracle finishes it in seconds), bit-exact levels and sigma for a
few full-graph single-source runs, and for the whole 4096-source workload the
size-independent identity sum_v bc[v] = sum_s sum_{t reachable} (d(s,t) - 1),
whose right side needs only a BFS per source (pinned on the golden graphs in
tests/test_oracle_golden.py)."""
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


@pytest.mark.parametrize("width,flags", [(3, bcg.PRUNE_DEGREE1), (6, bcg.PRUNE_DEGREE1), (3, 0),
                                         (3, bcg.PRUNE_TREES), (6, bcg.PRUNE_TREES), (0, bcg.PRUNE_TREES)])
def test_sample_per_vertex(big, width, flags):
    """48 of the workload's sources, per vertex against the oracle on the
    unpruned graph; width 0 is the automatic choice the benchmark uses."""
    offs, adj, src = big
    sample = src[:48]
    ref, ost = oracle.bc(offs, adj, sample, nthreads=oracle.max_threads())
    with bcg.Graph(offs, adj, flags) as G:
        G.set_batch_width(width)
        st = G.run(sample)
        assert_bc_close(G.bc(), ref, f"s20 sample w={width} flags={flags}")
        assert st.teps_edges == ost["teps_edges"]
        assert st.skipped == ost["skipped"]


def test_single_source_full_graph(big):
    offs, adj, src = big
    with bcg.Graph(offs, adj) as G:  # unpruned: every vertex gets a level
        done = 0
        for s in src:
            if offs[s + 1] == offs[s]:
                continue
            lvl, sig, dl = G.single_source(int(s))
            olvl, osig, odl, ov = oracle.single_source(offs, adj, int(s))
            assert not ov
            assert np.array_equal(lvl, olvl), s
            assert np.array_equal(sig, osig), s
            assert_bc_close(dl, odl, f"s20 delta s={s}")
            done += 1
            if done == 3:
                break


@pytest.fixture(scope="module")
def big_total(big):
    offs, adj, src = big
    return oracle.path_length_sum(offs, adj, src, nthreads=oracle.max_threads())


@pytest.mark.parametrize("flags", [bcg.PRUNE_DEGREE1, bcg.PRUNE_TREES])
def test_workload_bc_total(big, big_total, flags):
    """All 4096 sources of the benchmark workload, in the one-layer mode and
    in the benchmark's own pendant-tree mode: sum of bc equals the exact
    path-length total, and the TEPS edge count equals the oracle's BFS count."""
    offs, adj, src = big
    with bcg.Graph(offs, adj, flags) as G:
        st = G.run(src)
        bc = G.bc()
    assert np.all(bc >= -1e-9)
    assert abs(bc.sum() - big_total) <= 1e-9 * big_total, (bc.sum(), big_total)
    assert st.skipped == int(np.sum(np.diff(offs)[src] == 0))


@pytest.mark.parametrize("width,flags", [(3, bcg.PRUNE_TREES), (6, bcg.PRUNE_TREES), (3, bcg.PRUNE_DEGREE1)])
def test_batch_readout_bit_exact(big, width, flags):
    """One real batch of the benchmarked kernel (all `width` slots filled with
    workload sources), read out slot by slot: on every vertex the search
    holds, depth and sigma are bit-exact and delta within 1e-9 against the
    oracle's single-source Brandes on the unpruned graph.  Pendants never lie
    on a shortest path between searched vertices, so the searched graph's
    depths, counts and (reach-weighted) dependencies are those of the input."""
    offs, adj, src = big
    with bcg.Graph(offs, adj, flags) as G:
        anc, _ = G.pruning()
        kept = anc == np.arange(len(anc), dtype=anc.dtype)
        deg_kept = np.zeros(len(anc), dtype=np.int64)
        # roots: the first workload sources that the search holds (kept, with a kept edge)
        keep_nbr = kept[adj]
        owner = np.repeat(np.arange(len(anc)), np.diff(offs))
        np.add.at(deg_kept, owner[keep_nbr], 1)
        roots = [int(s) for s in src if kept[s] and deg_kept[s] > 0][:width]
        assert len(roots) == width
        lvl, sig, dl = G.debug_batch(roots, width)
    for k, r in enumerate(roots):
        olvl, osig, odl, ov = oracle.single_source(offs, adj, r)
        assert not ov
        held = kept & (lvl[k] >= 0)
        # every kept vertex the input search reaches is reached, at the same depth
        assert np.array_equal(lvl[k][kept], olvl[kept]), (width, k, r)
        assert held.sum() > 0.3 * kept.sum()
        assert np.array_equal(sig[k][held], osig[held]), (width, k, r)
        assert_bc_close(dl[k][held], odl[held], f"delta slot {k} root {r} w={width}")
        # the pendant vertices are not part of the search
        assert np.all(lvl[k][~kept] == -1)


GRID = "grid:w=2048,h=2048,drop=0.05,seed=3"


@pytest.fixture(scope="module")
def grid():
    offs, adj = bcg.generate(GRID)
    src = bcg.sample_sources(len(offs) - 1, 256, 3)
    return offs, adj, src


def test_grid_workload_total_and_two_sources(grid):
    """The 2048 x 2048 grid workload (5% of edges dropped, largest component,
    256 sources): path counts near 2^4000, so the run switches to extended
    counts; the bc total must meet the path-length identity and two full
    single-source runs must match the __float128 oracle."""
    offs, adj, src = grid
    total = oracle.path_length_sum(offs, adj, src, nthreads=oracle.max_threads())
    with bcg.Graph(offs, adj, bcg.PRUNE_DEGREE1) as G:
        st = G.run(src)
        bc = G.bc()
    assert st.extended_sigma == 1 and st.max_depth > 2000
    assert abs(bc.sum() - total) <= 1e-9 * total, (bc.sum(), total)
    with bcg.Graph(offs, adj) as G:
        for s in src[:2]:
            lvl, slog, dl = G.single_source_ext(int(s))
            ol, oslog, odl = oracle.single_source_q(offs, adj, int(s))
            assert np.array_equal(lvl, ol)
            fin = np.isfinite(oslog)
            assert np.max(np.abs(slog[fin] - oslog[fin])) < 1e-9
            assert oslog[fin].max() > 2000
            assert_bc_close(dl, odl, f"grid delta s={s}")
