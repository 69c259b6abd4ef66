"""GPU parity of the batched form (bcg_batch_*): many graphs, one packed launch.

Each graph's bc from the batched run must equal the oracle's all-sources BC of
that graph and the plain per-graph engine run (bcg_run over all vertices)
within 1e-9 relative.  Sigma is the same uint64 sum in both paths (the same
sweep kernel), so the bc bar carries it."""
import numpy as np
import pytest

import bcg
import oracle
import workloads
from test_gpu_parity import assert_bc_close

pytestmark = pytest.mark.gpu


def _mixed_graphs():
    specs = ["rmat:scale=9,ef=16,a=0.57,b=0.19,c=0.19,seed=5",
             "er:scale=8,ef=4,seed=6",
             "rmat:scale=7,ef=8,a=0.57,b=0.19,c=0.19,seed=7",
             "grid:w=12,h=9,drop=0.1,seed=8",
             "er:scale=6,ef=2,seed=9",
             "rmat:scale=10,ef=8,a=0.45,b=0.15,c=0.15,seed=10",
             "rmat:scale=5,ef=4,seed=11"]
    graphs = [bcg.generate(s) for s in specs]
    graphs.append(bcg.from_pairs([[0, 1], [1, 2], [2, 3], [3, 4]], 5))  # path
    graphs.append((np.zeros(4, np.uint32), np.zeros(0, np.uint32)))     # edgeless
    graphs.append(bcg.from_pairs([[0, 1], [0, 2], [0, 3], [4, 5]], 7))  # star + edge + isolated
    return graphs


def _plain(offs, adj):
    n = len(offs) - 1
    with bcg.Graph(offs, adj) as G:
        G.run(np.arange(n, dtype=np.uint32))
        return G.bc()


def test_batch_matches_oracle_and_plain():
    graphs = _mixed_graphs()
    with bcg.Batch(graphs) as B:
        st = B.run()
        info = B.info()
        assert info["captured"], "the packed launch was not captured into a CUDA graph"
        total_edges = 0
        for i, (offs, adj) in enumerate(graphs):
            n = len(offs) - 1
            ref, ost = oracle.bc(offs, adj, np.arange(n, dtype=np.uint32))
            got = B.bc(i)
            assert_bc_close(got, ref, f"graph {i} vs oracle")
            assert_bc_close(got, _plain(offs, adj), f"graph {i} vs plain run")
            total_edges += ost["teps_edges"]
        assert st.teps_edges == total_edges
        # a second run replays the captured graph and adds the same values again
        B.run()
        for i, (offs, adj) in enumerate(graphs):
            n = len(offs) - 1
            ref, _ = oracle.bc(offs, adj, np.arange(n, dtype=np.uint32))
            assert_bc_close(B.bc(i), 2 * ref, f"graph {i} accumulated")
        B.reset()
        assert not B.bc(0).any()


def test_batch_autotune_keeps_results():
    graphs = _mixed_graphs()[:6]
    with bcg.Batch(graphs) as B:
        w, tv, te = B.autotune(sample_batches=2)
        assert w in (1, 3, 6) and (tv, te) in ((32, 512), (32, 256), (32, 128), (16, 128), (16, 64))
        assert not B.bc(0).any()  # tuning runs are not left in the accumulators
        info = B.info()
        assert (info["width"], info["tile_vertices"], info["tile_entries"]) == (w, tv, te)
        B.run()
        for i, (offs, adj) in enumerate(graphs):
            n = len(offs) - 1
            ref, _ = oracle.bc(offs, adj, np.arange(n, dtype=np.uint32))
            assert_bc_close(B.bc(i), ref, f"graph {i} after autotune")


def test_batch_workload_prefix_matches_plain():
    """Small graphs of the seeded batched workload (scale <= 10), each against
    its own plain engine run."""
    specs = [s for s in workloads.batched_specs()[:60] if workloads.spec_scale_ef(s)[0] <= 10][:24]
    graphs = [bcg.generate(s) for s in specs]
    with bcg.Batch(graphs) as B:
        B.autotune()
        B.run()
        for i, (offs, adj) in enumerate(graphs):
            assert_bc_close(B.bc(i), _plain(offs, adj), specs[i])


def test_batch_rejects_bad_input():
    with pytest.raises(bcg.BcgError):
        bcg.Batch([])
    offs, adj = bcg.from_pairs([[0, 1]], 2)
    bad = adj.copy()
    bad[0] = 7
    with pytest.raises(bcg.BcgError):
        bcg.Batch([(offs, adj), (offs, bad)])
