"""The CPU oracle pinned against known answers (CPU only).

The reference ships no tests or expected outputs; the oracle is pinned
against networkx on small graphs (tests/golden/nx_golden.json, made by
tests/golden/make_golden.py) and against hand-derived values."""
import numpy as np
import pytest

import bcg
import oracle


def _csr(g):
    edges = np.array(g["edges"], dtype=np.uint64).reshape(-1, 2)
    return bcg.from_pairs(edges, g["n"])


def test_oracle_matches_networkx_bc(golden):
    for name, g in golden["graphs"].items():
        offs, adj = _csr(g)
        src = g["sources"] if g["sources"] is not None else list(range(g["n"]))
        bc, st = oracle.bc(offs, adj, src)
        # bc is the ordered-pair sum; networkx counts unordered pairs (the
        # reference writes bc/2, bc2d.c:1065)
        np.testing.assert_allclose(bc / 2, np.array(g["bc_half"]), rtol=1e-12, atol=1e-12, err_msg=name)


def test_oracle_levels_and_sigma_exact(golden):
    for name, g in golden["graphs"].items():
        offs, adj = _csr(g)
        for s, ref in g["per_source"].items():
            lvl, sig, _, ov = oracle.single_source(offs, adj, int(s))
            assert not ov
            assert lvl.tolist() == ref["level"], (name, s)
            assert sig.tolist() == ref["sigma"], (name, s)


def test_oracle_threads_agree():
    offs, adj = bcg.generate("rmat:scale=9,ef=8,seed=5")
    src = np.arange(0, 512, 3, dtype=np.uint32)
    b1, s1 = oracle.bc(offs, adj, src, nthreads=1)
    b4, s4 = oracle.bc(offs, adj, src, nthreads=4)
    np.testing.assert_allclose(b1, b4, rtol=1e-12, atol=1e-12)
    assert s1["teps_edges"] == s4["teps_edges"] and s1["skipped"] == s4["skipped"]


def test_oracle_hand_values():
    # path 0-1-2-3: bc/2 = [0, 2, 2, 0]; star centre with 4 leaves: C(4,2) = 6
    offs, adj = bcg.from_pairs([[0, 1], [1, 2], [2, 3]], 4)
    bc, _ = oracle.bc(offs, adj, range(4))
    assert (bc / 2).tolist() == [0.0, 2.0, 2.0, 0.0]
    offs, adj = bcg.from_pairs([[0, 1], [0, 2], [0, 3], [0, 4]], 5)
    bc, _ = oracle.bc(offs, adj, range(5))
    assert bc[0] / 2 == 6.0 and not bc[1:].any()
    # single source delta on the path from 0: delta = [3, 2, 1, 0]
    offs, adj = bcg.from_pairs([[0, 1], [1, 2], [2, 3]], 4)
    lvl, sig, dl, _ = oracle.single_source(offs, adj, 0)
    assert lvl.tolist() == [0, 1, 2, 3] and sig.tolist() == [1, 1, 1, 1]
    assert dl.tolist() == [3.0, 2.0, 1.0, 0.0]


def test_oracle_skips_degree_zero_and_counts_teps_edges():
    offs, adj = bcg.from_pairs([[0, 1], [1, 2], [4, 5]], 7)  # 3 and 6 isolated
    bc, st = oracle.bc(offs, adj, [3, 0, 6, 4])
    assert st["skipped"] == 2 and st["ran"] == 2
    assert st["teps_edges"] == 2 + 1  # component edges of sources 0 and 4


def test_oracle_detects_uint64_overflow():
    # layered graph: 64 levels of 2 vertices, complete bipartite between
    # consecutive levels -> sigma doubles each level and reaches 2^64 at the end
    L = 66
    pairs = []
    for i in range(L - 1):
        for a in range(2):
            for b in range(2):
                pairs.append([1 + 2 * i + a, 1 + 2 * (i + 1) + b])
    pairs += [[0, 1], [0, 2]]
    n = 1 + 2 * L
    offs, adj = bcg.from_pairs(pairs, n)
    _, sig, _, ov = oracle.single_source(offs, adj, 0)
    assert ov


@pytest.mark.parametrize("name", ["pendant_trees", "pendant_trees_subset"])
def test_pendant_golden_includes_tree_internal_vertices(golden, name):
    g = golden["graphs"][name]
    # vertex 5 sits inside a depth-2 pendant tree: its bc is non-zero
    assert g["bc_half"][5] > 0


def test_path_length_sum_identity(golden):
    """sum_v bc[v] = sum over sources s and reachable t != s of (d(s,t) - 1):
    pinned on the golden graphs, so the GPU tests can use it at full size."""
    for name, g in golden["graphs"].items():
        offs, adj = _csr(g)
        src = g["sources"] if g["sources"] is not None else list(range(g["n"]))
        total = oracle.path_length_sum(offs, adj, src)
        assert abs(sum(g["bc_half"]) * 2 - total) <= 1e-9 * max(total, 1), name
    offs, adj = bcg.generate("rmat:scale=10,ef=8,seed=5,pendant_frac=0.1,pendant_mean=4")
    src = bcg.sample_sources(len(offs) - 1, 200, 7)
    bc, _ = oracle.bc(offs, adj, src, nthreads=4)
    assert oracle.path_length_sum(offs, adj, src, nthreads=4) == pytest.approx(bc.sum(), rel=1e-12)
