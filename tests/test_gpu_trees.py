"""GPU parity of iterated pendant-tree pruning (BCG_PRUNE_TREES): kept-graph
search with tree weights plus the closed-form tree terms, against the oracle
on the unpruned graph (1e-9 relative), for all-source and k-source runs
whose sources sit in trees, on anchors and in the core, duplicates included."""
import numpy as np
import pytest

import bcg
import oracle
from test_gpu_parity import assert_bc_close

pytestmark = pytest.mark.gpu

SPECS = {
    "rmat11_trees4": "rmat:scale=11,ef=8,seed=9,pendant_frac=0.2,pendant_mean=4",
    "rmat10_trees12": "rmat:scale=10,ef=4,seed=3,pendant_frac=0.3,pendant_mean=12",
    "er10_sparse": "er:scale=10,ef=1,seed=6",
    "grid_holes": "grid:w=30,h=30,drop=0.35,seed=2",
}


@pytest.mark.parametrize("name", list(SPECS))
def test_trees_match_oracle(name):
    offs, adj = bcg.generate(SPECS[name])
    n = len(offs) - 1
    rng = np.random.default_rng(7)
    with bcg.Graph(offs, adj, bcg.PRUNE_TREES) as G:
        assert G.info()["pruned"] > 0
        for src in (np.arange(n, dtype=np.uint32),
                    rng.choice(n, size=min(n, 150), replace=False).astype(np.uint32),
                    np.array([0, 0, 1, n - 1, n - 1, n // 2], dtype=np.uint32)):
            G.reset()
            st = G.run(src)
            ref, ost = oracle.bc(offs, adj, src)
            assert_bc_close(G.bc(), ref, f"{name} trees")
            assert st.teps_edges == ost["teps_edges"]
            assert st.skipped == ost["skipped"]


def test_trees_fold_more_than_one_layer():
    offs, adj = bcg.generate(SPECS["rmat10_trees12"])
    with bcg.Graph(offs, adj, bcg.PRUNE_DEGREE1) as G1, bcg.Graph(offs, adj, bcg.PRUNE_TREES) as Gt:
        one = G1.info()["pruned"]
        many = Gt.info()["pruned"]
        assert many > one
        n = len(offs) - 1
        src = np.arange(n, dtype=np.uint32)
        G1.run(src)
        Gt.run(src)
        assert_bc_close(Gt.bc(), G1.bc(), "trees vs one layer")


def test_tree_component_and_refusals():
    # a path (a tree component) and a triangle with a tail
    offs, adj = bcg.from_pairs([[0, 1], [1, 2], [2, 3], [4, 5], [5, 6], [6, 4], [6, 7], [7, 8]], 9)
    ref, ost = oracle.bc(offs, adj, range(9))
    with bcg.Graph(offs, adj, bcg.PRUNE_TREES) as G:
        st = G.run(np.arange(9, dtype=np.uint32))
        assert_bc_close(G.bc(), ref, "path + triangle")
        assert st.teps_edges == ost["teps_edges"]
        # the path keeps vertex 1 (the last pair resolves to the smaller id);
        # the tail 7-8 folds into 6
        anc, reach = G.pruning()
        assert anc[0] == anc[2] == anc[3] == 1 and anc[7] == anc[8] == 6
        assert reach[1] == 3 and reach[6] == 2 and reach[4] == 0 and reach[8] == 0
        with pytest.raises(bcg.BcgError):
            G.single_source(0)
        reach = np.zeros(9, dtype=np.uint32)
        with pytest.raises(bcg.BcgError):
            bcg._check(bcg.lib().bcg_graph_set_reach(G.h, bcg._p32(reach)))


@pytest.mark.parametrize("spec", list(SPECS.values()) +
                         ["rmat:scale=20,ef=16,a=0.57,b=0.19,c=0.19,seed=2,pendant_frac=0.1,pendant_mean=4"])
def test_device_peeling_matches_host(spec):
    """The device peeling against the oracle's host restatement: the same
    number of peeled vertices, the same anchor for every vertex of a component
    that keeps a cycle (its 2-core is unique), and in every tree component
    exactly one kept vertex that all its vertices hang from."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    offs, adj = bcg.generate(spec)
    n = len(offs) - 1
    anc_h, _, np_h = oracle.peel_trees(offs, adj)
    with bcg.Graph(offs, adj, bcg.PRUNE_TREES) as G:
        anc_d, _ = G.pruning()
        np_d = G.info()["pruned"]
    assert np_d == np_h
    ncomp, lab = connected_components(csr_matrix((np.ones(len(adj)), adj, offs), shape=(n, n)), directed=False)
    vcount = np.bincount(lab, minlength=ncomp)
    ecount = np.bincount(lab, weights=np.diff(offs), minlength=ncomp) / 2
    tree_comp = ecount == vcount - 1
    in_tree = tree_comp[lab]
    assert np.array_equal(anc_d[~in_tree], anc_h[~in_tree])
    ids = np.arange(n, dtype=np.uint32)
    kept_d = anc_d == ids
    assert np.array_equal(np.bincount(lab[kept_d & in_tree], minlength=ncomp)[tree_comp], np.ones(tree_comp.sum()))
    assert np.all(lab[anc_d] == lab)
