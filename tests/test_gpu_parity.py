"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle.

Bars: BFS depths and sigma bit-exact; delta and bc within
1e-9 relative, written here as |gpu - oracle| <= 1e-9 * max(|oracle|, 1)."""
import numpy as np
import pytest

import bcg
import oracle

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def assert_bc_close(got, ref, msg=""):
    got = np.asarray(got)
    ref = np.asarray(ref)
    err = np.abs(got - ref)
    tol = RTOL * np.maximum(np.abs(ref), 1.0)
    bad = np.nonzero(err > tol)[0]
    assert bad.size == 0, f"{msg}: {bad.size} values off, first {bad[:5]} got {got[bad[:5]]} ref {ref[bad[:5]]}"


def _golden_csr(g):
    return bcg.from_pairs(np.array(g["edges"], dtype=np.uint64).reshape(-1, 2), g["n"])


GRAPHS = {
    "rmat10": "rmat:scale=10,ef=16,seed=11",
    "rmat12_s1": "rmat:scale=12,ef=16,a=0.57,b=0.19,c=0.19,seed=1",
    "er11": "er:scale=11,ef=8,seed=4",
    "grid40": "grid:w=40,h=30,drop=0.05,seed=3",
    "rmat11_pend": "rmat:scale=11,ef=8,seed=9,pendant_frac=0.1,pendant_mean=4",
}


@pytest.fixture(scope="module")
def graphs():
    return {k: bcg.generate(v) for k, v in GRAPHS.items()}


def test_device_present():
    assert bcg.device_count() >= 1


def test_single_source_exact_on_golden(golden):
    for name, g in golden["graphs"].items():
        offs, adj = _golden_csr(g)
        with bcg.Graph(offs, adj) as G:
            for s in g["per_source"]:
                s = int(s)
                lvl, sig, dl = G.single_source(s)
                olvl, osig, odl, _ = oracle.single_source(offs, adj, s)
                assert np.array_equal(lvl, olvl), (name, s)
                assert np.array_equal(sig, osig), (name, s)
                assert_bc_close(dl, odl, f"{name} delta s={s}")


@pytest.mark.parametrize("gname", list(GRAPHS))
def test_single_source_exact_synthetic(graphs, gname):
    offs, adj = graphs[gname]
    n = len(offs) - 1
    deg = np.diff(offs)
    cand = [int(np.argmax(deg)), int(np.nonzero(deg)[0][0]), int(np.nonzero(deg)[0][-1]), n // 3]
    with bcg.Graph(offs, adj) as G:
        for s in cand:
            lvl, sig, dl = G.single_source(s)
            olvl, osig, odl, ov = oracle.single_source(offs, adj, s)
            assert not ov
            assert np.array_equal(lvl, olvl), (gname, s)
            assert np.array_equal(sig, osig), (gname, s)
            assert_bc_close(dl, odl, f"{gname} delta s={s}")


def test_bc_all_sources_golden(golden):
    for name, g in golden["graphs"].items():
        offs, adj = _golden_csr(g)
        src = g["sources"] if g["sources"] is not None else list(range(g["n"]))
        for flags in (0, bcg.PRUNE_DEGREE1):
            with bcg.Graph(offs, adj, flags) as G:
                st = G.run(src)
                assert_bc_close(G.bc() / 2, np.array(g["bc_half"]), f"{name} flags={flags}")
                _, ost = oracle.bc(offs, adj, src)
                assert st.skipped == ost["skipped"], name
                assert st.teps_edges == ost["teps_edges"], name


@pytest.mark.parametrize("gname", list(GRAPHS))
@pytest.mark.parametrize("flags", [0, bcg.PRUNE_DEGREE1])
def test_bc_matches_oracle(graphs, gname, flags):
    offs, adj = graphs[gname]
    n = len(offs) - 1
    src = np.arange(n, dtype=np.uint32) if n <= 4096 else bcg.sample_sources(n, 512, 2)
    ref, ost = oracle.bc(offs, adj, src, nthreads=oracle.max_threads())
    with bcg.Graph(offs, adj, flags) as G:
        st = G.run(src)
        assert_bc_close(G.bc(), ref, f"{gname} flags={flags}")
        assert st.skipped == ost["skipped"]
        assert st.teps_edges == ost["teps_edges"]
        assert st.max_depth == ost["max_depth"] or flags


@pytest.mark.parametrize("width", [1, 3, 6])
def test_batch_widths_agree(graphs, width):
    offs, adj = graphs["rmat11_pend"]
    src = bcg.sample_sources(len(offs) - 1, 37, 5)
    ref, _ = oracle.bc(offs, adj, src)
    for flags in (0, bcg.PRUNE_DEGREE1):
        with bcg.Graph(offs, adj, flags) as G:
            G.set_batch_width(width)
            st = G.run(src)
            assert st.batch_width == width
            assert_bc_close(G.bc(), ref, f"width={width} flags={flags}")


def test_pruning_edge_cases():
    # star centre whose neighbours are all pendants, an isolated edge, a pendant
    # attached to a pendant-rich vertex, an isolated vertex, a path component
    pairs = [[0, 1], [0, 2], [0, 3],            # star: centre 0 with 3 pendants
             [4, 5],                            # isolated edge
             [6, 7], [7, 8], [8, 6], [6, 9], [6, 10], [7, 11], [11, 12],  # triangle + trees
             [14, 15], [15, 16], [16, 17]]      # path
    n = 18                                      # 13 isolated
    offs, adj = bcg.from_pairs(pairs, n)
    for src in (list(range(n)), [1, 2, 5, 9, 12, 13, 14], [0], [3]):
        ref, ost = oracle.bc(offs, adj, src)
        with bcg.Graph(offs, adj, bcg.PRUNE_DEGREE1) as G:
            anc, reach = G.pruning()
            assert reach[0] == 3 and anc[1] == 0 and anc[5] == 4 and anc[4] == 4
            # one layer only: 11 (left with one kept edge) and the path's
            # middle stay, each holding one folded vertex
            assert anc[11] == 11 and reach[11] == 1 and anc[12] == 11
            assert anc[15] == 15 and anc[16] == 16 and reach[15] == reach[16] == 1
            assert reach[1] == 0 and reach[13] == 0
            st = G.run(src)
            assert_bc_close(G.bc(), ref, f"src={src}")
            assert st.skipped == ost["skipped"]
            assert st.teps_edges == ost["teps_edges"]
            with pytest.raises(bcg.BcgError):
                G.single_source(0)  # a pruned graph is renumbered internally


def test_hub_chunks_all_modes():
    # vertex 0 adjacent to 9000 vertices (18 chunks of 512 adjacency entries)
    # plus a path through them: exercises split hubs in push, pull and
    # backward sweeps
    k = 9000
    pairs = [[0, i] for i in range(1, k + 1)] + [[i, i + 1] for i in range(1, k)] + [[k, k + 1], [k + 1, k + 2]]
    n = k + 3
    offs, adj = bcg.from_pairs(pairs, n)
    src = [0, 1, 4500, k + 2, 17]
    ref, _ = oracle.bc(offs, adj, src)
    for ratio_width in (1, 3, 6):
        with bcg.Graph(offs, adj) as G:
            G.set_batch_width(ratio_width)
            G.run(src)
            assert_bc_close(G.bc(), ref, f"width={ratio_width}")
    lvl, sig, dl = bcg.Graph(offs, adj).single_source(k + 2)
    olvl, osig, odl, _ = oracle.single_source(offs, adj, k + 2)
    assert np.array_equal(lvl, olvl) and np.array_equal(sig, osig)
    assert_bc_close(dl, odl, "hub delta")


def test_accumulates_and_resets(graphs):
    offs, adj = graphs["rmat10"]
    with bcg.Graph(offs, adj) as G:
        G.run([1, 2, 3])
        G.run([4, 5])
        ref, _ = oracle.bc(offs, adj, [1, 2, 3, 4, 5])
        assert_bc_close(G.bc(), ref, "accumulate")
        G.reset()
        assert not G.bc().any()


def test_duplicates_and_errors(graphs):
    offs, adj = graphs["rmat10"]
    n = len(offs) - 1
    ref, _ = oracle.bc(offs, adj, [7, 7, 9])
    with bcg.Graph(offs, adj, bcg.PRUNE_DEGREE1) as G:
        G.run([7, 7, 9])
        assert_bc_close(G.bc(), ref, "duplicates")
        with pytest.raises(bcg.BcgError) as e:
            G.run([n])
        assert e.value.code == bcg.ERR_ARG
    with pytest.raises(bcg.BcgError):
        bcg.Graph(np.array([0, 1, 2], np.uint32), np.array([1, 5], np.uint32))  # id >= n


def test_edgeless_graph():
    offs = np.zeros(6, np.uint32)
    adj = np.zeros(0, np.uint32)
    with bcg.Graph(offs, adj) as G:
        st = G.run(range(5))
        assert st.skipped == 5 and st.roots == 0
        assert not G.bc().any()


def test_directed_push_only():
    # directed lists (bc2d -U): adjacency of v holds u for each line "u v"
    pairs = [[0, 1], [1, 2], [2, 3], [0, 2], [3, 1]]
    offs, adj = bcg.from_pairs(pairs, 4, undirected=False)
    ref, _ = oracle.bc(offs, adj, range(4))
    with bcg.Graph(offs, adj, bcg.DIRECTED) as G:
        G.run(range(4))
        assert_bc_close(G.bc(), ref, "directed")


def test_one_shot_matches_handle(graphs):
    offs, adj = graphs["rmat11_pend"]
    src = bcg.sample_sources(len(offs) - 1, 64, 3)
    bc1, st = bcg.bc_csr(offs, adj, src, bcg.PRUNE_DEGREE1)
    ref, _ = oracle.bc(offs, adj, src)
    assert_bc_close(bc1, ref, "one-shot")


def test_rmat12_all_sources_full():
    """R-MAT scale 12, ef 16, (0.57,0.19,0.19,0.05), seed 1, all sources."""
    offs, adj = bcg.generate("rmat:scale=12,ef=16,a=0.57,b=0.19,c=0.19,seed=1")
    n = len(offs) - 1
    src = np.arange(n, dtype=np.uint32)
    ref, ost = oracle.bc(offs, adj, src, nthreads=oracle.max_threads())
    with bcg.Graph(offs, adj) as G:
        st = G.run(src)
        assert_bc_close(G.bc(), ref, "rmat12 all sources")
        assert st.teps_edges == ost["teps_edges"]
    for s in (0, 1, 100, 4095):
        if offs[s + 1] == offs[s]:
            continue
        with bcg.Graph(offs, adj) as G:
            lvl, sig, dl = G.single_source(s)
        olvl, osig, odl, _ = oracle.single_source(offs, adj, s)
        assert np.array_equal(lvl, olvl) and np.array_equal(sig, osig)
        assert_bc_close(dl, odl, f"rmat12 delta s={s}")


@pytest.mark.parametrize("ratio", ["0", "1e30"])
def test_every_sweep_pulls_or_pushes(graphs, ratio, monkeypatch):
    """Forward sweeps forced to one kind (ratio 0: every sweep pulls, 1e30:
    every sweep pushes) on the pendant graph, whose deep levels have frontiers
    of a few tiles: a pull there walks about one tile of the unvisited ring
    per CTA, so CTAs leave its barrier far apart.  The ring window of each
    pull must be the same in every CTA (a tile walked twice doubles sigma
    below it, a tile skipped leaves vertices undiscovered)."""
    monkeypatch.setenv("BCG_PUSH_PULL_RATIO", ratio)
    offs, adj = graphs["rmat11_pend"]
    deg = np.diff(offs)
    with bcg.Graph(offs, adj) as G:
        for s in [int(v) for v in np.nonzero(deg)[0][:60]]:
            lvl, sig, dl = G.single_source(s)
            olvl, osig, odl, _ = oracle.single_source(offs, adj, s)
            assert np.array_equal(lvl, olvl), (ratio, s)
            assert np.array_equal(sig, osig), (ratio, s)
            assert_bc_close(dl, odl, f"ratio={ratio} delta s={s}")
    src = bcg.sample_sources(len(offs) - 1, 37, 5)
    ref, _ = oracle.bc(offs, adj, src)
    for width in (1, 3, 6):
        with bcg.Graph(offs, adj) as G:
            G.set_batch_width(width)
            G.run(src)
            assert_bc_close(G.bc(), ref, f"ratio={ratio} width={width}")


def test_run_slots_and_add_scaled(graphs):
    """bcg_run_slots searches roots in batches of a width without touching bc
    (here 8 roots: two batches of 6); every root's depths and dependencies
    match the oracle's single-source run.  bcg_add_scaled then commits a list
    of roots into bc, which must equal the oracle's bc of those sources."""
    import ctypes
    import torch
    offs, adj = graphs["rmat10"]
    n = len(offs) - 1
    deg = np.diff(offs)
    roots = np.array([int(v) for v in np.nonzero(deg)[0][:8]], dtype=np.uint32)
    nb = (len(roots) + 5) // 6
    d_delta = torch.zeros(nb * 6 * n, dtype=torch.float64, device="cuda")
    level = np.empty(len(roots) * n, dtype=np.int32)
    visited = np.zeros(len(roots), dtype=np.uint64)
    wsum = np.zeros(len(roots), dtype=np.uint64)
    L = bcg.lib()
    with bcg.Graph(offs, adj) as G:
        rc = L.bcg_run_slots(G.h, 6, roots.ctypes.data_as(bcg._u32p), len(roots), ctypes.c_void_p(d_delta.data_ptr()),
                             level.ctypes.data_as(ctypes.c_void_p), visited.ctypes.data_as(ctypes.c_void_p),
                             wsum.ctypes.data_as(ctypes.c_void_p))
        assert rc == 0, bcg.lib().bcg_last_error()
        assert not G.bc().any()
        dl = d_delta.cpu().numpy()
        for k, r in enumerate(roots):
            olvl, osig, odl, _ = oracle.single_source(offs, adj, int(r))
            assert np.array_equal(level[k * n:(k + 1) * n], olvl), int(r)
            assert_bc_close(dl[k * n:(k + 1) * n], odl, f"slot delta root={r}")
            assert visited[k] == np.count_nonzero(olvl >= 0)
            assert wsum[k] == visited[k]  # no pruning: every reached vertex weighs 1
        count = 5
        slot = np.arange(count, dtype=np.uint32)
        mult = np.ones(count)
        root_add = np.zeros(count)
        rc = L.bcg_add_scaled(G.h, ctypes.c_void_p(d_delta.data_ptr()), count, slot.ctypes.data_as(bcg._u32p),
                              mult.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), roots.ctypes.data_as(bcg._u32p),
                              root_add.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert rc == 0, bcg.lib().bcg_last_error()
        ref, _ = oracle.bc(offs, adj, roots[:count])
        assert_bc_close(G.bc(), ref, "committed roots")
