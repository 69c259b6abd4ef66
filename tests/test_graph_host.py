"""Host-side ingest, normalisation, CSR build and generators (CPU only)."""
import hashlib
import math
import os

import numpy as np
import pytest

import bcg


def _lists(offs, adj):
    return [adj[offs[v]:offs[v + 1]].tolist() for v in range(len(offs) - 1)]


def test_reader_format_and_normalisation(tmp_path):
    # read_graph bc2d.c:214-247: '#' lines are comments, "u v" pairs, then
    # mirror (bc2d.c:152-170) and norm_graph (bc2d.c:430-453)
    p = tmp_path / "g.txt"
    p.write_text("# Directed graph\n# Nodes: 6 Edges: 7\n0 1\n1 0\n2 2\n1 2\n1 2\n3 4 # trailing comment\n\n4 5\n")
    offs, adj = bcg.read_edgelist(str(p), 6)
    # "3 4 # ..." contains '#', so the whole line is a comment (as in the reference)
    assert _lists(offs, adj) == [[1], [0, 2], [1], [], [5], [4]]
    offs_d, adj_d = bcg.read_edgelist(str(p), 6, undirected=False)
    # directed: list of v holds u for every line "u v" (the reference's CSC column)
    assert _lists(offs_d, adj_d) == [[1], [0], [1], [], [], [4]]


def test_reader_rejects_out_of_range_id(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("0 1\n1 7\n")
    with pytest.raises(bcg.BcgError) as e:
        bcg.read_edgelist(str(p), 4)
    assert e.value.code == bcg.ERR_IO
    assert "line 2" in str(e.value) and "(1, 7)" in str(e.value)


def test_reader_missing_file(tmp_path):
    with pytest.raises(bcg.BcgError) as e:
        bcg.read_edgelist(str(tmp_path / "nope.txt"), 4)
    assert e.value.code == bcg.ERR_IO


def test_write_read_roundtrip(tmp_path):
    offs, adj = bcg.generate("rmat:scale=8,ef=8,seed=3")
    p = str(tmp_path / "rt.txt")
    bcg.write_edgelist(p, offs, adj)
    o2, a2 = bcg.read_edgelist(p, len(offs) - 1)
    assert np.array_equal(offs, o2) and np.array_equal(adj, a2)


def test_csr_invariants_generators():
    for spec in ("rmat:scale=10,ef=16,seed=1", "er:scale=9,ef=8,seed=4", "grid:w=20,h=15,drop=0.1,seed=3",
                 "rmat:scale=9,ef=8,seed=2,pendant_frac=0.1,pendant_mean=4"):
        offs, adj = bcg.generate(spec)
        n = len(offs) - 1
        assert offs[0] == 0 and offs[-1] == len(adj)
        deg = np.diff(offs.astype(np.int64))
        assert (deg >= 0).all()
        rows = np.repeat(np.arange(n), deg)
        assert (adj < n).all() and not (adj == rows).any(), spec  # ids in range, no loops
        for v in range(n):
            lst = adj[offs[v]:offs[v + 1]]
            assert (np.diff(lst.astype(np.int64)) > 0).all(), spec  # sorted, unique
        # symmetric
        fw = set(zip(rows.tolist(), adj.tolist()))
        assert all((b, a) in fw for a, b in fw), spec


def test_generators_deterministic():
    a = bcg.generate("rmat:scale=11,ef=16,seed=7,pendant_frac=0.1,pendant_mean=4")
    b = bcg.generate("rmat:scale=11,ef=16,seed=7,pendant_frac=0.1,pendant_mean=4")
    c = bcg.generate("rmat:scale=11,ef=16,seed=8,pendant_frac=0.1,pendant_mean=4")
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not np.array_equal(a[1], c[1])


# --- Python restatement of the generators (splitmix64, chunked streams) ----
M64 = (1 << 64) - 1


def splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return state, z ^ (z >> 31)


def stream_seed(seed, idx):
    s = seed ^ ((0xD1B54A32D192ED03 * (idx + 1)) & M64)
    _, z = splitmix64(s)
    return z


def test_rmat_restatement_matches():
    scale, ef, a, b, c, seed = 7, 4, 0.57, 0.19, 0.19, 5
    m = ef << scale
    st = stream_seed(seed, 0)  # one chunk of 65536 draws covers m
    pairs = []
    for _ in range(m):
        u = v = 0
        for bit in range(scale - 1, -1, -1):
            st, z = splitmix64(st)
            r = (z >> 11) * (1.0 / 9007199254740992.0)
            if r < a:
                pass
            elif r < a + b:
                v |= 1 << bit
            elif r < a + b + c:
                u |= 1 << bit
            else:
                u |= 1 << bit
                v |= 1 << bit
        pairs.append((u, v))
    n = 1 << scale
    adj = [set() for _ in range(n)]
    for u, v in pairs:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    offs, got = bcg.generate(f"rmat:scale={scale},ef={ef},a={a},b={b},c={c},seed={seed}")
    assert _lists(offs, got) == [sorted(s) for s in adj]


def test_sample_sources_distinct_and_seeded():
    s1 = bcg.sample_sources(1000, 300, 2)
    s2 = bcg.sample_sources(1000, 300, 2)
    assert np.array_equal(s1, s2) and len(set(s1.tolist())) == 300 and s1.max() < 1000
    assert not np.array_equal(s1, bcg.sample_sources(1000, 300, 3))
    with pytest.raises(bcg.BcgError):
        bcg.sample_sources(10, 11, 1)


def test_pendant_tree_sizes():
    # 10% of 2^10 anchors, Geometric(mean 4) trees: ~410 extra vertices
    offs, adj = bcg.generate("rmat:scale=10,ef=8,seed=3,pendant_frac=0.1,pendant_mean=4")
    extra = len(offs) - 1 - 1024
    assert 250 < extra < 600
    # every tree vertex has degree >= 1 and the trees are forests hanging off
    # the R-MAT part: edges among tree vertices + anchor edges = extra
    deg = np.diff(offs)
    assert (deg[1024:] >= 1).all()


def test_grid_largest_component():
    offs, adj = bcg.generate("grid:w=30,h=30,drop=0.3,seed=3")
    n = len(offs) - 1
    assert 0 < n <= 900
    # connected: BFS from 0 reaches everything
    seen = np.zeros(n, bool)
    seen[0] = True
    frontier = [0]
    while frontier:
        nxt = []
        for u in frontier:
            for w in adj[offs[u]:offs[u + 1]]:
                if not seen[w]:
                    seen[w] = True
                    nxt.append(int(w))
        frontier = nxt
    assert seen.all()


def test_bad_specs():
    for spec in ("nope:scale=3", "rmat:scale=0", "rmat:scale=5,a=0.9,b=0.9", "grid:w=3,h=3,drop=1.5",
                 "rmat:scale=abc"):
        with pytest.raises(bcg.BcgError):
            bcg.generate(spec)


def test_benchmark_graph_shape():
    """Benchmark graph: R-MAT s20 ef16 + pendant trees on 10% (mean size 4)."""
    if os.environ.get("BCG_SKIP_BIG"):
        pytest.skip("big graph disabled")
    offs, adj = bcg.generate("rmat:scale=20,ef=16,a=0.57,b=0.19,c=0.19,seed=2,pendant_frac=0.1,pendant_mean=4")
    n = len(offs) - 1
    assert 1_048_576 + 300_000 < n < 1_048_576 + 550_000
    assert 2 * 10_000_000 < len(adj) < 2 * 17_000_000
    h = hashlib.sha256(offs.tobytes() + adj.tobytes()).hexdigest()
    assert len(h) == 64
