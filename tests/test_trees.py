"""Iterated pendant-tree pruning: the oracle's host restatement (CPU only).

oracle/trees_ref.cpp is compiled into a small harness.  On a forest
every vertex is peeled (or is the last vertex of its tree), no core search
runs, and the closed-form tree terms must equal the oracle's Brandes bc for
any source multiset."""
import os
import subprocess

import numpy as np
import pytest

import bcg
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cstdio>
#include <vector>
#include "trees_ref.hpp"
using namespace oracle_trees;
int main() {
    unsigned n, m, k;
    if (scanf("%u %u %u", &n, &m, &k) != 3) return 1;
    std::vector<uint32_t> offs(n + 1), adj(m), cnt(n, 0);
    for (auto &x : offs) scanf("%u", &x);
    for (auto &x : adj) scanf("%u", &x);
    for (unsigned i = 0; i < k; ++i) { unsigned s; scanf("%u", &s); if (offs[s + 1] > offs[s]) ++cnt[s]; }
    TreeInfo t;
    std::vector<uint32_t> cdeg, ext, intl, o2, a2;
    peel_trees(offs.data(), adj.data(), n, t, cdeg, ext, intl, o2, a2);
    label_components(o2.data(), a2.data(), n, intl, t);
    std::vector<double> acc;
    tree_bc(t, cnt, acc);
    printf("%zu %zu\n", t.order.size(), a2.size());
    for (unsigned v = 0; v < n; ++v) printf("%.17g %u\n", acc[v], t.anchor[v]);
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("trees")
    (d / "h.cpp").write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "oracle"), "-I",
                    os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "oracle", "trees_ref.cpp"), str(d / "h.cpp"), "-o", str(exe)],
                   check=True)

    def run(offs, adj, src):
        n = len(offs) - 1
        txt = f"{n} {len(adj)} {len(src)}\n" + " ".join(map(str, offs)) + "\n" + " ".join(map(str, adj)) + "\n"
        txt += " ".join(map(str, src)) + "\n"
        out = subprocess.run([str(exe)], input=txt, capture_output=True, text=True, check=True).stdout.split("\n")
        peeled, core_nnz = map(int, out[0].split())
        vals = [line.split() for line in out[1:1 + n]]
        return peeled, core_nnz, np.array([float(a) for a, _ in vals]), np.array([int(b) for _, b in vals])

    return run


def _forest(rng, sizes):
    pairs, base = [], 0
    for k in sizes:
        for i in range(1, k):
            pairs.append((base + i, base + int(rng.integers(0, i))))  # random recursive tree
        base += k
    return bcg.from_pairs(np.array(pairs, dtype=np.uint64).reshape(-1, 2), base)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_forest_tree_terms_equal_brandes(harness, seed):
    rng = np.random.default_rng(seed)
    offs, adj = _forest(rng, [1, 2, 3, 7, 20, 41])
    n = len(offs) - 1
    for src in (np.arange(n), rng.integers(0, n, size=30), np.array([5, 5, 5, 10])):
        peeled, core_nnz, acc, _ = harness(offs, adj, src)
        ref, _ = oracle.bc(offs, adj, np.asarray(src, dtype=np.uint32))
        assert core_nnz == 0
        np.testing.assert_allclose(acc, ref, rtol=1e-12, atol=1e-9)


def test_peeling_anchors_and_core(harness):
    # triangle 0-1-2 with a path 2-3-4 and a star 1-5,1-6, plus an isolated edge 7-8
    offs, adj = bcg.from_pairs([[0, 1], [1, 2], [2, 0], [2, 3], [3, 4], [1, 5], [1, 6], [7, 8]], 9)
    peeled, core_nnz, acc, anchor = harness(offs, adj, [])
    assert core_nnz == 6 and peeled == 5  # 3, 4, 5, 6 and one end of the isolated edge
    assert anchor.tolist()[:7] == [0, 1, 2, 2, 2, 1, 1]
    assert anchor[7] == anchor[8] and anchor[7] in (7, 8)


RELABEL = r"""
#include <cstdio>
#include <vector>
#include "trees_ref.hpp"
using namespace oracle_trees;
int main() {
    unsigned n, m;
    if (scanf("%u %u", &n, &m) != 2) return 1;
    std::vector<uint32_t> offs(n + 1), adj(m);
    for (auto &x : offs) scanf("%u", &x);
    for (auto &x : adj) scanf("%u", &x);
    TreeInfo t;
    std::vector<uint32_t> cdeg, ext, intl, o2, a2;
    const uint32_t nlive = peel_trees(offs.data(), adj.data(), n, t, cdeg, ext, intl, o2, a2);
    printf("%u\n", nlive);
    for (auto x : t.parent) printf("%u ", x == kNoRoot ? 0u : 1u); printf("\n");
    for (auto x : cdeg) printf("%u ", x); printf("\n");
    for (auto x : ext) printf("%u ", x); printf("\n");
    for (auto x : o2) printf("%u ", x); printf("\n");
    for (auto x : a2) printf("%u ", x); printf("\n");
}
"""


def test_relabel_keeps_the_kept_graph(tmp_path):
    """The kept graph (every edge between two unpeeled vertices) comes out
    renumbered with its vertices that keep an edge first, in their original
    order; the renumbered CSR is that graph."""
    (tmp_path / "r.cpp").write_text(RELABEL)
    exe = tmp_path / "r"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "oracle"), "-I",
                    os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "oracle", "trees_ref.cpp"), str(tmp_path / "r.cpp"), "-o", str(exe)],
                   check=True)
    offs, adj = bcg.generate("rmat:scale=9,ef=4,seed=5,pendant_frac=0.3,pendant_mean=5")
    n = len(offs) - 1
    txt = f"{n} {len(adj)}\n" + " ".join(map(str, offs)) + "\n" + " ".join(map(str, adj)) + "\n"
    out = subprocess.run([str(exe)], input=txt, capture_output=True, text=True, check=True).stdout.split("\n")
    nlive = int(out[0])
    peeled, cdeg, ext, o2, a2 = (np.array(out[i].split(), dtype=np.int64) for i in range(1, 6))
    kept = [[] if peeled[v] else [u for u in adj[offs[v]:offs[v + 1]] if not peeled[u]] for v in range(n)]
    assert cdeg.tolist() == [len(k) for k in kept]
    assert nlive == int((cdeg > 0).sum()) and 0 < nlive < n
    assert sorted(ext.tolist()) == list(range(n))
    assert np.all(cdeg[ext[:nlive]] > 0) and np.all(cdeg[ext[nlive:]] == 0)
    assert np.all(np.diff(ext[:nlive]) > 0)  # original order kept
    intl = np.empty(n, dtype=np.int64)
    intl[ext] = np.arange(n)
    for i in range(n):
        v = ext[i]
        assert a2[o2[i]:o2[i + 1]].tolist() == intl[np.array(kept[v], dtype=np.int64)].tolist()


COMPONENTS = r"""
#include <cstdio>
#include <vector>
#include "trees_ref.hpp"
using namespace oracle_trees;
int main() {
    unsigned n, m;
    if (scanf("%u %u", &n, &m) != 2) return 1;
    std::vector<uint32_t> offs(n + 1), adj(m);
    for (auto &x : offs) scanf("%u", &x);
    for (auto &x : adj) scanf("%u", &x);
    TreeInfo t;
    std::vector<uint32_t> cdeg, ext, intl, o2, a2;
    peel_trees(offs.data(), adj.data(), n, t, cdeg, ext, intl, o2, a2);
    label_components(o2.data(), a2.data(), n, intl, t);
    printf("%zu\n", t.comp_n.size());
    for (auto x : t.comp) printf("%u ", x); printf("\n");
    for (auto x : t.comp_n) printf("%lu ", (unsigned long)x); printf("\n");
}
"""


@pytest.mark.parametrize("spec", ["er:scale=14,ef=1,seed=11", "rmat:scale=13,ef=2,seed=4,pendant_frac=0.3,pendant_mean=6"])
def test_parallel_components_match_scipy(tmp_path, spec):
    """Peeling and the union-find component labels, built with OpenMP and run
    on 8 threads, against scipy's connected components of the input graph:
    the same partition, numbered in the order of each component's first
    vertex, with the right sizes."""
    scipy_cc = pytest.importorskip("scipy.sparse.csgraph")
    import scipy.sparse as sp
    (tmp_path / "c.cpp").write_text(COMPONENTS)
    exe = tmp_path / "c"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-I", os.path.join(ROOT, "oracle"), "-I",
                    os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "oracle", "trees_ref.cpp"), str(tmp_path / "c.cpp"), "-o", str(exe)],
                   check=True)
    offs, adj = bcg.generate(spec)
    n = len(offs) - 1
    txt = f"{n} {len(adj)}\n" + " ".join(map(str, offs)) + "\n" + " ".join(map(str, adj)) + "\n"
    env = dict(os.environ, OMP_NUM_THREADS="8")
    for _ in range(3):  # thread interleavings differ from run to run
        out = subprocess.run([str(exe)], input=txt, capture_output=True, text=True, check=True, env=env).stdout.split("\n")
        ncomp = int(out[0])
        comp = np.array(out[1].split(), dtype=np.int64)
        comp_n = np.array(out[2].split(), dtype=np.int64)
        g = sp.csr_matrix((np.ones(len(adj)), adj.astype(np.int64), offs.astype(np.int64)), shape=(n, n))
        nref, lab = scipy_cc.connected_components(g, directed=False)
        assert ncomp == nref
        # renumber scipy's labels by first vertex, as the harness does
        first = {}
        for v in range(n):
            first.setdefault(lab[v], len(first))
        ref = np.array([first[x] for x in lab])
        assert np.array_equal(comp, ref)
        assert np.array_equal(comp_n, np.bincount(ref, minlength=nref))


@pytest.mark.parametrize("spec", ["rmat:scale=10,ef=16,seed=7,pendant_frac=0.1,pendant_mean=4",
                                  "rmat:scale=11,ef=8,seed=3,pendant_frac=0.3,pendant_mean=6",
                                  "rmat:scale=9,ef=2,seed=4"])
def test_pruned_cpu_brandes_matches_oracle(spec):
    """oracle.bc_trees (peeling, reach-weighted searches of the kept graph from
    the sources' anchors, closed-form tree terms) against the unpruned
    Brandes oracle: the same bc, TEPS edges and skipped sources."""
    offs, adj = bcg.generate(spec)
    n = len(offs) - 1
    for src in (np.arange(n, dtype=np.uint32), bcg.sample_sources(n, 90, 5)):
        ref, ost = oracle.bc(offs, adj, src, nthreads=4)
        got, st = oracle.bc_trees(offs, adj, src, nthreads=4)
        assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-12
        assert st["teps_edges"] == ost["teps_edges"] and st["skipped"] == ost["skipped"]


def test_pruned_cpu_brandes_edge_cases():
    # a star, an isolated edge, a triangle with trees, isolated vertices, a
    # path; sources repeated, pendant, isolated and in tree components
    pairs = [[0, 1], [0, 2], [0, 3], [4, 5], [6, 7], [7, 8], [8, 6], [6, 9], [6, 10], [7, 11], [11, 12],
             [14, 15], [15, 16], [16, 17]]
    offs, adj = bcg.from_pairs(pairs, 18)
    for src in (list(range(18)), [1, 1, 2, 5, 9, 12, 13, 14, 14], [13], [3]):
        ref, ost = oracle.bc(offs, adj, src)
        got, st = oracle.bc_trees(offs, adj, src)
        assert np.max(np.abs(got - ref)) < 1e-12, src
        assert st["teps_edges"] == ost["teps_edges"] and st["skipped"] == ost["skipped"]
