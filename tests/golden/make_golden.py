"""Generates tests/golden/nx_golden.json: known-answer vectors for Brandes BC.

The reference (ck-bc program/bc-cuda) ships no tests or expected outputs, so
its quantities are pinned on small graphs against networkx (third-party,
installed in the build container, version recorded in the file):
  - bc_half: networkx.betweenness_centrality(G, normalized=False) for the
    all-sources case, or betweenness_centrality_subset(G, sources, V,
    normalized=False) for a source subset.  For undirected graphs networkx
    counts each unordered pair once, which is the reference's written value
    bc/2 (bc2d.c:1065).
  - level / sigma per listed source: networkx.single_source_shortest_path_length
    and the number of shortest paths counted with networkx.all_shortest_paths.
Run:  python tests/golden/make_golden.py   (rewrites the JSON in place)
"""
import json
import os

import networkx as nx

HERE = os.path.dirname(os.path.abspath(__file__))


def relabel(G):
    mapping = {v: i for i, v in enumerate(sorted(G.nodes(), key=lambda x: str(x)))}
    if all(isinstance(v, int) for v in G.nodes()):
        mapping = {v: i for i, v in enumerate(sorted(G.nodes()))}
    return nx.relabel_nodes(G, mapping)


def graphs():
    out = []
    out.append(("path6", nx.path_graph(6), None))
    out.append(("star5", nx.star_graph(5), None))
    out.append(("cycle7", nx.cycle_graph(7), None))
    out.append(("complete5", nx.complete_graph(5), None))
    out.append(("grid3x3", relabel(nx.grid_2d_graph(3, 3)), None))
    out.append(("grid4x5", relabel(nx.grid_2d_graph(4, 5)), None))
    two = nx.disjoint_union(nx.path_graph(4), nx.cycle_graph(3))
    two.add_node(7)  # isolated vertex
    out.append(("two_components_isolated", two, None))
    # a triangle with pendant trees of depth 1 and 2 and an isolated edge
    T = nx.Graph([(0, 1), (1, 2), (2, 0), (0, 3), (0, 4), (1, 5), (5, 6), (5, 7), (2, 8), (9, 10)])
    out.append(("pendant_trees", T, None))
    out.append(("pendant_trees_subset", T, [3, 5, 9, 1]))
    B = nx.barbell_graph(4, 3)
    out.append(("barbell4_3", B, None))
    out.append(("gnp40_seed7", nx.gnp_random_graph(40, 0.08, seed=7), None))
    out.append(("gnp40_seed7_subset", nx.gnp_random_graph(40, 0.08, seed=7), [0, 3, 11, 17, 29]))
    out.append(("ba60_seed3", nx.barabasi_albert_graph(60, 2, seed=3), None))
    out.append(("wheel8", nx.wheel_graph(8), None))
    out.append(("ladder6", nx.ladder_graph(6), None))
    out.append(("tree_r2_h4", nx.balanced_tree(2, 4), None))
    return out


def sigma_levels(G, s):
    lv = nx.single_source_shortest_path_length(G, s)
    sig = {}
    for t in G.nodes():
        if t == s:
            sig[t] = 1
        elif t in lv:
            sig[t] = sum(1 for _ in nx.all_shortest_paths(G, s, t))
        else:
            sig[t] = 0
    n = G.number_of_nodes()
    return [lv.get(v, -1) for v in range(n)], [sig[v] for v in range(n)]


def main():
    data = {"networkx_version": nx.__version__, "graphs": {}}
    for name, G, sources in graphs():
        n = G.number_of_nodes()
        assert sorted(G.nodes()) == list(range(n)), name
        edges = sorted([sorted(e) for e in G.edges()])
        if sources is None:
            bc = nx.betweenness_centrality(G, normalized=False)
        else:
            bc = nx.betweenness_centrality_subset(G, sources, list(G.nodes()), normalized=False)
        probe = sources if sources is not None else sorted({0, n // 2, n - 1})
        per = {}
        for s in probe:
            lv, sg = sigma_levels(G, s)
            per[str(s)] = {"level": lv, "sigma": sg}
        data["graphs"][name] = {"n": n, "edges": edges, "sources": sources,
                                "bc_half": [bc[v] for v in range(n)], "per_source": per}
    with open(os.path.join(HERE, "nx_golden.json"), "w") as f:
        json.dump(data, f, indent=0, sort_keys=True)


if __name__ == "__main__":
    main()
