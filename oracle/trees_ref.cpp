// ORACLE — test infrastructure only (never linked into the product).
//
// Host restatement of iterated pendant-tree pruning and of the closed-form
// betweenness of the tree vertices, which the engine computes on the device
// (ck-bc_b200/csrc/trees_gpu.cu).  tests/test_trees.py pins the closed form
// against the Brandes oracle on forests, and tests/test_gpu_trees.py checks
// the device peeling's kept set and subtree weights against this one.  The
// reference folds one layer of degree-1 vertices (degree_reduction,
// bc2d.c:314-419); this restatement folds whole trees.
//
// Peeling removes degree-1 vertices until none is left (a FIFO queue); every
// removed vertex v records the neighbour it hung from (parent[v]), so the
// removed vertices form trees rooted at the remaining ("core") vertices, their
// anchors.  A component that is a tree keeps one vertex, the last one peeled
// to degree 0.
//
// Exactness (ordered pairs (s, t), s a requested source):
//   - A path between two vertices of one tree, or between a tree vertex and
//     anything outside its tree, is unique inside the tree and enters the
//     core only through the anchor.  So a tree vertex v lies on the path of
//     (s, t) exactly when s and t sit in different branches at v (its child
//     subtrees and "the rest of the component"), and
//       bc[v] += sum over branches B at v of (sources in B) * (n_comp - 1 - |B|).
//   - An anchor a gets the same terms for its child subtrees.
#include <algorithm>
#include <cstdint>
#include <deque>
#include <vector>

#include "trees_ref.hpp"

namespace oracle_trees {

uint32_t peel_trees(const uint32_t *offs, const uint32_t *adj, uint32_t n, TreeInfo &t, std::vector<uint32_t> &cdeg,
                    std::vector<uint32_t> &ext, std::vector<uint32_t> &intl, std::vector<uint32_t> &offs2,
                    std::vector<uint32_t> &adj2) {
    std::vector<uint32_t> deg(n);
    for (uint32_t v = 0; v < n; ++v) deg[v] = offs[v + 1] - offs[v];
    t.parent.assign(n, kNoRoot);
    t.order.clear();
    std::vector<uint8_t> removed(n, 0);
    std::deque<uint32_t> q;
    for (uint32_t v = 0; v < n; ++v)
        if (deg[v] == 1) q.push_back(v);
    while (!q.empty()) {
        const uint32_t v = q.front();
        q.pop_front();
        if (removed[v] || deg[v] != 1) continue;  // its last neighbour went first
        uint32_t p = kNoRoot;
        for (uint32_t e = offs[v]; e < offs[v + 1]; ++e)
            if (!removed[adj[e]]) {
                p = adj[e];
                break;
            }
        removed[v] = 1;
        t.parent[v] = p;
        t.order.push_back(v);
        if (--deg[p] == 1) q.push_back(p);
    }
    // subtree sizes (children are removed before their parents) and anchors
    // (parents are settled after their children: walk the order backwards)
    t.sz.assign(n, 1);
    for (uint32_t v : t.order) t.sz[t.parent[v]] += t.sz[v];
    t.anchor.resize(n);
    for (uint32_t v = 0; v < n; ++v) t.anchor[v] = v;
    for (size_t i = t.order.size(); i-- > 0;) {
        const uint32_t v = t.order[i];
        const uint32_t p = t.parent[v];
        t.anchor[v] = removed[p] ? t.anchor[p] : p;
    }
    // the kept graph, renumbered: the kept vertices that keep an edge come
    // first (in their order), then the rest; ids keep their relative order,
    // so sorted lists stay sorted (count, number, scan, fill)
    cdeg.assign(n, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t vi = 0; vi < (int64_t)n; ++vi) {
        const uint32_t v = (uint32_t)vi;
        uint32_t c = 0;
        if (!removed[v])
            for (uint32_t e = offs[v]; e < offs[v + 1]; ++e) c += !removed[adj[e]];
        cdeg[v] = c;
    }
    ext.resize(n);
    intl.resize(n);
    uint32_t nlive = 0;
    for (uint32_t v = 0; v < n; ++v)
        if (cdeg[v]) ext[nlive++] = v;
    uint32_t k = nlive;
    for (uint32_t v = 0; v < n; ++v)
        if (!cdeg[v]) ext[k++] = v;
    for (uint32_t i = 0; i < n; ++i) intl[ext[i]] = i;
    offs2.assign((size_t)n + 1, 0);
    for (uint32_t i = 0; i < n; ++i) offs2[i + 1] = offs2[i] + cdeg[ext[i]];
    adj2.resize(offs2[n]);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < (int64_t)nlive; ++i) {
        const uint32_t v = ext[i];
        uint32_t *dst = adj2.data() + offs2[i];
        for (uint32_t e = offs[v]; e < offs[v + 1]; ++e)
            if (!removed[adj[e]]) *dst++ = intl[adj[e]];
    }
    return nlive;
}

// Components of the kept graph (offs/adj over internal ids; intl maps a
// vertex's id to its internal id, empty: the same), extended to every vertex
// through its anchor.  Union-find over the edges in parallel, always linking
// the larger root under the smaller.
void label_components(const uint32_t *offs, const uint32_t *adj, uint32_t n, const std::vector<uint32_t> &intl,
                      TreeInfo &t) {
    std::vector<uint32_t> root(n);
    for (uint32_t v = 0; v < n; ++v) root[v] = v;
    auto find = [&](uint32_t v) {
        uint32_t r = __atomic_load_n(&root[v], __ATOMIC_RELAXED);
        while (r != v) {
            const uint32_t g = __atomic_load_n(&root[r], __ATOMIC_RELAXED);
            __atomic_compare_exchange_n(&root[v], &r, g, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);  // halving
            v = r;
            r = g;
        }
        return v;
    };
#pragma omp parallel for schedule(dynamic, 2048)
    for (int64_t vi = 0; vi < (int64_t)n; ++vi) {
        const uint32_t v = (uint32_t)vi;
        for (uint32_t e = offs[v]; e < offs[v + 1]; ++e) {
            uint32_t a = v, b = adj[e];
            if (b <= a) continue;  // each edge once (lists are symmetric)
            for (;;) {
                a = find(a);
                b = find(b);
                if (a == b) break;
                if (a < b) std::swap(a, b);  // link the larger root a under b
                uint32_t expect = a;
                if (__atomic_compare_exchange_n(&root[a], &expect, b, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED))
                    break;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)n; ++v) __atomic_store_n(&root[v], find((uint32_t)v), __ATOMIC_RELAXED);
    // dense component numbers, in the order of each component's first vertex
    std::vector<uint32_t> id(n, kNoRoot);
    t.comp.assign(n, kNoRoot);
    t.comp_n.clear();
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t a = t.anchor[v];
        const uint32_t r = root[intl.empty() ? a : intl[a]];
        if (id[r] == kNoRoot) {
            id[r] = (uint32_t)t.comp_n.size();
            t.comp_n.push_back(0);
        }
        t.comp[v] = id[r];
        ++t.comp_n[id[r]];
    }
}

void tree_bc(const TreeInfo &t, const std::vector<uint32_t> &cnt, std::vector<double> &acc) {
    const size_t n = t.parent.size();
    // sources per component and per subtree (a vertex's own count included)
    std::vector<uint64_t> comp_src(t.comp_n.size(), 0);
    for (size_t v = 0; v < n; ++v) comp_src[t.comp[v]] += cnt[v];
    std::vector<uint64_t> sub(cnt.begin(), cnt.end());
    for (uint32_t v : t.order) sub[t.parent[v]] += sub[v];
    acc.assign(n, 0.0);
    for (uint32_t v : t.order) {
        const double nc = (double)t.comp_n[t.comp[v]];
        // v's subtree is a branch at its parent (a tree vertex or the anchor)
        acc[t.parent[v]] += (double)sub[v] * (nc - 1.0 - (double)t.sz[v]);
        // the rest of the component is a branch at v
        acc[v] += (double)(comp_src[t.comp[v]] - sub[v]) * ((double)t.sz[v] - 1.0);
    }
}

}  // namespace oracle_trees

// C entry for the Python wrapper: anchors and subtree sizes of every vertex
// after peeling, and the number of peeled vertices.
extern "C" int oracle_peel_trees(uint32_t n, const uint32_t *offs, const uint32_t *adj, uint32_t *anchor,
                                 uint32_t *sz, uint64_t *npeeled) {
    oracle_trees::TreeInfo t;
    std::vector<uint32_t> cdeg, ext, intl, o2, a2;
    oracle_trees::peel_trees(offs, adj, n, t, cdeg, ext, intl, o2, a2);
    for (uint32_t v = 0; v < n; ++v) {
        anchor[v] = t.anchor[v];
        sz[v] = t.sz[v];
    }
    *npeeled = t.order.size();
    return 0;
}
