// Iterative pendant-tree pruning (BCG_PRUNE_TREES): the reference folds one
// layer of degree-1 vertices (degree_reduction, bc2d.c:314-419); here whole
// trees hanging off the graph's 2-core are folded and their betweenness is
// computed in closed form.
//
// Peeling removes degree-1 vertices until none is left; every removed vertex v
// records the neighbour it hung from (parent[v]), so the removed vertices form
// trees rooted at the remaining ("core") vertices, their anchors.  A component
// that is a tree keeps one vertex, the last one peeled to degree 0.
//
// Exactness (ordered pairs (s, t), s a requested source):
//   - A path between two vertices of one tree, or between a tree vertex and
//     anything outside its tree, is unique inside the tree and enters the
//     core only through the anchor.  So a tree vertex v lies on the path of
//     (s, t) exactly when s and t sit in different branches at v (its child
//     subtrees and "the rest of the component"), and
//       bc[v] += sum over branches B at v of (sources in B) * (n_comp - 1 - |B|).
//   - An anchor a gets the same terms for its child subtrees; pairs with the
//     source outside its tree are counted by the core search below.
//   - The core is searched from every anchor a that is requested or holds
//     requested sources in its tree, with weight mult(a) = [a in S] +
//     (sources in T_a), and every core vertex weighs 1 + reach (its tree's
//     size - 1) as a target (the engine's reach weights, init_delta
//     cuda_kernels.cu:1089-1098).  Tree sources have no other core term: their
//     paths through a are in the tree terms above.
#include <algorithm>
#include <cstdint>
#include <deque>
#include <vector>

#include "engine_internal.hpp"

namespace bcg {

void peel_trees(const uint32_t *offs, const uint32_t *adj, uint32_t n, TreeInfo &t,
                std::vector<uint32_t> &core_offs, std::vector<uint32_t> &core_adj) {
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
    // connected components of the input graph
    t.comp.assign(n, kNoRoot);
    t.comp_n.clear();
    std::vector<uint32_t> stack;
    for (uint32_t s = 0; s < n; ++s) {
        if (t.comp[s] != kNoRoot) continue;
        const uint32_t c = (uint32_t)t.comp_n.size();
        uint64_t cnt = 0;
        t.comp[s] = c;
        stack.push_back(s);
        while (!stack.empty()) {
            const uint32_t v = stack.back();
            stack.pop_back();
            ++cnt;
            for (uint32_t e = offs[v]; e < offs[v + 1]; ++e)
                if (t.comp[adj[e]] == kNoRoot) {
                    t.comp[adj[e]] = c;
                    stack.push_back(adj[e]);
                }
        }
        t.comp_n.push_back(cnt);
    }
    // the core: every edge between two kept vertices
    core_offs.assign((size_t)n + 1, 0);
    core_adj.clear();
    for (uint32_t v = 0; v < n; ++v) {
        if (!removed[v])
            for (uint32_t e = offs[v]; e < offs[v + 1]; ++e)
                if (!removed[adj[e]]) core_adj.push_back(adj[e]);
        core_offs[v + 1] = (uint32_t)core_adj.size();
    }
}

uint32_t relabel_live(const std::vector<uint32_t> &offs, const std::vector<uint32_t> &adj, uint32_t n,
                      std::vector<uint32_t> &ext, std::vector<uint32_t> &intl, std::vector<uint32_t> &offs2,
                      std::vector<uint32_t> &adj2) {
    ext.resize(n);
    intl.resize(n);
    uint32_t nlive = 0;
    for (uint32_t v = 0; v < n; ++v)
        if (offs[v + 1] > offs[v]) ext[nlive++] = v;
    uint32_t k = nlive;
    for (uint32_t v = 0; v < n; ++v)
        if (offs[v + 1] == offs[v]) ext[k++] = v;
    for (uint32_t i = 0; i < n; ++i) intl[ext[i]] = i;
    offs2.assign((size_t)n + 1, 0);
    for (uint32_t i = 0; i < n; ++i) offs2[i + 1] = offs2[i] + (offs[ext[i] + 1] - offs[ext[i]]);
    adj2.resize(adj.size());
    // ids keep their relative order, so sorted lists stay sorted
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < (int64_t)nlive; ++i) {
        const uint32_t v = ext[i];
        uint32_t *dst = adj2.data() + offs2[i];
        for (uint32_t e = offs[v]; e < offs[v + 1]; ++e) *dst++ = intl[adj[e]];
    }
    return nlive;
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

}  // namespace bcg
