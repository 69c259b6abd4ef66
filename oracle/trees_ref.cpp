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
#include <chrono>
#include <deque>
#include <vector>

#include "trees_ref.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

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

// ---------------------------------------------------------------------------
// Tree-pruned Brandes on the host: the same quantity as oracle_bc, computed the
// way the engine's BCG_PRUNE_TREES mode does (peel, search the kept graph from
// every anchor that holds requested sources with reach weights, add the tree
// terms in closed form).  bench.py times it as the pruned CPU leg beside the
// unpruned one; tests/test_trees.py pins it to oracle_bc.

namespace oracle_trees {

// One search of the kept graph (internal ids, CSR o2/a2) from root r: every
// vertex weighs 1 + reach as a target, so delta starts at reach; mult times
// the dependencies go to acc (the root's own excluded).  lvl must be -1 on
// entry and is left -1 on exit.  Returns the visited vertices.
static uint32_t weighted_one(const uint32_t *o2, const uint32_t *a2, const double *reach, uint32_t r, double mult,
                             int32_t *lvl, uint64_t *sigma, double *delta, uint32_t *queue, double *acc,
                             int *overflow) {
    uint32_t head = 0, tail = 0;
    lvl[r] = 0;
    sigma[r] = 1;
    delta[r] = reach[r];
    queue[tail++] = r;
    while (head < tail) {
        const uint32_t c = queue[head++];
        for (uint32_t e = o2[c]; e < o2[c + 1]; ++e) {
            const uint32_t w = a2[e];
            if (lvl[w] < 0) {
                lvl[w] = lvl[c] + 1;
                sigma[w] = 0;
                delta[w] = reach[w];
                queue[tail++] = w;
            }
            if (lvl[w] == lvl[c] + 1) {
                const uint64_t t = sigma[w] + sigma[c];
                if (t < sigma[w]) *overflow = 1;
                sigma[w] = t;
            }
        }
    }
    // children before parents: walk the queue backwards
    for (uint32_t i = tail; i-- > 1;) {
        const uint32_t w = queue[i];
        const double xw = (1.0 + delta[w]) / (double)sigma[w];
        for (uint32_t e = o2[w]; e < o2[w + 1]; ++e) {
            const uint32_t v = a2[e];
            if (lvl[v] == lvl[w] - 1) delta[v] += (double)sigma[v] * xw;
        }
        acc[w] += mult * delta[w];
    }
    for (uint32_t i = 0; i < tail; ++i) lvl[queue[i]] = -1;
    return tail;
}

}  // namespace oracle_trees

struct oracle_trees_stats {
    uint64_t skipped;     // sources of degree 0
    uint64_t roots;       // anchors searched
    uint64_t teps_edges;  // per source, the edges of its component in the input graph
    double peel_seconds;  // peeling and component labels
    int overflow;         // a uint64 path count wrapped
};

extern "C" int oracle_bc_trees(uint32_t n, const uint32_t *offs, const uint32_t *adj, const uint32_t *sources,
                               uint64_t nsrc, int nthreads, double *bc, oracle_trees_stats *st) {
    using namespace oracle_trees;
    const auto t0 = std::chrono::steady_clock::now();
    TreeInfo t;
    std::vector<uint32_t> cdeg, ext, intl, o2, a2;
    const uint32_t nlive = peel_trees(offs, adj, n, t, cdeg, ext, intl, o2, a2);
    label_components(o2.data(), a2.data(), n, intl, t);
    const auto t1 = std::chrono::steady_clock::now();
    // edges per component of the input graph
    std::vector<uint64_t> comp_deg(t.comp_n.size(), 0);
    for (uint32_t v = 0; v < n; ++v) comp_deg[t.comp[v]] += offs[v + 1] - offs[v];
    // source multiplicities: per vertex (tree terms) and per anchor (searches)
    std::vector<uint32_t> cnt(n, 0);
    std::vector<double> mult(nlive, 0.0);
    uint64_t skipped = 0, teps = 0;
    for (uint64_t i = 0; i < nsrc; ++i) {
        const uint32_t s = sources[i];
        if (s >= n) return -1;
        if (offs[s + 1] == offs[s]) {
            ++skipped;
            continue;
        }
        ++cnt[s];
        teps += comp_deg[t.comp[s]] / 2;
        const uint32_t ia = intl[t.anchor[s]];
        if (ia < nlive) mult[ia] += 1.0;  // an anchor with kept edges: searched
    }
    std::vector<uint32_t> roots;
    for (uint32_t i = 0; i < nlive; ++i)
        if (mult[i] > 0.0) roots.push_back(i);
    std::vector<double> reach(nlive);
    for (uint32_t i = 0; i < nlive; ++i) reach[i] = (double)t.sz[ext[i]] - 1.0;
    int nt = nthreads > 0 ? nthreads : 1;
#ifndef _OPENMP
    nt = 1;
#endif
    std::vector<double> part((size_t)nt * nlive, 0.0);
    int overflow = 0;
#pragma omp parallel num_threads(nt) reduction(| : overflow)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        std::vector<int32_t> lvl(nlive, -1);
        std::vector<uint64_t> sigma(nlive);
        std::vector<double> delta(nlive);
        std::vector<uint32_t> queue(nlive);
        double *acc = part.data() + (size_t)tid * nlive;
#pragma omp for schedule(dynamic, 1)
        for (int64_t k = 0; k < (int64_t)roots.size(); ++k) {
            const uint32_t r = roots[k];
            weighted_one(o2.data(), a2.data(), reach.data(), r, mult[r], lvl.data(), sigma.data(), delta.data(),
                         queue.data(), acc, &overflow);
        }
    }
    // thread partials in thread order, then the tree terms
    for (uint32_t i = 0; i < nlive; ++i) {
        double s = 0.0;
        for (int k = 0; k < nt; ++k) s += part[(size_t)k * nlive + i];
        bc[ext[i]] += s;
    }
    std::vector<double> tacc;
    tree_bc(t, cnt, tacc);
    for (uint32_t v = 0; v < n; ++v) bc[v] += tacc[v];
    if (st) {
        st->skipped = skipped;
        st->roots = roots.size();
        st->teps_edges = teps;
        st->peel_seconds = std::chrono::duration<double>(t1 - t0).count();
        st->overflow = overflow;
    }
    return 0;
}
