// ORACLE — test infrastructure only: host restatement of pendant-tree
// peeling and the closed-form tree terms (see trees_ref.cpp).
#pragma once
#include <cstdint>
#include <vector>

namespace oracle_trees {

constexpr uint32_t kNoRoot = 0xFFFFFFFFu;

struct TreeInfo {
    std::vector<uint32_t> parent;  // vertex it hung from when peeled; kNoRoot for kept (core) vertices
    std::vector<uint32_t> order;   // peeled vertices, in peeling order (children before parents)
    std::vector<uint32_t> sz;      // vertices in the subtree (a kept vertex: 1 + its trees)
    std::vector<uint32_t> anchor;  // the kept vertex a vertex's tree hangs from (itself if kept)
    std::vector<uint32_t> comp;    // connected component of the input graph
    std::vector<uint64_t> comp_n;  // vertices per component
};

// Peels every pendant tree; returns the kept graph renumbered so the vertices
// that keep an edge come first (ext[i] = id of internal vertex i, intl its
// inverse, offs2/adj2 the renumbered CSR, cdeg[v] = v's kept degree) and the
// number of vertices that keep an edge.
uint32_t peel_trees(const uint32_t *offs, const uint32_t *adj, uint32_t n, TreeInfo &t, std::vector<uint32_t> &cdeg,
                    std::vector<uint32_t> &ext, std::vector<uint32_t> &intl, std::vector<uint32_t> &offs2,
                    std::vector<uint32_t> &adj2);
// Components of every vertex from the kept graph's CSR (internal ids).
void label_components(const uint32_t *offs, const uint32_t *adj, uint32_t n, const std::vector<uint32_t> &intl,
                      TreeInfo &t);
// Closed-form bc of the tree vertices for the source multiplicities cnt[v].
void tree_bc(const TreeInfo &t, const std::vector<uint32_t> &cnt, std::vector<double> &acc);

}  // namespace oracle_trees
