// Host-side state of one graph on the device, shared by the engine's
// translation units (engine.cu: single graphs; batch.cu: packed unions of
// graphs).  Not part of the public ABI.
#pragma once
#include <vector>

#include "bcg.h"
#include "engine.cuh"

using bcg::Ctrl;
using bcg::kNoRoot;
using bcg::RootStat;
using bcg::Tile;
using bcg::kDefaultWaitNs;
using bcg::kTileEdges;
using bcg::kTileVerts;

namespace bcg {
// Pendant trees of a graph on the device (BCG_PRUNE_TREES, and one peeling
// round for BCG_PRUNE_DEGREE1; trees_gpu.cu), caller's numbering.
struct TreeDev {
    uint32_t *parent = nullptr;  // vertex it hung from when peeled; kNoRoot for kept vertices
    uint32_t *sz = nullptr;      // vertices in the subtree (a kept vertex: 1 + its trees)
    uint32_t *comp = nullptr;    // component of the input graph (a root's internal id)
    unsigned long long *comp_n = nullptr;  // vertices per component, indexed by root
    uint32_t *order = nullptr;   // peeled vertices, round by round
    uint32_t *anchor = nullptr;  // kept vertex a peeled vertex's tree hangs from (itself when kept)
    uint32_t *intl = nullptr;    // caller's id -> internal id of the searched graph
    uint32_t *cdeg = nullptr;    // degree in the kept graph
    std::vector<uint32_t> round_off;  // start of each round in order, and the end
    uint32_t npeeled = 0;
    // per-run scratch: the run's sources (uploaded by tree_source_info), their
    // planning words, and the closed-form tree terms
    uint32_t *cnt = nullptr, *src = nullptr;
    uint4 *info = nullptr;
    size_t src_cap = 0;
    uint64_t nsrc = 0;
    unsigned long long *sub = nullptr, *csrc = nullptr, *acc = nullptr;
};
}  // namespace bcg

struct bcg_graph {
    int device = 0;
    uint32_t n = 0;
    uint64_t nnz = 0, nnz_pruned = 0;
    uint32_t flags = 0;
    uint32_t npruned = 0;
    uint32_t *d_offs = nullptr, *d_adj = nullptr;
    uint2 *d_vinfo = nullptr;
    double *d_bc = nullptr;
    Tile *d_tiles = nullptr;
    uint32_t ntiles = 0, nhub = 0, nhubchunks = 0;
    unsigned long long *d_hub_acc = nullptr;
    unsigned int *d_hub_cnt = nullptr;
    uint32_t *d_tile_of = nullptr, *d_tmark = nullptr;
    uint32_t *d_lists = nullptr, *d_lbase = nullptr, *d_lcnt = nullptr;
    uint32_t *d_ulist = nullptr;  // ring of 2 * ntiles (tiles with unvisited vertices)
    unsigned long long list_cap = 0;
    unsigned char *d_rows = nullptr;  // n state rows of row_bytes(state_width)
    uint32_t state_width = 0;
    Ctrl *d_ctrl = nullptr;
    uint32_t *d_roots = nullptr, *d_pend = nullptr;
    double *d_mult = nullptr;
    RootStat *d_rstat = nullptr;
    size_t run_cap = 0;
    std::vector<uint32_t> h_deg;     // original degree (source skip test)
    uint32_t forced_width = 0;
    uint32_t tile_vcap = kTileVerts, tile_ecap = kTileEdges;  // tile shape (autotuned by batches)
    std::vector<uint32_t> tile_breaks;  // sorted vertices where a new tile must start
    float ratio = 0.2f;
    uint32_t mark_ratio = 8;  // child marks in backward sweeps (BatchArgs::mark_ratio)
    bool trees = false;               // pruned: pendant trees (or one layer) folded (tdev)
    bcg::TreeDev tdev;
    uint2 *d_vinfo_trees = nullptr;   // degree/reach words built by the peeling (until creation ends)
    int32_t *d_level_out = nullptr;   // depths exported by bcg_run_root_levels
    int32_t *d_slot_level = nullptr;  // depths exported by bcg_run_slots (width * n)
    size_t slot_level_cap = 0;
    // A pruned graph numbers the searched vertices internally: the vertices with
    // kept edges first (caller's order), then the rest, so the tiles cover
    // [0, tile_n) only.  tdev.intl: caller's id -> internal id; d_ext:
    // internal id -> caller's id, where the sweep adds each vertex's bc.
    uint32_t tile_n = 0;              // vertices covered by tiles (0: all n)
    uint32_t *d_ext = nullptr;
    int sigma_mode = 0;               // 0 auto (exact, extended on overflow), 1 exact only, 2 extended
    double *d_bc_save = nullptr;      // accumulators before an automatic-mode run
    unsigned long long wait_ns = kDefaultWaitNs;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace bcg {

// Device memory of graphs and of their creation, from a library-owned
// stream-ordered pool of the current device that keeps up to 1 GiB reserved
// once it is freed: creating and destroying graphs one after another then
// neither maps fresh memory nor waits in cudaFree.  tmp_alloc / tmp_free are
// ordered on stream st like a kernel; dev_alloc / dev_free on the default
// stream.  Whoever frees memory that work on another stream may still use
// synchronises the device first (graph_free and the reallocating paths do).
cudaError_t tmp_alloc(void **p, size_t bytes, cudaStream_t st);
cudaError_t tmp_free(void *p, cudaStream_t st);
template <class T>
cudaError_t tmp_alloc(T **p, size_t bytes, cudaStream_t st) {
    return tmp_alloc(reinterpret_cast<void **>(p), bytes, st);
}
template <class T>
cudaError_t dev_alloc(T **p, size_t bytes) {
    return tmp_alloc(reinterpret_cast<void **>(p), bytes, 0);
}
inline cudaError_t dev_free(void *p) { return tmp_free(p, 0); }

// ext: sigma and X as extended-range numbers (ext64.cuh) instead of uint64 / double
int launch_sweep(int S, const BatchArgs &a, cudaStream_t st, int *grid_out, bool ext = false);

// Component-packed batches already on the device (see BatchArgs::xbeg).
struct PackedRun {
    const uint32_t *xbeg, *xroots;
    const unsigned char *xslot;
    const unsigned long long *xpf, *xpu;
    const uint32_t *xtiles, *xrbeg;
    const uint2 *xrange;
    const bcg::SlotOut *xout;  // nullptr: dependencies into the union's bc
    double *slot_delta;        // with xout: S * n doubles of per-slot dependencies
    uint32_t nbatch;
    RootStat *rstat;  // nbatch * S per-slot totals
};

// Grows the state rows, hub accumulators and level lists for width S.
int ensure_state(bcg_graph *g, uint32_t S);
// Enqueues one packed launch on st (memsets + the sweep kernel; no host
// synchronisation, so it can be captured into a CUDA graph).
int enqueue_packed(bcg_graph *g, const PackedRun &p, uint32_t S, cudaStream_t st);
// Reads the control block after the stream has finished: error / overflow.
int check_ctrl(bcg_graph *g, cudaStream_t st);
// Rebuilds the work tiles with another shape (vcap vertices, ecap entries).
int graph_retile(bcg_graph *g, uint32_t vcap, uint32_t ecap, bool force = false);
// Peels the pendant trees of the input CSR (device arrays d_offs0 / d_adj0,
// nnz entries; check_ids: verify every id < n first; at most max_rounds
// peeling rounds, 1 for the one-layer mode) and builds g's kept
// graph in internal numbering (d_offs, d_adj, d_ext, tile_n, degree/reach
// words in d_vinfo_trees) and the tree arrays (tdev).  h_offs2: the kept
// graph's offsets.
int prepare_trees(bcg_graph *g, const uint32_t *d_offs0, const uint32_t *d_adj0, uint64_t nnz, bool check_ids,
                  uint32_t max_rounds, std::vector<uint32_t> &h_offs2);
// Uploads the k sources src (caller's ids, all < n) and reads back, per
// source s, {anchor a of s, kept degree of a, internal id of a, tree size of
// a}; the sources stay on the device for tree_terms.  Synchronises st.
int tree_source_info(bcg_graph *g, const uint32_t *src, uint64_t k, std::vector<uint4> &info, cudaStream_t st);
// Adds the closed-form betweenness of the tree vertices (and the anchors'
// tree terms) for the sources of the last tree_source_info call (duplicates
// count; sources of degree 0 add nothing) into g's bc, on stream st;
// *launches counts its kernels.
int tree_terms(bcg_graph *g, cudaStream_t st, uint64_t *launches);
void tree_free(bcg_graph *g);
// Uploads ngraphs host CSR graphs as one disjoint union (graph order[p] at
// union position p, its vertex v at base[order[p]] + v; with by_active the
// graphs with most non-isolated vertices come first).  hdeg: union degrees.
int make_union(uint32_t ngraphs, const uint32_t *const *offsets, const uint32_t *const *adj, const uint32_t *n,
               bool by_active, std::vector<uint32_t> &order, std::vector<uint32_t> &base,
               std::vector<uint32_t> &hdeg, bcg_graph **out);

}  // namespace bcg
