// Graph handle, work tiles and the bcg_* C ABI.
//
// Reference counterparts:
//   initcuda / fincuda            cuda_kernels.cu:1123-1198, 1201-1232
//   degree_reduction              bc2d.c:314-419   (host qsort + merge, one layer)
//   init_bc_1degree(_device)      bc2d.c:455-465, cuda_kernels.cu:1083-1087
//   per-source loop + skip        bc2d.c:1016-1050
//   get_bc                        cuda_kernels.cu:1039-1041
//
// Pendant pruning (both flags) runs on the device in trees_gpu.cu:
// BCG_PRUNE_DEGREE1 is its first peeling round, which folds exactly the
// reference's layer: a vertex p of degree 1 whose neighbour a does not also
// have degree 1 is folded into a, and of an isolated edge {p, a} the larger
// id is folded into the smaller.  The kept graph is renumbered and searched
// with reach weights (init_delta, cuda_kernels.cu:1089-1098); the folded
// vertices' bc and the anchors' terms for their trees are added in closed
// form.  Unlike the reference, a vertex whose every neighbour was folded
// (isolated in the pruned graph) still gets its exact bc, and vertices
// outside a root's component get nothing from it (the reference adds
// reach * (reach_v0 + 1) to them, cuda_kernels.cu:274, 1095).
#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "bcg_common.hpp"
#include "engine.cuh"
#include "engine_internal.hpp"

namespace bcg {


#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return set_error(e_ == cudaErrorMemoryAllocation ? BCG_ERR_OOM : BCG_ERR_CUDA, \
                             "%s failed: %s", #call, cudaGetErrorString(e_));             \
    } while (0)

// ---------------------------------------------------------------------------
// Degree words of an unpruned graph.
// ---------------------------------------------------------------------------

__global__ void k_vinfo_plain(uint32_t n, const uint32_t *__restrict__ offs, uint2 *__restrict__ vinfo) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) vinfo[v] = make_uint2(offs[v + 1] - offs[v], 0u);
}

// ---------------------------------------------------------------------------
// Work tiles (host, from the original row starts).
// ---------------------------------------------------------------------------

// Runs of at most vcap consecutive vertices with at most ecap adjacency
// entries; a vertex with more than ecap entries is split into ecap-entry
// chunks (vcap <= 32, ecap <= kTileEdges: the sweep kernel's lane and
// staging limits).
// Only vertices [0, tn) get tiles.  A tile never spans a vertex listed in
// `breaks` (sorted) and the vertex before it.  tile_of[v] = index of v's tile (of its first chunk, with
// kHubFlag, when v is split).
static void build_tiles(const uint32_t *offs, uint32_t n, uint32_t tn, uint32_t vcap, uint32_t ecap,
                        const std::vector<uint32_t> &breaks, std::vector<Tile> &tiles, uint32_t &nhub,
                        uint32_t &nhubchunks, std::vector<uint32_t> &tile_of) {
    tiles.clear();
    tile_of.assign(n, 0);  // vertices past tn (no edges: never reached) keep tile 0
    n = tn;
    nhub = 0;
    nhubchunks = 0;
    uint32_t v = 0;
    size_t nb = 0;  // next break point
    while (v < n) {
        while (nb < breaks.size() && breaks[nb] <= v) ++nb;
        const uint32_t stop = nb < breaks.size() ? breaks[nb] : n;
        const uint32_t dv = offs[v + 1] - offs[v];
        if (dv > ecap) {
            const uint32_t nch = (dv + ecap - 1) / ecap;
            tile_of[v] = (uint32_t)tiles.size() | kHubFlag;
            for (uint32_t c = 0; c < nch; ++c) {
                Tile t{};
                t.v0 = v; t.v1 = v + 1;
                t.e0 = offs[v] + c * ecap;
                t.e1 = std::min(offs[v + 1], t.e0 + ecap);
                t.hub = (int32_t)nhub;
                t.nchunks = nch;
                t.hslot = nhubchunks++;
                t.hchunk = c;
                tiles.push_back(t);
            }
            ++nhub;
            ++v;
            continue;
        }
        const uint32_t start = v;
        uint32_t sum = 0;
        while (v < stop && v - start < vcap) {
            const uint32_t d = offs[v + 1] - offs[v];
            if (d > ecap || sum + d > ecap) break;
            sum += d;
            tile_of[v] = (uint32_t)tiles.size();
            ++v;
        }
        Tile t{};
        t.v0 = start; t.v1 = v;
        t.e0 = offs[start]; t.e1 = offs[v];
        t.hub = -1;
        t.nchunks = 1;
        tiles.push_back(t);
    }
}

}  // namespace bcg

using namespace bcg;


namespace bcg {

namespace {
std::mutex g_pool_mu;
std::vector<cudaMemPool_t> g_pools;  // per device, created on first use
}  // namespace

cudaError_t tmp_alloc(void **p, size_t bytes, cudaStream_t st) {
    *p = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (g_pools.size() <= (size_t)dev) g_pools.resize((size_t)dev + 1, nullptr);
        if (!g_pools[dev]) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if ((e = cudaMemPoolCreate(&g_pools[dev], &props)) != cudaSuccess) {
                g_pools[dev] = nullptr;
                return e;
            }
            uint64_t keep = 1ull << 30;
            cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = g_pools[dev];
    }
    return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 16), pool, st);
}

cudaError_t tmp_free(void *p, cudaStream_t st) { return p ? cudaFreeAsync(p, st) : cudaSuccess; }

static void graph_free(bcg_graph *g) {
    if (!g) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != g->device) cudaSetDevice(g->device);
    cudaDeviceSynchronize();  // work on any stream may still read the buffers
    dev_free(g->d_offs); dev_free(g->d_adj); dev_free(g->d_vinfo);
    dev_free(g->d_bc);
    dev_free(g->d_tiles); dev_free(g->d_hub_acc); dev_free(g->d_hub_cnt);
    dev_free(g->d_tile_of); dev_free(g->d_tmark); dev_free(g->d_lists);
    dev_free(g->d_lbase); dev_free(g->d_lcnt); dev_free(g->d_ulist); dev_free(g->d_bc_save);
    tree_free(g);
    dev_free(g->d_vinfo_trees);
    dev_free(g->d_level_out);
    dev_free(g->d_slot_level);
    dev_free(g->d_ext);
    dev_free(g->d_rows); dev_free(g->d_ctrl);
    dev_free(g->d_roots); dev_free(g->d_pend); dev_free(g->d_mult); dev_free(g->d_rstat);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (cur >= 0 && cur != g->device) cudaSetDevice(cur);
    delete g;
}

int ensure_state(bcg_graph *g, uint32_t S) {
    if (g->state_width >= S) return BCG_OK;  // row_bytes grows with S
    CK(cudaDeviceSynchronize());  // earlier runs (any stream) are done with the old buffers
    dev_free(g->d_rows); g->d_rows = nullptr;
    dev_free(g->d_hub_acc); g->d_hub_acc = nullptr;
    dev_free(g->d_lists); g->d_lists = nullptr;
    g->state_width = 0;
    CK(dev_alloc(&g->d_rows, (size_t)g->n * row_bytes((int)S)));
    // one slot per hub chunk, written by the chunk before it is read
    CK(dev_alloc(&g->d_hub_acc, (size_t)std::max(1u, g->nhubchunks) * S * sizeof(unsigned long long)));
    // every (tile, level) pair is listed at most once per batch: a tile is on
    // level d's list only if one of its vertices (or chunks) first reaches d,
    // so the lists of one batch hold at most S * (n + ntiles) entries
    g->list_cap = (unsigned long long)S * ((unsigned long long)g->n + g->ntiles);
    CK(dev_alloc(&g->d_lists, g->list_cap * sizeof(uint32_t)));
    CK(cudaDeviceSynchronize());  // the new buffers are ready for any stream
    g->state_width = S;
    return BCG_OK;
}

static int ensure_run(bcg_graph *g, size_t slots) {
    if (g->run_cap >= slots) return BCG_OK;
    CK(cudaDeviceSynchronize());
    dev_free(g->d_roots); dev_free(g->d_pend); dev_free(g->d_mult); dev_free(g->d_rstat);
    g->d_roots = g->d_pend = nullptr; g->d_mult = nullptr; g->d_rstat = nullptr;
    g->run_cap = 0;
    size_t cap = std::max<size_t>(slots, 64);
    CK(dev_alloc(&g->d_roots, cap * sizeof(uint32_t)));
    CK(dev_alloc(&g->d_pend, cap * sizeof(uint32_t)));
    CK(dev_alloc(&g->d_mult, cap * sizeof(double)));
    CK(dev_alloc(&g->d_rstat, cap * sizeof(RootStat)));
    CK(cudaDeviceSynchronize());
    g->run_cap = cap;
    return BCG_OK;
}

// Sources per batch: the widest S in {6, 3, 1} whose state rows (one per
// searched vertex, row_bytes(S) each) fit the budget that keeps them
// L2-resident, and not wider than the number of roots needs.
static uint32_t choose_width(const bcg_graph *g, uint64_t nroots) {
    if (g->forced_width) return g->forced_width;
    double budget = 64.0 * 1024 * 1024;
    if (const char *e = getenv("BCG_STATE_BUDGET_MB")) budget = atof(e) * 1024 * 1024;
    const double nrows = g->tile_n ? g->tile_n : g->n;  // a pruned graph searches the kept vertices only
    // low-degree graphs (mean degree below 6: grids, meshes, long chains) have
    // small frontiers and many levels, so sweeps cost barriers, not gathers,
    // and the widest batch wins whether or not the rows fit L2 (measured on a
    // 2048 x 2048 grid: 0.11 / 0.20 / 0.22 G TEPS at widths 1 / 3 / 6)
    if ((double)g->nnz_pruned < 6.0 * nrows) budget = 1e30;
    uint32_t S = 6;
    if (nrows * row_bytes(6) > budget || nroots <= 3) S = 3;
    if (S == 3 && (nrows * row_bytes(3) > budget || nroots <= 1)) S = 1;
    return S;
}

// Work tiles of the current shape and the per-tile buffers.
static int setup_tiles(bcg_graph *g, const uint32_t *h_offs) {
    const uint32_t n = g->n;
    std::vector<Tile> tiles;
    std::vector<uint32_t> tile_of;
    build_tiles(h_offs, n, g->tile_n ? g->tile_n : n, g->tile_vcap, g->tile_ecap, g->tile_breaks, tiles, g->nhub,
                g->nhubchunks, tile_of);
    g->ntiles = (uint32_t)tiles.size();
    CK(dev_alloc(&g->d_tiles, std::max<size_t>(1, tiles.size()) * sizeof(Tile)));
    if (!tiles.empty())
        CK(cudaMemcpy(g->d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice));
    CK(dev_alloc(&g->d_tile_of, (size_t)n * sizeof(uint32_t)));
    CK(cudaMemcpy(g->d_tile_of, tile_of.data(), (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CK(dev_alloc(&g->d_tmark, std::max<size_t>(1, tiles.size()) * sizeof(uint32_t)));
    CK(dev_alloc(&g->d_ulist, 2 * std::max<size_t>(1, tiles.size()) * sizeof(uint32_t)));
    CK(dev_alloc(&g->d_hub_cnt, (size_t)std::max(1u, g->nhub) * sizeof(unsigned int)));
    CK(cudaMemset(g->d_hub_cnt, 0, (size_t)std::max(1u, g->nhub) * sizeof(unsigned int)));
    CK(cudaDeviceSynchronize());  // the new buffers are ready for any stream
    return BCG_OK;
}

// h_offs: offsets of the searched graph (tiles); h_offs_in: of the input
// graph (the degree-0 source skip test).
static int create_common(bcg_graph *g, const uint32_t *h_offs, const uint32_t *h_offs_in) {
    const uint32_t n = g->n;
    // 4 entries of tail padding (the sweep copies 16-byte aligned ranges)
    CK(dev_alloc(&g->d_vinfo, ((size_t)n + 4) * sizeof(uint2)));
    CK(cudaMemset(g->d_vinfo, 0, ((size_t)n + 4) * sizeof(uint2)));
    CK(dev_alloc(&g->d_bc, (size_t)n * sizeof(double)));
    CK(cudaMemset(g->d_bc, 0, (size_t)n * sizeof(double)));
    CK(dev_alloc(&g->d_ctrl, sizeof(Ctrl)));
    CK(cudaEventCreate(&g->ev0));
    CK(cudaEventCreate(&g->ev1));
    g->h_deg.resize(n);
    uint32_t *hd = g->h_deg.data();
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)n; ++v) hd[v] = h_offs_in[v + 1] - h_offs_in[v];
    // a pruned graph's degree words come from the peeling (graph_create_impl
    // copies them over these)
    k_vinfo_plain<<<(n + 255) / 256, 256>>>(n, g->d_offs, g->d_vinfo);
    CK(cudaGetLastError());
    g->nnz_pruned = g->nnz;
    CK(dev_alloc(&g->d_lbase, (size_t)(kMaxLevel + 3) * sizeof(uint32_t)));
    CK(dev_alloc(&g->d_lcnt, (size_t)(kMaxLevel + 3) * sizeof(uint32_t)));
    const int rc = setup_tiles(g, h_offs);
    if (rc) return rc;
    CK(cudaDeviceSynchronize());
    return BCG_OK;
}

int graph_retile(bcg_graph *g, uint32_t vcap, uint32_t ecap, bool force) {
    if (vcap < 1 || vcap > (uint32_t)kTileVerts || ecap < 1 || ecap > (uint32_t)kTileEdges)
        return set_error(BCG_ERR_ARG, "tile shape %ux%u outside 1..%d vertices, 1..%d entries", vcap, ecap,
                         kTileVerts, kTileEdges);
    if (!force && vcap == g->tile_vcap && ecap == g->tile_ecap) return BCG_OK;
    std::vector<uint32_t> h_offs((size_t)g->n + 1);
    CK(cudaMemcpy(h_offs.data(), g->d_offs, h_offs.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    CK(cudaDeviceSynchronize());
    dev_free(g->d_tiles); dev_free(g->d_tile_of); dev_free(g->d_tmark); dev_free(g->d_ulist);
    dev_free(g->d_hub_cnt); dev_free(g->d_hub_acc); dev_free(g->d_lists);
    g->d_tiles = nullptr; g->d_tile_of = g->d_tmark = g->d_ulist = g->d_lists = nullptr;
    g->d_hub_cnt = nullptr; g->d_hub_acc = nullptr;
    g->state_width = 0;  // hub accumulators and lists are sized by the tiles
    g->tile_vcap = vcap;
    g->tile_ecap = ecap;
    return setup_tiles(g, h_offs.data());
}

static int check_device() {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_error(BCG_ERR_NOGPU, "no CUDA device: %s", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
    return BCG_OK;
}

static int validate_csr(const uint32_t *offs, const uint32_t *adj, uint32_t n, uint64_t nnz) {
    if (offs[0] != 0 || offs[n] != nnz) return set_error(BCG_ERR_ARG, "offsets[0] must be 0 and offsets[n] == nnz");
    uint64_t bad_offs = 0, bad_adj = 0;
#pragma omp parallel for reduction(+ : bad_offs) schedule(static)
    for (int64_t v = 0; v < (int64_t)n; ++v) bad_offs += offs[v + 1] < offs[v];
#pragma omp parallel for reduction(+ : bad_adj) schedule(static)
    for (int64_t e = 0; e < (int64_t)nnz; ++e) bad_adj += adj[e] >= n;
    if (bad_offs)
        for (uint32_t v = 0; v < n; ++v)
            if (offs[v + 1] < offs[v]) return set_error(BCG_ERR_ARG, "offsets not non-decreasing at %u", v);
    if (bad_adj)
        for (uint64_t e = 0; e < nnz; ++e)
            if (adj[e] >= n) return set_error(BCG_ERR_ARG, "adj[%" PRIu64 "] = %u >= n", e, adj[e]);
    return BCG_OK;
}

struct RunPlan {
    std::vector<uint32_t> roots, pend;
    std::vector<double> mult;
    std::vector<uint64_t> count;  // sources mapped to each root
    uint64_t skipped = 0;
    // pruned: sources in components that are trees (no search needed)
    uint64_t tree_only = 0, tree_edges = 0, tree_verts = 0;
    uint64_t launches = 0;  // kernels the planning launched (the source gather)
};

// A pruned graph: the closed-form bc of the tree vertices (and the anchors' tree
// terms) for this run's sources, added on the device after the search.
static int add_tree_terms(bcg_graph *g, const RunPlan &p, cudaStream_t st, bcg_stats *stats) {
    uint64_t nl = 0;
    const int rc = tree_terms(g, st, &nl);
    if (rc) return rc;
    if (stats) {
        stats->teps_edges += p.tree_edges;
        stats->comp_vertices += p.tree_verts;
        stats->launches += nl;
    }
    return BCG_OK;
}

// A pruned graph reads each source's anchor words from the device first
// (tree_source_info on stream st), which also leaves the sources there for
// the tree terms.
static int plan_run(bcg_graph *g, const uint32_t *src, uint64_t nsrc, RunPlan &p, cudaStream_t st) {
    for (uint64_t i = 0; i < nsrc; ++i)
        if (src[i] >= g->n) return set_error(BCG_ERR_ARG, "source %u >= n=%u", src[i], g->n);
    std::vector<uint4> info;
    if (g->trees) {
        const int rc = tree_source_info(g, src, nsrc, info, st);
        if (rc) return rc;
        if (nsrc) p.launches += 1;
    }
    std::unordered_map<uint32_t, uint32_t> idx;
    idx.reserve(nsrc * 2 + 1);
    for (uint64_t i = 0; i < nsrc; ++i) {
        const uint32_t s = src[i];
        if (g->h_deg[s] == 0) { ++p.skipped; continue; }
        uint32_t r = s, root = s;
        if (g->trees) {
            const uint4 w = info[i];  // {anchor, its kept degree, internal id, tree size}
            if (w.y == 0) {
                // a tree component: no kept edges, its bc is all in the tree
                // terms (the kept vertex is the last one of its tree: its
                // tree size is the component)
                ++p.tree_only;
                p.tree_edges += w.w - 1;
                p.tree_verts += w.w;
                continue;
            }
            r = w.x;
            root = w.z;
        }
        auto it = idx.find(r);
        uint32_t k;
        if (it == idx.end()) {
            k = (uint32_t)p.roots.size();
            idx.emplace(r, k);
            p.roots.push_back(root);
            p.pend.push_back(0);
            p.mult.push_back(0.0);
            p.count.push_back(0);
        } else {
            k = it->second;
        }
        p.mult[k] += 1.0;
        p.count[k] += 1;
    }
    return BCG_OK;
}

// BatchArgs fields common to every launch on g.
static void fill_args(bcg_graph *g, BatchArgs &a) {
    a.n = g->tile_n ? g->tile_n : g->n;
    a.ext = g->d_ext;
    a.offs = g->d_offs;
    a.adj = g->d_adj;
    a.vinfo = g->d_vinfo;
    a.tiles = g->d_tiles;
    a.ntiles = g->ntiles;
    a.tile_of = g->d_tile_of;
    a.tmark = g->d_tmark;
    a.lists = g->d_lists;
    a.list_cap = g->list_cap;
    a.ulist = g->d_ulist;
    a.lbase = g->d_lbase;
    a.lcnt = g->d_lcnt;
    a.rows = g->d_rows;
    a.bc = g->d_bc;
    a.hub_acc = g->d_hub_acc;
    a.hub_cnt = g->d_hub_cnt;
    a.ctrl = g->d_ctrl;
    a.nnz = g->nnz_pruned;
    a.push_pull_ratio = g->ratio;
    a.mark_ratio = g->mark_ratio;
    a.directed = (g->flags & BCG_DIRECTED) ? 1 : 0;
}

// Debug outputs of a run (internal numbering; slot k of batch b at
// (b * width + k) * n): width = the run's batch width.
struct DebugOut {
    uint32_t width = 0;  // 0: not a debug run
    int32_t *level = nullptr;
    unsigned long long *sigma = nullptr;
    double *delta = nullptr;
};

// rs_out (with stats): every root's own totals, in plan order.
static int run_plan(bcg_graph *g, const RunPlan &p, cudaStream_t st, bcg_stats *stats, const DebugOut &dbg,
                    std::vector<RootStat> *rs_out = nullptr) {
    const bool debug = dbg.width != 0;
    const uint64_t nroots = p.roots.size();
    if (stats) {
        stats->skipped = p.skipped;
        stats->roots = nroots;
        stats->launches = p.launches;
    }
    if (nroots == 0) return BCG_OK;
    const uint32_t S = debug ? dbg.width : choose_width(g, nroots);
    int rc = ensure_state(g, S);
    if (rc) return rc;
    const uint64_t nbatch = (nroots + S - 1) / S;
    const size_t slots = nbatch * S;
    rc = ensure_run(g, slots);
    if (rc) return rc;
    std::vector<uint32_t> roots(slots, kNoRoot), pend(slots, 0);
    std::vector<double> mult(slots, 0.0);
    for (uint64_t i = 0; i < nroots; ++i) { roots[i] = p.roots[i]; pend[i] = p.pend[i]; mult[i] = p.mult[i]; }
    CK(cudaMemcpyAsync(g->d_roots, roots.data(), slots * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(g->d_pend, pend.data(), slots * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(g->d_mult, mult.data(), slots * sizeof(double), cudaMemcpyHostToDevice, st));
    BatchArgs a{};
    fill_args(g, a);
    a.dbg_level = dbg.level;
    a.dbg_sigma = dbg.sigma;
    a.dbg_delta = dbg.delta;
    // optional per-sweep trace: BCG_TRACE_FILE=<path> appends one CSV line per
    // sweep (batch, kind, level, tiles walked, pairs discovered, end time)
    const char *trace_path = getenv("BCG_TRACE_FILE");
    TraceRec *d_trace = nullptr;
    unsigned int *d_tcnt = nullptr;
    const unsigned int trace_cap = 1u << 20;
    if (trace_path && *trace_path) {
        CK(dev_alloc(&d_trace, trace_cap * sizeof(TraceRec)));
        CK(dev_alloc(&d_tcnt, sizeof(unsigned int)));
        CK(cudaMemsetAsync(d_tcnt, 0, sizeof(unsigned int), st));
        a.trace = d_trace;
        a.trace_cap = trace_cap;
        a.trace_cnt = d_tcnt;
    }
    // Sigma is exact uint64 unless the graph runs in extended mode; in the
    // automatic mode a run whose counts overflow is redone in extended mode
    // from a saved copy of the accumulators.
    const bool autoext = g->sigma_mode == 0;
    bool ext = g->sigma_mode == 2;
    if (autoext) {
        if (!g->d_bc_save) CK(dev_alloc(&g->d_bc_save, (size_t)g->n * sizeof(double)));
        CK(cudaMemcpyAsync(g->d_bc_save, g->d_bc, (size_t)g->n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    for (;;) {
        CK(cudaEventRecord(g->ev0, st));
        // tile marks key on the batch index modulo 2^16, so one launch runs at
        // most 65535 batches and the marks are cleared before every launch
        const uint64_t per_launch = 65535;
        for (uint64_t b0 = 0; b0 < nbatch; b0 += per_launch) {
            const uint64_t nb = std::min(per_launch, nbatch - b0);
            CK(cudaMemsetAsync(g->d_ctrl, 0, sizeof(Ctrl), st));
            CK(cudaMemcpyAsync(&g->d_ctrl->wait_ns, &g->wait_ns, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                               st));
            CK(cudaMemsetAsync(g->d_tmark, 0, (size_t)std::max(1u, g->ntiles) * sizeof(uint32_t), st));
            CK(cudaMemsetAsync(g->d_hub_cnt, 0, (size_t)std::max(1u, g->nhub) * sizeof(unsigned int), st));
            a.roots = g->d_roots + b0 * S;
            a.mult = g->d_mult + b0 * S;
            a.pend = g->d_pend + b0 * S;
            a.rstat = g->d_rstat + b0 * S;
            // debug outputs: slot k of batch b at ((b * S) + k) * n
            const size_t dofs = (size_t)b0 * S * a.n;
            a.dbg_level = dbg.level ? dbg.level + dofs : nullptr;
            a.dbg_sigma = dbg.sigma ? dbg.sigma + dofs : nullptr;
            a.dbg_delta = dbg.delta ? dbg.delta + dofs : nullptr;
            a.nbatch = (uint32_t)nb;
            int grid = 0;
            rc = launch_sweep((int)S, a, st, &grid, ext);
            if (rc) return rc;
            if (stats) ++stats->launches;
            if (b0 + nb < nbatch) {
                // errors of this launch are read before the control block is reused
                CK(cudaStreamSynchronize(st));
                Ctrl c{};
                CK(cudaMemcpy(&c, g->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
                if (c.error || c.overflow) break;
            }
        }
        CK(cudaEventRecord(g->ev1, st));
        if (d_trace) {
            CK(cudaStreamSynchronize(st));
            unsigned int cnt = 0;
            CK(cudaMemcpy(&cnt, d_tcnt, sizeof(cnt), cudaMemcpyDeviceToHost));
            std::vector<TraceRec> recs(cnt);
            if (cnt) CK(cudaMemcpy(recs.data(), d_trace, cnt * sizeof(TraceRec), cudaMemcpyDeviceToHost));
            CK(cudaMemsetAsync(d_tcnt, 0, sizeof(unsigned int), st));
            if (FILE *f = fopen(trace_path, "a")) {
                fprintf(f, "# width %u roots %zu tiles %u\n", S, (size_t)nroots, g->ntiles);
                for (const TraceRec &r : recs)
                    fprintf(f, "%u,%u,%u,%u,%llu,%llu\n", r.batch, r.kind, r.level, r.nwork, r.disc, r.t_ns);
                fclose(f);
            }
        }
        if (!stats && !debug && !autoext) break;
        CK(cudaStreamSynchronize(st));
        Ctrl c{};
        CK(cudaMemcpy(&c, g->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
        if (c.error && c.error != BCG_ERR_OVERFLOW) {
            dev_free(d_trace);
            dev_free(d_tcnt);
            return set_error(c.error, "device reported error %d (%s)", c.error,
                             c.error == BCG_ERR_TIMEOUT ? "a bounded wait gave up" : "level limit exceeded");
        }
        if (c.overflow || c.error == BCG_ERR_OVERFLOW) {
            if (autoext && !ext) {
                CK(cudaMemcpyAsync(g->d_bc, g->d_bc_save, (size_t)g->n * sizeof(double), cudaMemcpyDeviceToDevice,
                                   st));
                ext = true;
                continue;
            }
            dev_free(d_trace);
            dev_free(d_tcnt);
            return set_error(BCG_ERR_OVERFLOW, "a shortest-path count exceeded 2^64");
        }
        break;
    }
    dev_free(d_trace);
    dev_free(d_tcnt);
    if (!stats) return BCG_OK;
    if (stats) {
        std::vector<RootStat> rs(slots);
        CK(cudaMemcpy(rs.data(), g->d_rstat, slots * sizeof(RootStat), cudaMemcpyDeviceToHost));
        if (rs_out) rs_out->assign(rs.begin(), rs.begin() + nroots);
        uint64_t teps = 0, vis = 0, cv = 0, se = 0;
        uint32_t md = 0;
        for (uint64_t i = 0; i < nroots; ++i) {
            teps += p.count[i] * (rs[i].mc2 / 2);
            cv += p.count[i] * rs[i].wsum;
            vis += rs[i].visited;
            // mc2 = sum of (deg + 2 reach) and wsum = sum of (1 + reach) over
            // the visited vertices: the searched degrees sum to mc2 - 2 (wsum - visited)
            se += (rs[i].mc2 - 2 * (rs[i].wsum - rs[i].visited)) / 2;
            md = std::max(md, rs[i].depth);
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, g->ev0, g->ev1);
        stats->batches = nbatch;
        stats->teps_edges = teps;
        stats->visited = vis;
        stats->comp_vertices = cv;
        stats->max_depth = md;
        stats->batch_width = S;
        stats->kernel_ms = ms;
        stats->extended_sigma = ext ? 1u : 0u;
        stats->search_edges = se;
    }
    return BCG_OK;
}

int enqueue_packed(bcg_graph *g, const PackedRun &p, uint32_t S, cudaStream_t st) {
    if (p.nbatch == 0) return BCG_OK;
    // tile marks key on the batch index modulo 2^16 (one launch, <= 65535 batches)
    if (p.nbatch > 65535) return set_error(BCG_ERR_RANGE, "%u packed batches exceed one launch (65535)", p.nbatch);
    int rc = ensure_state(g, S);
    if (rc) return rc;
    const size_t nh = std::max(1u, g->nhub);
    CK(cudaMemsetAsync(g->d_hub_cnt, 0, nh * sizeof(unsigned int), st));
    CK(cudaMemsetAsync(g->d_ctrl, 0, sizeof(Ctrl), st));  // wait bound 0: the kernel's default
    CK(cudaMemsetAsync(g->d_tmark, 0, (size_t)std::max(1u, g->ntiles) * sizeof(uint32_t), st));
    BatchArgs a{};
    fill_args(g, a);
    a.rstat = p.rstat;
    a.nbatch = p.nbatch;
    a.xbeg = p.xbeg;
    a.xroots = p.xroots;
    a.xslot = p.xslot;
    a.xpf = p.xpf;
    a.xpu = p.xpu;
    a.xtiles = p.xtiles;
    a.xrbeg = p.xrbeg;
    a.xrange = p.xrange;
    a.xout = p.xout;
    a.slot_delta = p.xout ? p.slot_delta : nullptr;
    int grid = 0;
    return launch_sweep((int)S, a, st, &grid);
}

int check_ctrl(bcg_graph *g, cudaStream_t st) {
    CK(cudaStreamSynchronize(st));
    Ctrl c{};
    CK(cudaMemcpy(&c, g->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    if (c.overflow || c.error == BCG_ERR_OVERFLOW)
        return set_error(BCG_ERR_OVERFLOW, "a shortest-path count exceeded 2^64");
    if (c.error) return set_error(c.error, "device reported error %d (%s)", c.error,
                                  c.error == BCG_ERR_TIMEOUT ? "a bounded wait gave up" : "level limit exceeded");
    return BCG_OK;
}

}  // namespace bcg

extern "C" {

int bcg_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

static int graph_create_impl(const uint32_t *offsets, const uint32_t *adj, uint32_t n, uint64_t nnz,
                             uint32_t flags, bool device_in, bcg_graph **out) {
    clear_error();
    if (!out) return set_error(BCG_ERR_ARG, "null output handle");
    *out = nullptr;
    if (!offsets || (nnz && !adj) || n == 0) return set_error(BCG_ERR_ARG, "null CSR or n == 0");
    if (nnz > 0xFFFFFFFFull || n > 0xFFFFFFFEu) return set_error(BCG_ERR_RANGE, "graph exceeds 32-bit ids/offsets");
    int rc = check_device();
    if (rc) return rc;
    std::vector<uint32_t> h_offs;
    const uint32_t *ho = offsets;
    if (device_in) {
        h_offs.resize((size_t)n + 1);
        cudaError_t e = cudaMemcpy(h_offs.data(), offsets, ((size_t)n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return set_error(BCG_ERR_CUDA, "reading offsets: %s", cudaGetErrorString(e));
        ho = h_offs.data();
        if (ho[0] != 0 || ho[n] != nnz) return set_error(BCG_ERR_ARG, "offsets[0] must be 0 and offsets[n] == nnz");
        for (uint32_t v = 0; v < n; ++v)
            if (ho[v + 1] < ho[v]) return set_error(BCG_ERR_ARG, "offsets not non-decreasing at %u", v);
    } else {
        rc = validate_csr(offsets, adj, n, nnz);
        if (rc) return rc;
    }
    // pendant pruning: the device peels the trees (BCG_PRUNE_TREES) or one
    // layer of degree-1 vertices (BCG_PRUNE_DEGREE1: one peeling round) and
    // keeps the kept graph only, renumbered
    const bool trees = (flags & (BCG_PRUNE_TREES | BCG_PRUNE_DEGREE1)) && !(flags & BCG_DIRECTED);
    const uint32_t max_rounds = (flags & BCG_PRUNE_TREES) ? 0xFFFFFFFFu : 1u;
    if (flags & BCG_PRUNE_TREES) flags &= ~BCG_PRUNE_DEGREE1;
    bcg_graph *g = new bcg_graph();
    cudaGetDevice(&g->device);
    g->n = n;
    g->nnz = nnz;
    g->flags = flags;
    if (const char *e = getenv("BCG_PUSH_PULL_RATIO")) g->ratio = (float)atof(e);
    if (const char *e = getenv("BCG_CHILD_MARK_RATIO")) g->mark_ratio = (uint32_t)std::min(strtoul(e, nullptr, 10), 1024ul);
    if (const char *e = getenv("BCG_TILE_SHAPE")) {  // "<vertices>x<entries>", e.g. 32x128
        unsigned tv = 0, te = 0;
        if (sscanf(e, "%ux%u", &tv, &te) == 2 && tv >= 1 && tv <= (unsigned)kTileVerts && te >= 1 &&
            te <= (unsigned)kTileEdges) {
            g->tile_vcap = tv;
            g->tile_ecap = te;
        }
    }
    auto fail = [&](int code) { graph_free(g); return code; };
    cudaError_t e;
    std::vector<uint32_t> h_offs2;
    if (trees) {
        // the input CSR on the device (a temporary copy for host input)
        const uint32_t *d_offs0 = offsets, *d_adj0 = adj;
        uint32_t *t_offs = nullptr, *t_adj = nullptr;
        auto drop = [&]() { tmp_free(t_offs, 0); tmp_free(t_adj, 0); };
        if (!device_in) {
            if ((e = tmp_alloc(&t_offs, ((size_t)n + 1) * sizeof(uint32_t), 0)) != cudaSuccess ||
                (e = tmp_alloc(&t_adj, std::max<uint64_t>(nnz, 1) * sizeof(uint32_t), 0)) != cudaSuccess ||
                (e = cudaMemcpy(t_offs, offsets, ((size_t)n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice)) !=
                    cudaSuccess ||
                (nnz && (e = cudaMemcpy(t_adj, adj, nnz * sizeof(uint32_t), cudaMemcpyHostToDevice)) != cudaSuccess)) {
                drop();
                return fail(set_error(e == cudaErrorMemoryAllocation ? BCG_ERR_OOM : BCG_ERR_CUDA,
                                      "uploading CSR: %s", cudaGetErrorString(e)));
            }
            d_offs0 = t_offs;
            d_adj0 = t_adj;
        }
        rc = prepare_trees(g, d_offs0, d_adj0, nnz, device_in, max_rounds, h_offs2);
        drop();
        if (rc) return fail(rc);
        g->nnz = h_offs2[n];  // kept entries, while the common setup runs
    } else {
        // 4 entries of tail padding on offsets and adjacency: the sweep copies
        // their ranges in 16-byte aligned pieces that may end up to 12 bytes
        // past the last entry
        if ((e = dev_alloc(&g->d_offs, ((size_t)n + 1 + 4) * sizeof(uint32_t))) != cudaSuccess ||
            (e = dev_alloc(&g->d_adj, (nnz + 4) * sizeof(uint32_t))) != cudaSuccess)
            return fail(set_error(BCG_ERR_OOM, "cudaMalloc CSR: %s", cudaGetErrorString(e)));
        const cudaMemcpyKind kind = device_in ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if ((e = cudaMemcpy(g->d_offs, offsets, ((size_t)n + 1) * sizeof(uint32_t), kind)) != cudaSuccess ||
            (e = cudaMemset(g->d_offs + n + 1, 0, 4 * sizeof(uint32_t))) != cudaSuccess ||
            (nnz && (e = cudaMemcpy(g->d_adj, adj, nnz * sizeof(uint32_t), kind)) != cudaSuccess) ||
            (e = cudaMemset(g->d_adj + nnz, 0, 4 * sizeof(uint32_t))) != cudaSuccess)
            return fail(set_error(BCG_ERR_CUDA, "uploading CSR: %s", cudaGetErrorString(e)));
    }
    rc = create_common(g, trees ? h_offs2.data() : ho, ho);
    if (rc) return fail(rc);
    if (trees) {
        // kept-graph degrees and tree weights (reach) for the searches
        g->trees = true;
        g->nnz = nnz;
        if ((e = cudaMemcpy(g->d_vinfo, g->d_vinfo_trees, (size_t)n * sizeof(uint2), cudaMemcpyDeviceToDevice)) !=
            cudaSuccess)
            return fail(set_error(BCG_ERR_CUDA, "tree weights: %s", cudaGetErrorString(e)));
        dev_free(g->d_vinfo_trees);
        g->d_vinfo_trees = nullptr;
    }
    *out = g;
    return BCG_OK;
}

int bcg_graph_create(const uint32_t *offsets, const uint32_t *adj, uint32_t n, uint64_t nnz, uint32_t flags,
                     bcg_graph **out) {
    return graph_create_impl(offsets, adj, n, nnz, flags, false, out);
}

int bcg_graph_create_device(const uint32_t *d_offsets, const uint32_t *d_adj, uint32_t n, uint64_t nnz,
                            uint32_t flags, bcg_graph **out) {
    return graph_create_impl(d_offsets, d_adj, n, nnz, flags, true, out);
}

int bcg_graph_destroy(bcg_graph *g) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    graph_free(g);
    return BCG_OK;
}

int bcg_reset_bc(bcg_graph *g) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    CK(cudaMemset(g->d_bc, 0, (size_t)g->n * sizeof(double)));
    return BCG_OK;
}

int bcg_run(bcg_graph *g, const uint32_t *sources, uint64_t nsrc, bcg_stats *stats) {
    clear_error();
    if (!g || (nsrc && !sources)) return set_error(BCG_ERR_ARG, "null argument");
    bcg_stats local{};
    bcg_stats *st = stats ? stats : &local;
    *st = bcg_stats{};
    st->sources = nsrc;
    RunPlan p;
    int rc = plan_run(g, sources, nsrc, p, 0);
    if (rc) return rc;
    rc = run_plan(g, p, 0, st, DebugOut{});
    if (rc || !g->trees) return rc;
    return add_tree_terms(g, p, 0, st);
}

int bcg_run_device(bcg_graph *g, const uint32_t *d_sources, uint64_t nsrc, void *stream, bcg_stats *stats) {
    clear_error();
    if (!g || (nsrc && !d_sources)) return set_error(BCG_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<uint32_t> h(nsrc);
    if (nsrc) {
        CK(cudaMemcpyAsync(h.data(), d_sources, nsrc * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    if (stats) { *stats = bcg_stats{}; stats->sources = nsrc; }
    RunPlan p;
    int rc = plan_run(g, h.data(), nsrc, p, st);
    if (rc) return rc;
    rc = run_plan(g, p, st, stats, DebugOut{});
    if (rc || !g->trees) return rc;
    return add_tree_terms(g, p, st, stats);
}

int bcg_get_bc(bcg_graph *g, double *bc_host) {
    clear_error();
    if (!g || !bc_host) return set_error(BCG_ERR_ARG, "null argument");
    CK(cudaMemcpy(bc_host, g->d_bc, (size_t)g->n * sizeof(double), cudaMemcpyDeviceToHost));
    return BCG_OK;
}

int bcg_bc_device_ptr(bcg_graph *g, double **d_bc) {
    clear_error();
    if (!g || !d_bc) return set_error(BCG_ERR_ARG, "null argument");
    *d_bc = g->d_bc;
    return BCG_OK;
}

int bcg_bc_csr(const uint32_t *offsets, const uint32_t *adj, uint32_t n, uint64_t nnz, const uint32_t *sources,
               uint64_t nsrc, uint32_t flags, double *bc_out, bcg_stats *stats) {
    clear_error();
    if (!bc_out) return set_error(BCG_ERR_ARG, "null bc_out");
    bcg_graph *g = nullptr;
    int rc = bcg_graph_create(offsets, adj, n, nnz, flags, &g);
    if (rc) return rc;
    rc = bcg_run(g, sources, nsrc, stats);
    if (!rc) rc = bcg_get_bc(g, bc_out);
    graph_free(g);
    return rc;
}

// One batch of up to `width` roots (caller's ids) run in debug mode: every
// slot's levels and sigma after the forward pass and delta after the
// backward pass, copied out slot-major in the caller's numbering (nroots * n
// values each; vertices the search does not hold, i.e. the folded vertices
// of a pruned graph, read level -1, sigma 0, delta 0).  The bc
// accumulator is saved and restored around the run.
static int debug_batch_impl(bcg_graph *g, uint32_t width, const uint32_t *roots, uint32_t nroots, int32_t *level,
                            uint64_t *sigma, double *delta) {
    if (!g || (nroots && !roots)) return set_error(BCG_ERR_ARG, "null argument");
    if (width != 1 && width != 3 && width != 6) return set_error(BCG_ERR_ARG, "batch width %u not in {1,3,6}", width);
    if (nroots == 0 || nroots > width) return set_error(BCG_ERR_ARG, "%u roots for a batch of width %u", nroots, width);
    const size_t n = g->n;
    const size_t ns = g->tile_n ? g->tile_n : g->n;  // searched vertices (the kernel's stride)
    RunPlan p;
    for (uint32_t k = 0; k < nroots; ++k)
        if (roots[k] >= g->n) return set_error(BCG_ERR_ARG, "root %u >= n=%u", roots[k], g->n);
    std::vector<uint4> info;
    std::vector<uint32_t> intl;  // pruned: caller's id -> internal id
    if (g->trees) {
        int rc = tree_source_info(g, roots, nroots, info, 0);
        if (rc) return rc;
        intl.resize(n);
        CK(cudaMemcpy(intl.data(), g->tdev.intl, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    for (uint32_t k = 0; k < nroots; ++k) {
        const uint32_t r = roots[k];
        const uint32_t ri = g->trees ? info[k].z : r;
        if (g->trees && (info[k].x != r || info[k].y == 0 || ri >= ns))
            return set_error(BCG_ERR_ARG, "root %u is not searched: it lies in a pendant tree or has no kept edge", r);
        p.roots.push_back(ri);
        p.pend.push_back(0);
        p.mult.push_back(1.0);
        p.count.push_back(1);
    }
    const size_t cells = ns * width;
    double *d_save = nullptr;
    unsigned long long *d_sig = nullptr;
    double *d_del = nullptr;
    int32_t *d_lvl = nullptr;
    auto cleanup = [&]() { dev_free(d_save); dev_free(d_sig); dev_free(d_del); dev_free(d_lvl); };
    if (dev_alloc(&d_save, n * sizeof(double)) != cudaSuccess ||
        dev_alloc(&d_sig, cells * sizeof(unsigned long long)) != cudaSuccess ||
        dev_alloc(&d_del, cells * sizeof(double)) != cudaSuccess ||
        dev_alloc(&d_lvl, cells * sizeof(int32_t)) != cudaSuccess) {
        cleanup();
        return set_error(BCG_ERR_OOM, "debug-batch scratch allocation failed");
    }
    int rc = BCG_OK;
    if (cudaMemcpy(d_save, g->d_bc, n * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess ||
        cudaMemset(d_del, 0, cells * sizeof(double)) != cudaSuccess) {
        cleanup();
        return set_error(BCG_ERR_CUDA, "debug-batch setup failed");
    }
    DebugOut dbg;
    dbg.width = width;
    dbg.level = d_lvl;
    dbg.sigma = d_sig;
    dbg.delta = d_del;
    rc = run_plan(g, p, 0, nullptr, dbg);
    std::vector<int32_t> hl;
    std::vector<unsigned long long> hs;
    std::vector<double> hd;
    if (!rc) {
        hl.resize(cells);
        hs.resize(cells);
        hd.resize(cells);
        if (cudaMemcpy(hl.data(), d_lvl, cells * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(hs.data(), d_sig, cells * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(hd.data(), d_del, cells * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = set_error(BCG_ERR_CUDA, "reading the debug outputs failed");
    }
    cudaMemcpy(g->d_bc, d_save, n * sizeof(double), cudaMemcpyDeviceToDevice);
    cleanup();
    if (rc) return rc;
    for (uint32_t k = 0; k < nroots; ++k) {
        for (size_t v = 0; v < n; ++v) {
            const size_t vi = g->trees ? intl[v] : v;
            const bool held = vi < ns;
            const int32_t L = held ? hl[k * ns + vi] : -1;
            if (level) level[k * n + v] = L;
            if (sigma) sigma[k * n + v] = (held && L >= 0) ? hs[k * ns + vi] : 0ull;
            if (delta) delta[k * n + v] = (held && L >= 0) ? hd[k * ns + vi] : 0.0;
        }
    }
    return BCG_OK;
}

static int single_source_impl(bcg_graph *g, uint32_t src, int32_t *level, uint64_t *sigma, double *delta) {
    if (g->trees) return set_error(BCG_ERR_ARG, "single-source runs are not available on a pruned graph");
    if (src >= g->n) return set_error(BCG_ERR_ARG, "source %u >= n=%u", src, g->n);
    return debug_batch_impl(g, 1, &src, 1, level, sigma, delta);
}

int bcg_single_source(bcg_graph *g, uint32_t src, int32_t *level, uint64_t *sigma, double *delta) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    const int mode = g->sigma_mode;
    g->sigma_mode = 1;  // uint64 counts: an overflow is an error here
    const int rc = single_source_impl(g, src, level, sigma, delta);
    g->sigma_mode = mode;
    return rc;
}

int bcg_single_source_ext(bcg_graph *g, uint32_t src, int32_t *level, uint64_t *sigma_ext, double *delta) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    const int mode = g->sigma_mode;
    g->sigma_mode = 2;
    const int rc = single_source_impl(g, src, level, sigma_ext, delta);
    g->sigma_mode = mode;
    return rc;
}

int bcg_debug_batch(bcg_graph *g, uint32_t width, const uint32_t *roots, uint32_t nroots, int32_t *level,
                    uint64_t *sigma, double *delta) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    const int mode = g->sigma_mode;
    g->sigma_mode = 1;
    const int rc = debug_batch_impl(g, width, roots, nroots, level, sigma, delta);
    g->sigma_mode = mode;
    return rc;
}

int bcg_set_sigma_mode(bcg_graph *g, int mode) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    if (mode < 0 || mode > 2) return set_error(BCG_ERR_ARG, "sigma mode %d not in {0, 1, 2}", mode);
    g->sigma_mode = mode;
    return BCG_OK;
}

int bcg_graph_pruning(bcg_graph *g, uint32_t *anchor, uint32_t *reach) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    const size_t n = g->n;
    if (anchor) {
        if (g->trees) CK(cudaMemcpy(anchor, g->tdev.anchor, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        else for (size_t v = 0; v < n; ++v) anchor[v] = (uint32_t)v;
    }
    if (reach) {
        memset(reach, 0, n * sizeof(uint32_t));
        if (g->trees) {
            // a kept vertex's subtree size less itself; peeled vertices 0
            std::vector<uint32_t> anc(n);
            CK(cudaMemcpy(anc.data(), g->tdev.anchor, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(reach, g->tdev.sz, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
            for (size_t v = 0; v < n; ++v) reach[v] = anc[v] == v ? reach[v] - 1u : 0u;
        }
    }
    return BCG_OK;
}

int bcg_graph_info(bcg_graph *g, uint32_t *n, uint64_t *nnz, uint64_t *nnz_pruned, uint32_t *pruned_vertices) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    if (n) *n = g->n;
    if (nnz) *nnz = g->nnz;
    if (nnz_pruned) *nnz_pruned = g->nnz_pruned;
    if (pruned_vertices) *pruned_vertices = g->npruned;
    return BCG_OK;
}

int bcg_graph_set_reach(bcg_graph *g, const uint32_t *reach) {
    clear_error();
    if (!g || !reach) return set_error(BCG_ERR_ARG, "null argument");
    if (g->trees) return set_error(BCG_ERR_ARG, "graph was created with a pruning flag");
    const size_t n = g->n;
    std::vector<uint2> vi(n);
    for (size_t v = 0; v < n; ++v) vi[v] = make_uint2(g->h_deg[v], reach[v]);
    CK(cudaMemcpy(g->d_vinfo, vi.data(), n * sizeof(uint2), cudaMemcpyHostToDevice));
    return BCG_OK;
}

int bcg_run_weighted(bcg_graph *g, const uint32_t *roots, const double *mult, const uint32_t *pend,
                     uint64_t nroots, bcg_stats *stats) {
    clear_error();
    if (!g || (nroots && (!roots || !mult))) return set_error(BCG_ERR_ARG, "null argument");
    if (g->trees) return set_error(BCG_ERR_ARG, "graph was created with a pruning flag");
    bcg_stats local{};
    bcg_stats *st = stats ? stats : &local;
    *st = bcg_stats{};
    st->sources = nroots;
    RunPlan p;
    for (uint64_t i = 0; i < nroots; ++i) {
        if (roots[i] >= g->n) return set_error(BCG_ERR_ARG, "root %u >= n=%u", roots[i], g->n);
        p.roots.push_back(roots[i]);
        p.mult.push_back(mult[i]);
        p.pend.push_back(pend ? pend[i] : 0u);
        p.count.push_back(1);
    }
    return run_plan(g, p, 0, st, DebugOut{});
}

// Roots committed by one bcg_add_scaled call (passed by value).
constexpr uint32_t kMaxAdd = 64;
struct AddList {
    uint32_t count;
    uint32_t slot[kMaxAdd], root[kMaxAdd];
    double mult[kMaxAdd], root_add[kMaxAdd];
};

// For each listed root j in order: bc[v] += mult_j * delta_j[v] (v != root_j),
// bc[root_j] += root_add_j.
__global__ void k_add_scaled(uint32_t n, double *__restrict__ bc, const double *__restrict__ delta, AddList l) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double acc = bc[v];
    for (uint32_t j = 0; j < l.count; ++j)
        acc += (v == l.root[j]) ? l.root_add[j] : l.mult[j] * delta[(size_t)l.slot[j] * n + v];
    bc[v] = acc;
}

int bcg_run_slots(bcg_graph *g, uint32_t width, const uint32_t *roots, uint32_t nroots, double *d_delta,
                  int32_t *level, uint64_t *visited, uint64_t *wsum) {
    clear_error();
    if (!g || (nroots && !roots) || !d_delta) return set_error(BCG_ERR_ARG, "null argument");
    if (g->trees) return set_error(BCG_ERR_ARG, "graph was created with a pruning flag");
    if (width != 1 && width != 3 && width != 6) return set_error(BCG_ERR_ARG, "batch width %u not in {1,3,6}", width);
    if (nroots == 0) return set_error(BCG_ERR_ARG, "no roots");
    const size_t n = g->n, cells = n * (((size_t)nroots + width - 1) / width * width);
    RunPlan p;
    for (uint32_t k = 0; k < nroots; ++k) {
        if (roots[k] >= g->n) return set_error(BCG_ERR_ARG, "root %u >= n=%u", roots[k], g->n);
        p.roots.push_back(roots[k]);
        p.pend.push_back(0);
        p.mult.push_back(0.0);  // nothing is added to bc: the dependencies go to d_delta
        p.count.push_back(1);
    }
    if (g->slot_level_cap < cells) {
        dev_free(g->d_slot_level);
        g->d_slot_level = nullptr;
        g->slot_level_cap = 0;
        CK(dev_alloc(&g->d_slot_level, cells * sizeof(int32_t)));
        g->slot_level_cap = cells;
    }
    CK(cudaMemsetAsync(d_delta, 0, cells * sizeof(double), 0));
    DebugOut out;
    out.width = width;
    out.level = g->d_slot_level;
    out.delta = d_delta;
    bcg_stats st{};
    std::vector<RootStat> rs;
    int rc = run_plan(g, p, 0, &st, out, &rs);
    if (rc) return rc;
    if (level) CK(cudaMemcpy(level, g->d_slot_level, (size_t)nroots * n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (uint32_t k = 0; k < nroots; ++k) {
        if (visited) visited[k] = rs[k].visited;
        if (wsum) wsum[k] = rs[k].wsum;
    }
    return BCG_OK;
}

int bcg_add_scaled(bcg_graph *g, const double *d_delta, uint32_t count, const uint32_t *slot, const double *mult,
                   const uint32_t *root, const double *root_add) {
    clear_error();
    if (!g || !d_delta || (count && (!slot || !mult || !root || !root_add))) return set_error(BCG_ERR_ARG, "null argument");
    if (count > kMaxAdd) return set_error(BCG_ERR_ARG, "%u roots in one call (at most %u)", count, kMaxAdd);
    if (count == 0) return BCG_OK;
    AddList l{};
    l.count = count;
    for (uint32_t j = 0; j < count; ++j) {
        if (root[j] >= g->n) return set_error(BCG_ERR_ARG, "root %u >= n=%u", root[j], g->n);
        l.slot[j] = slot[j];
        l.root[j] = root[j];
        l.mult[j] = mult[j];
        l.root_add[j] = root_add[j];
    }
    const uint32_t n = g->n;
    k_add_scaled<<<(n + 255) / 256, 256>>>(n, g->d_bc, d_delta, l);
    CK(cudaGetLastError());
    return BCG_OK;
}

int bcg_run_root_levels(bcg_graph *g, uint32_t root, double mult, uint32_t pend, int32_t *level,
                        bcg_stats *stats) {
    clear_error();
    if (!g || !level) return set_error(BCG_ERR_ARG, "null argument");
    if (g->trees) return set_error(BCG_ERR_ARG, "graph was created with a pruning flag");
    if (root >= g->n) return set_error(BCG_ERR_ARG, "root %u >= n=%u", root, g->n);
    bcg_stats local{};
    bcg_stats *st = stats ? stats : &local;
    *st = bcg_stats{};
    st->sources = 1;
    RunPlan p;
    p.roots.push_back(root);
    p.mult.push_back(mult);
    p.pend.push_back(pend);
    p.count.push_back(1);
    if (!g->d_level_out) CK(dev_alloc(&g->d_level_out, (size_t)g->n * sizeof(int32_t)));
    DebugOut out;  // width 1, levels only: bc accumulates as in a plain run
    out.width = 1;
    out.level = g->d_level_out;
    int rc = run_plan(g, p, 0, st, out);
    if (rc) return rc;
    CK(cudaMemcpy(level, g->d_level_out, (size_t)g->n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return BCG_OK;
}

int bcg_set_batch_width(bcg_graph *g, uint32_t width) {
    clear_error();
    if (!g) return set_error(BCG_ERR_ARG, "null handle");
    if (width != 0 && width != 1 && width != 3 && width != 6)
        return set_error(BCG_ERR_ARG, "batch width must be 0, 1, 3 or 6");
    g->forced_width = width;
    return BCG_OK;
}

}  // extern "C"
