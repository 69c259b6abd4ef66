// libbc2d_compat.so: the reference's bc2d.h mono-path ABI (include/bc2d_compat.h)
// implemented on libbcg.  Errors print and exit like the reference's
// MY_CUDA_CHECK (cudamacro.h:1-7), since the ABI has no status returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bc2d_compat.h"
#include "bcg.h"

extern "C" {
extern uint64_t N;  // vertex count, defined by the reference's bc2d.c
}

namespace {

bcg_graph *g_graph = nullptr;
std::vector<uint32_t> g_deg;       // degree of every vertex (CSC column lengths)
std::vector<uint32_t> g_count;     // vertices per level of the current source
uint32_t g_v0 = 0;
uint32_t g_reach_v0 = 0;
bool g_pending = false;            // the current source's search has not run yet
bool g_committed = true;           // the current source's dependencies are in bc
uint64_t g_reach_visited = 0;      // sum of reach over the vertices it reached, root excluded

// Sources searched ahead: the driver asks for its sources one at a time, in
// increasing order, skipping degree 0 (bc2d.c:1016-1036), so the first
// source of a block is searched together with the next candidates of that
// order, in batches of 6 in one launch (bcg_run_slots: nothing added to
// bc).  The driver commits each source in update_bc_cuda; the commits are
// added to bc in that order by one kernel when the next block is searched
// or bc is read (bcg_add_scaled).  A candidate it never asks for is dropped.
constexpr uint32_t kWidth = 6;
constexpr uint32_t kMaxAhead = 30;               // five batches
constexpr size_t kAheadBytes = 64ull << 20;      // depths + dependencies of a block
struct Ahead {
    uint32_t cap = kWidth;                       // roots per block (a multiple of kWidth)
    uint32_t nroots = 0;
    uint32_t roots[kMaxAhead] = {};
    uint64_t visited[kMaxAhead] = {}, wsum[kMaxAhead] = {};
    std::vector<int32_t> level;                  // cap * n depths (-1 = not reached)
    double *d_delta = nullptr;                   // cap * n dependencies on the device
    // committed sources not yet added to bc
    uint32_t ncommit = 0;
    uint32_t cslot[kMaxAhead] = {}, croot[kMaxAhead] = {};
    double cmult[kMaxAhead] = {}, cadd[kMaxAhead] = {};
} g_ahead;
uint32_t g_slot = 0;               // the current source's slot in g_ahead


[[noreturn]] void fail(const char *what, int rc) {
    fprintf(stderr, "bc2d_compat: %s failed (%d): %s\n", what, rc, bcg_last_error());
    exit(EXIT_FAILURE);
}

void flush_commits() {
    if (!g_ahead.ncommit) return;
    int rc = bcg_add_scaled(g_graph, g_ahead.d_delta, g_ahead.ncommit, g_ahead.cslot, g_ahead.cmult, g_ahead.croot,
                            g_ahead.cadd);
    if (rc) fail("update_bc_cuda", rc);
    g_ahead.ncommit = 0;
}

}  // namespace

extern "C" {

size_t initcuda(uint64_t ned, LOCINT *col, LOCINT *row) {
    const uint32_t n = (uint32_t)N;
    int rc = bcg_graph_create(col, row, n, ned, 0u, &g_graph);
    if (rc) fail("initcuda", rc);
    g_deg.resize(n);
    for (uint32_t v = 0; v < n; ++v) g_deg[v] = col[v + 1] - col[v];
    g_ahead = Ahead{};
    const size_t per_root = (size_t)n * (sizeof(double) + sizeof(int32_t));
    size_t cap = kAheadBytes / per_root / kWidth * kWidth;
    g_ahead.cap = (uint32_t)std::min<size_t>(kMaxAhead, std::max<size_t>(kWidth, cap));
    g_ahead.level.assign((size_t)g_ahead.cap * n, -1);
    if (cudaMalloc(&g_ahead.d_delta, (size_t)g_ahead.cap * n * sizeof(double)) != cudaSuccess) {
        fprintf(stderr, "bc2d_compat: initcuda: cudaMalloc of %zu bytes failed\n",
                (size_t)g_ahead.cap * n * sizeof(double));
        exit(EXIT_FAILURE);
    }
    printf("ROWBL = %i - ROWPP = %i\n", (int)n, (int)n);
    return (size_t)(n + 1) * 4 + ned * 4 + (size_t)n * (8 + 8 + 16);
}

void init_bc_1degree_device(LOCINT *reach) {
    int rc = bcg_graph_set_reach(g_graph, reach);
    if (rc) fail("init_bc_1degree_device", rc);
}

void get_deg(LOCINT *deg) { memcpy(deg, g_deg.data(), g_deg.size() * sizeof(uint32_t)); }

void setcuda(uint64_t, LOCINT *, LOCINT *, LOCINT reach_v0) {
    g_reach_v0 = reach_v0;
    g_count.clear();
}

// The driver's per-source sequence (bc_func_mono, bc2d.c:504-580) is
// setcuda, set_mlp_cuda, then scan_col_csc_cuda_mono per level inside its
// timer, the scan_frt_csc_cuda_mono calls, pre_update_bc_cuda and
// update_bc_cuda.  Each source costs one slot of a searched-ahead block: the
// first level call finds (or searches) it, the later calls return the
// per-level counts it found, and update_bc_cuda commits its dependencies,
// weighted by the root's folded pendants (added to bc with the block's other
// commits, in commit order).
void set_mlp_cuda(LOCINT row, int, int) {
    g_v0 = row;
    g_pending = true;
    g_committed = false;
    g_count.clear();
}

static void search_source() {
    const uint32_t n = (uint32_t)g_deg.size();
    uint32_t slot = kMaxAhead;
    for (uint32_t k = 0; k < g_ahead.nroots; ++k)
        if (g_ahead.roots[k] == g_v0) slot = k;
    if (slot == kMaxAhead) {
        // a new block: this source and the next candidates of the driver's
        // order (the block's dependencies are about to be overwritten)
        flush_commits();
        uint32_t nr = 0;
        g_ahead.roots[nr++] = g_v0;
        for (uint32_t v = g_v0 + 1; v < n && nr < g_ahead.cap; ++v)
            if (g_deg[v]) g_ahead.roots[nr++] = v;
        g_ahead.nroots = 0;
        int rc = bcg_run_slots(g_graph, kWidth, g_ahead.roots, nr, g_ahead.d_delta, g_ahead.level.data(),
                               g_ahead.visited, g_ahead.wsum);
        if (rc) fail("scan_col_csc_cuda_mono", rc);
        g_ahead.nroots = nr;
        slot = 0;
    }
    g_slot = slot;
    g_pending = false;
    g_count.clear();
    const int32_t *lv = g_ahead.level.data() + (size_t)slot * n;
    for (uint32_t v = 0; v < n; ++v) {
        const int32_t l = lv[v];
        if (l < 0) continue;
        if ((size_t)l >= g_count.size()) g_count.resize(l + 1, 0);
        ++g_count[l];
    }
    // wsum = sum of (1 + reach) over the reached vertices
    g_reach_visited = g_ahead.wsum[slot] - g_ahead.visited[slot] - g_reach_v0;
}

LOCINT scan_col_csc_cuda_mono(int, int level) {
    if (g_pending) search_source();
    return (level >= 0 && (size_t)level < g_count.size()) ? g_count[level] : 0u;
}

LOCINT scan_frt_csc_cuda_mono(int, int ncol, int) { return (LOCINT)ncol; }

void pre_update_bc_cuda(LOCINT *, uint64_t, LOCINT *all) {
    if (g_pending) search_source();
    *all = (LOCINT)g_reach_visited;
}

// Commits bc[v] += (reach_v0 + 1) * delta_v0(v) for v != v0 and the source
// term bc[v0] += reach_v0 * (W - 2) (update_bc, cuda_kernels.cu:263-277,
// without its contributions to unreached vertices: the definition's bc).
void update_bc_cuda(uint64_t, int, const uint64_t) {
    if (g_pending) search_source();  // a driver that skipped the level calls
    if (g_committed) return;
    if (g_ahead.ncommit == kMaxAhead) flush_commits();  // a driver that repeats sources
    const uint64_t W = g_ahead.wsum[g_slot];
    const uint32_t j = g_ahead.ncommit++;
    g_ahead.cslot[j] = g_slot;
    g_ahead.croot[j] = g_v0;
    g_ahead.cmult[j] = (double)g_reach_v0 + 1.0;
    g_ahead.cadd[j] = (g_reach_v0 && W >= 2) ? (double)g_reach_v0 * (double)(W - 2) : 0.0;
    g_committed = true;
}

void get_msk(LOCINT *msk) {
    const size_t n = g_deg.size();
    const int32_t *lv = g_ahead.level.data() + (size_t)g_slot * n;
    memset(msk, 0, ((n + 31) / 32) * sizeof(uint32_t));
    for (size_t v = 0; v < n; ++v)
        if (lv[v] >= 0) msk[v / 32] |= 1u << (v % 32);
}

void get_bc(float *bc) {
    flush_commits();
    std::vector<double> b(g_deg.size());
    int rc = bcg_get_bc(g_graph, b.data());
    if (rc) fail("get_bc", rc);
    for (size_t v = 0; v < b.size(); ++v) bc[v] = (float)b[v];
}

void fincuda(void) {
    if (g_graph) bcg_graph_destroy(g_graph);
    g_graph = nullptr;
    cudaFree(g_ahead.d_delta);
    g_ahead = Ahead{};
}

void *CudaMallocHostSet(size_t size, int val) {
    void *p = nullptr;
    cudaError_t e = cudaMallocHost(&p, size);
    if (e != cudaSuccess) {
        fprintf(stderr, "Cuda error in CudaMallocHostSet : %s.\n", cudaGetErrorString(e));
        exit(EXIT_FAILURE);
    }
    memset(p, val, size);
    return p;
}

void CudaFreeHost(void *ptr) {
    if (ptr) cudaFreeHost(ptr);
}

}  // extern "C"
