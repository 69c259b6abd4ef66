// libbc2d_compat.so: the reference's bc2d.h mono-path ABI (include/bc2d_compat.h)
// implemented on libbcg.  Errors print and exit like the reference's
// MY_CUDA_CHECK (cudamacro.h:1-7), since the ABI has no status returns.
#include <cuda_runtime.h>

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
std::vector<int32_t> g_level;      // BFS depth of the current source (-1 = not reached)
std::vector<uint32_t> g_count;     // vertices per level of the current source
uint32_t g_v0 = 0;
uint32_t g_reach_v0 = 0;
bool g_pending = false;            // the current source's search has not run yet
uint64_t g_reach_visited = 0;      // sum of reach over the vertices it reached, root excluded

[[noreturn]] void fail(const char *what, int rc) {
    fprintf(stderr, "bc2d_compat: %s failed (%d): %s\n", what, rc, bcg_last_error());
    exit(EXIT_FAILURE);
}

}  // namespace

extern "C" {

size_t initcuda(uint64_t ned, LOCINT *col, LOCINT *row) {
    const uint32_t n = (uint32_t)N;
    int rc = bcg_graph_create(col, row, n, ned, 0u, &g_graph);
    if (rc) fail("initcuda", rc);
    g_deg.resize(n);
    for (uint32_t v = 0; v < n; ++v) g_deg[v] = col[v + 1] - col[v];
    g_level.assign(n, -1);
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
// update_bc_cuda.  The engine does the whole source in one search: the first
// level call runs it (weighted by the root's folded pendants, exporting the
// depths), the later calls return the per-level counts it found, and
// update_bc_cuda has nothing left to do.
void set_mlp_cuda(LOCINT row, int, int) {
    g_v0 = row;
    g_pending = true;
    g_count.clear();
}

static void run_source() {
    const double mult = (double)g_reach_v0 + 1.0;
    bcg_stats st{};
    int rc = bcg_run_root_levels(g_graph, g_v0, mult, g_reach_v0, g_level.data(), &st);
    if (rc) fail("scan_col_csc_cuda_mono", rc);
    g_pending = false;
    g_count.clear();
    for (int32_t l : g_level) {
        if (l < 0) continue;
        if ((size_t)l >= g_count.size()) g_count.resize(l + 1, 0);
        ++g_count[l];
    }
    // comp_vertices = sum of (1 + reach) over the reached vertices
    g_reach_visited = st.comp_vertices - st.visited - g_reach_v0;
}

LOCINT scan_col_csc_cuda_mono(int, int level) {
    if (g_pending) run_source();
    return (level >= 0 && (size_t)level < g_count.size()) ? g_count[level] : 0u;
}

LOCINT scan_frt_csc_cuda_mono(int, int ncol, int) { return (LOCINT)ncol; }

void pre_update_bc_cuda(LOCINT *, uint64_t, LOCINT *all) {
    if (g_pending) run_source();
    *all = (LOCINT)g_reach_visited;
}

void update_bc_cuda(uint64_t, int, const uint64_t) {
    if (g_pending) run_source();  // a driver that skipped the level calls
}

void get_msk(LOCINT *msk) {
    const size_t n = g_level.size();
    memset(msk, 0, ((n + 31) / 32) * sizeof(uint32_t));
    for (size_t v = 0; v < n; ++v)
        if (g_level[v] >= 0) msk[v / 32] |= 1u << (v % 32);
}

void get_bc(float *bc) {
    std::vector<double> b(g_deg.size());
    int rc = bcg_get_bc(g_graph, b.data());
    if (rc) fail("get_bc", rc);
    for (size_t v = 0; v < b.size(); ++v) bc[v] = (float)b[v];
}

void fincuda(void) {
    if (g_graph) bcg_graph_destroy(g_graph);
    g_graph = nullptr;
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
