// bcg_bc_noalloc: exact BC over a device-resident CSR that allocates no device
// memory.  It is the bcg_run path (graph preparation + the persistent sweep
// kernel, sweep.cu) with every scratch buffer carved out of one file-scope
// static __device__ array of fixed size instead of cudaMalloc'd buffers, so
// graphs are limited to BCG_NOALLOC_MAX_VERTICES vertices,
// BCG_NOALLOC_MAX_ADJ adjacency entries and BCG_NOALLOC_MAX_SOURCES sources
// per call.  The preparation that bcg_graph_create does on the host (CSR
// checks, work tiles, source plan) runs here as small device kernels into the
// same scratch.  No pruning; undirected graphs only.
//
// Setup: the first call on a device (with that device current) takes the
// array's address with cudaGetSymbolAddress, which loads this module; the
// address is kept per device for the life of the process.
//
// Scratch that must start at zero and is cleared by every call: the status
// block, the sweep control block, the tile marks, the hub arrival counters,
// and the 16-byte tail pads of the adjacency, offsets and degree copies (and
// d_bc when not accumulating).  Everything else (state rows, level lists, the
// unvisited-tile ring, roots, the hub chunk slots, the saved accumulators) is
// written before it is read.  One scratch per device: calls that overlap on the same device race
// on it.
//
// Path counts: exact uint64 first; when one overflows (large grids, long
// chains of diamonds), the accumulators saved before the sweep are put back
// and the sweep runs again with extended-range counts (ext64.cuh), as
// bcg_run does in its automatic mode.
#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "bcg_common.hpp"
#include "engine.cuh"

namespace bcg {

int launch_sweep(int S, const BatchArgs &a, cudaStream_t st, int *grid_out, bool ext = false);

namespace {

constexpr uint64_t kNaMaxN = BCG_NOALLOC_MAX_VERTICES;
constexpr uint64_t kNaMaxAdj = BCG_NOALLOC_MAX_ADJ;
constexpr uint64_t kNaMaxSrc = BCG_NOALLOC_MAX_SOURCES;
constexpr int kNaMaxWidth = 6;
// every tile holds at least one non-hub vertex or one kTileEdges-entry hub
// chunk: tiles <= (n - hubs) + sum over hubs of ceil(deg / kTileEdges)
// <= n + adj / kTileEdges
constexpr uint64_t kNaMaxTiles = kNaMaxN + kNaMaxAdj / kTileEdges;
constexpr uint64_t kNaMaxHubs = kNaMaxAdj / (kTileEdges + 1) + 1;  // a hub has more than kTileEdges entries
// a hub of degree g has ceil(g / kTileEdges) <= g / kTileEdges + 1 chunks
constexpr uint64_t kNaMaxHubChunks = kNaMaxAdj / kTileEdges + kNaMaxHubs;
constexpr uint64_t kNaMaxSlots = kNaMaxSrc + kNaMaxWidth;
constexpr int kNaMaxDevices = 64;

// What a failed device-side check found.
enum : uint32_t { kBadNone = 0, kBadOffsets = 1, kBadAdjacency = 2, kBadSource = 3, kBadTiles = 4 };

struct NaStatus {
    int error;           // BCG_ERR_ARG when a check failed
    uint32_t what;       // kBad*
    unsigned long long index;  // offending vertex / entry / source position
    uint32_t ntiles;
    uint32_t nhub;
    uint32_t nroots;
    uint32_t skipped;
};

constexpr size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of the scratch regions (each 256-byte aligned).
constexpr size_t kOffStatus = 0;
constexpr size_t kOffCtrl = kOffStatus + up256(sizeof(NaStatus));
constexpr size_t kOffAdj = kOffCtrl + up256(sizeof(Ctrl));
constexpr size_t kOffVinfo = kOffAdj + up256((kNaMaxAdj + 4) * sizeof(uint32_t));
// offsets are copied too: the sweep reads them in 16-byte aligned pieces
// that may run 4 entries past n + 1 (zeroed tail)
constexpr size_t kOffOffs = kOffVinfo + up256((kNaMaxN + 4) * sizeof(uint2));
constexpr size_t kOffTiles = kOffOffs + up256((kNaMaxN + 1 + 4) * sizeof(uint32_t));
constexpr size_t kOffTileOf = kOffTiles + up256(kNaMaxTiles * sizeof(Tile));
constexpr size_t kOffTmark = kOffTileOf + up256(kNaMaxN * sizeof(uint32_t));
constexpr size_t kOffLists = kOffTmark + up256(kNaMaxTiles * sizeof(uint32_t));
constexpr size_t kOffLbase = kOffLists + up256(kNaMaxWidth * (kNaMaxN + kNaMaxTiles) * sizeof(uint32_t));
constexpr size_t kOffLcnt = kOffLbase + up256((kMaxLevel + 3) * sizeof(uint32_t));
constexpr size_t kOffUlist = kOffLcnt + up256((kMaxLevel + 3) * sizeof(uint32_t));
constexpr size_t kOffRows = kOffUlist + up256(2 * kNaMaxTiles * sizeof(uint32_t));
constexpr size_t kOffHubAcc = kOffRows + up256(kNaMaxN * row_bytes(kNaMaxWidth));
constexpr size_t kOffHubCnt = kOffHubAcc + up256(kNaMaxHubChunks * kNaMaxWidth * sizeof(unsigned long long));
constexpr size_t kOffRoots = kOffHubCnt + up256(kNaMaxHubs * sizeof(unsigned int));
constexpr size_t kOffPend = kOffRoots + up256(kNaMaxSlots * sizeof(uint32_t));
constexpr size_t kOffMult = kOffPend + up256(kNaMaxSlots * sizeof(uint32_t));
constexpr size_t kOffRstat = kOffMult + up256(kNaMaxSlots * sizeof(double));
constexpr size_t kOffBcSave = kOffRstat + up256(kNaMaxSlots * sizeof(RootStat));
constexpr size_t kScratchBytes = kOffBcSave + up256(kNaMaxN * sizeof(double));
static_assert(kScratchBytes <= (size_t)20 << 20, "no-allocation scratch is meant to stay under 20 MiB");
static_assert(kOffAdj == kOffCtrl + up256(sizeof(Ctrl)) && kOffCtrl > kOffStatus,
              "status and control blocks lead the scratch so one memset clears both");

}  // namespace
}  // namespace bcg

// The scratch of bcg_bc_noalloc: one per device, about 19 MiB.
static __device__ __align__(256) unsigned char g_noalloc_scratch[bcg::kScratchBytes];

namespace bcg {
namespace {

std::mutex g_na_mu;
unsigned char *g_na_ptr[kNaMaxDevices] = {};

__device__ void na_fail(NaStatus *st, uint32_t what, unsigned long long index) {
    if (atomicCAS(&st->error, 0, BCG_ERR_ARG) == 0) {
        st->what = what;
        st->index = index;
    }
}

// offsets[0] == 0, offsets[n] == nnz, non-decreasing (one thread per entry of offsets).
__global__ void k_na_check_offsets(uint32_t n, unsigned long long nnz, const uint32_t *__restrict__ offs,
                                   NaStatus *st) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v > n) return;
    const uint32_t o = offs[v];
    const bool bad = (v == 0 && o != 0) || (v == n && (unsigned long long)o != nnz) || (v < n && offs[v + 1] < o);
    if (bad) na_fail(st, kBadOffsets, v);
}

// every adjacency id < n (grid-stride over the copy)
__global__ void k_na_check_adj(uint32_t n, unsigned long long nnz, const uint32_t *__restrict__ adj, NaStatus *st) {
    for (unsigned long long e = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (unsigned long long)gridDim.x * blockDim.x)
        if (adj[e] >= n) na_fail(st, kBadAdjacency, e);
}

__global__ void k_na_vinfo(uint32_t n, const uint32_t *__restrict__ offs, uint2 *__restrict__ vinfo) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) vinfo[v] = make_uint2(offs[v + 1] - offs[v], 0u);
}

// Work tiles, the same greedy partition bcg_graph_create builds on the host:
// runs of up to kTileVerts (32) consecutive vertices with at most kTileEdges
// (512 by default) adjacency entries, and vertices with more than kTileEdges
// entries split into kTileEdges-entry chunks.  One thread: the partition is
// sequential and the graphs here are small.
__global__ void k_na_tiles(uint32_t n, const uint32_t *__restrict__ offs, Tile *__restrict__ tiles,
                           uint32_t *__restrict__ tile_of, NaStatus *st) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (st->error) return;  // offsets were rejected: nothing below may trust them
    uint32_t nt = 0, nhub = 0, nchunk = 0, v = 0;
    while (v < n) {
        const uint32_t dv = offs[v + 1] - offs[v];
        if (dv > (uint32_t)kTileEdges) {
            const uint32_t nch = (dv + kTileEdges - 1) / kTileEdges;
            if ((uint64_t)nt + nch > kNaMaxTiles || nhub >= kNaMaxHubs) {
                na_fail(st, kBadTiles, v);
                return;
            }
            tile_of[v] = nt | kHubFlag;
            for (uint32_t c = 0; c < nch; ++c) {
                Tile t{};
                t.v0 = v;
                t.v1 = v + 1;
                t.e0 = offs[v] + c * kTileEdges;
                t.e1 = min(offs[v + 1], t.e0 + (uint32_t)kTileEdges);
                t.hub = (int32_t)nhub;
                t.nchunks = nch;
                t.hslot = nchunk++;
                t.hchunk = c;
                tiles[nt++] = t;
            }
            ++nhub;
            ++v;
            continue;
        }
        if ((uint64_t)nt + 1 > kNaMaxTiles) {
            na_fail(st, kBadTiles, v);
            return;
        }
        const uint32_t start = v;
        uint32_t sum = 0;
        while (v < n && v - start < (uint32_t)kTileVerts) {
            const uint32_t d = offs[v + 1] - offs[v];
            if (d > (uint32_t)kTileEdges || sum + d > (uint32_t)kTileEdges) break;
            sum += d;
            tile_of[v] = nt;
            ++v;
        }
        Tile t{};
        t.v0 = start;
        t.v1 = v;
        t.e0 = offs[start];
        t.e1 = offs[v];
        t.hub = -1;
        t.nchunks = 1;
        tiles[nt++] = t;
    }
    st->ntiles = nt;
    st->nhub = nhub;
}

// Source plan: sources of degree 0 are skipped (bc2d.c:1026-1034), the rest
// become roots in list order with weight 1; the slots up to the next multiple
// of 6 are empty.  One CTA of 1024 threads, a block-wide scan per 1024 sources.
__global__ void __launch_bounds__(1024) k_na_roots(uint32_t n, const uint32_t *__restrict__ offs,
                                                   const uint32_t *__restrict__ src, uint32_t nsrc,
                                                   uint32_t *__restrict__ roots, double *__restrict__ mult,
                                                   uint32_t *__restrict__ pend, NaStatus *st) {
    __shared__ uint32_t wpre[32];
    __shared__ uint32_t chunk_total;
    __shared__ uint32_t base;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    uint32_t skipped = 0;
    for (uint32_t i0 = 0; i0 < nsrc; i0 += blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        uint32_t s = 0;
        bool keep = false;
        if (i < nsrc) {
            s = src[i];
            if (s >= n)
                na_fail(st, kBadSource, i);
            else if (offs[s + 1] > offs[s])
                keep = true;
            else
                ++skipped;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wpre[warp] = __popc(bal);
        __syncthreads();
        if (warp == 0) {
            const uint32_t x = lane < (blockDim.x >> 5) ? wpre[lane] : 0u;
            uint32_t inc = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= (uint32_t)o) inc += y;
            }
            if (lane < (blockDim.x >> 5)) wpre[lane] = inc - x;
            if (lane == 31) chunk_total = inc;
        }
        __syncthreads();
        if (keep) {
            const uint32_t pos = base + wpre[warp] + __popc(bal & ((1u << lane) - 1u));
            roots[pos] = s;
            mult[pos] = 1.0;
            pend[pos] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) base += chunk_total;
        __syncthreads();
    }
    if (skipped) atomicAdd(&st->skipped, skipped);
    const uint32_t nr = base;
    const uint32_t padded = (nr + kNaMaxWidth - 1) / kNaMaxWidth * kNaMaxWidth;
    for (uint32_t j = nr + threadIdx.x; j < padded; j += blockDim.x) {
        roots[j] = kNoRoot;
        mult[j] = 0.0;
        pend[j] = 0;
    }
    if (threadIdx.x == 0) st->nroots = nr;
}

// Address of this device's scratch; the first call per device takes it with
// cudaGetSymbolAddress (the device must be current).
int na_scratch(unsigned char **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(BCG_ERR_NOGPU, "no CUDA device: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kNaMaxDevices)
        return set_error(BCG_ERR_ARG, "device %d outside the %d devices the no-allocation path tracks", dev,
                         kNaMaxDevices);
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(e == cudaErrorNoKernelImageForDevice ? BCG_ERR_NOGPU : BCG_ERR_CUDA,
                             "cudaGetSymbolAddress of the no-allocation scratch on device %d: %s", dev,
                             cudaGetErrorString(e));
        g_na_ptr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_na_ptr[dev];
    return BCG_OK;
}

const char *bad_name(uint32_t what) {
    switch (what) {
        case kBadOffsets: return "offsets (offsets[0] must be 0, offsets[n] == nnz, non-decreasing) at vertex";
        case kBadAdjacency: return "adjacency id >= n at entry";
        case kBadSource: return "source id >= n at position";
        case kBadTiles: return "work-tile capacity exceeded at vertex";
        default: return "device check failed at";
    }
}

}  // namespace
}  // namespace bcg

using namespace bcg;

#define NA_CK(call)                                                                                  \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return set_error(BCG_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

extern "C" int bcg_bc_noalloc(const uint32_t *d_offsets, const uint32_t *d_adj, uint32_t n, uint64_t nnz,
                              const uint32_t *d_sources, uint64_t nsrc, double *d_bc, int accumulate,
                              void *stream) {
    clear_error();
    if (n > kNaMaxN)
        return set_error(BCG_ERR_RANGE, "n = %u exceeds the no-allocation limit of %llu vertices", n,
                         (unsigned long long)kNaMaxN);
    if (nnz > kNaMaxAdj)
        return set_error(BCG_ERR_RANGE, "nnz = %llu exceeds the no-allocation limit of %llu adjacency entries",
                         (unsigned long long)nnz, (unsigned long long)kNaMaxAdj);
    if (nsrc > kNaMaxSrc)
        return set_error(BCG_ERR_RANGE, "%llu sources exceed the no-allocation limit of %llu per call",
                         (unsigned long long)nsrc, (unsigned long long)kNaMaxSrc);
    if (n == 0) return BCG_OK;
    if (!d_offsets || (nnz && !d_adj) || (nsrc && !d_sources) || !d_bc)
        return set_error(BCG_ERR_ARG, "null device pointer");
    unsigned char *scr = nullptr;
    int rc = na_scratch(&scr);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;

    NaStatus *d_status = reinterpret_cast<NaStatus *>(scr + kOffStatus);
    Ctrl *d_ctrl = reinterpret_cast<Ctrl *>(scr + kOffCtrl);
    uint32_t *d_adjc = reinterpret_cast<uint32_t *>(scr + kOffAdj);
    uint2 *d_vinfo = reinterpret_cast<uint2 *>(scr + kOffVinfo);
    uint32_t *d_offc = reinterpret_cast<uint32_t *>(scr + kOffOffs);
    Tile *d_tiles = reinterpret_cast<Tile *>(scr + kOffTiles);
    uint32_t *d_tile_of = reinterpret_cast<uint32_t *>(scr + kOffTileOf);
    uint32_t *d_tmark = reinterpret_cast<uint32_t *>(scr + kOffTmark);
    uint32_t *d_roots = reinterpret_cast<uint32_t *>(scr + kOffRoots);
    uint32_t *d_pend = reinterpret_cast<uint32_t *>(scr + kOffPend);
    double *d_mult = reinterpret_cast<double *>(scr + kOffMult);

    // status + control blocks, then the adjacency copy with its zeroed tail pad
    // (the sweep stages adjacency ranges in 16-byte chunks past e1)
    NA_CK(cudaMemsetAsync(scr, 0, kOffAdj, st));
    if (nnz) NA_CK(cudaMemcpyAsync(d_adjc, d_adj, nnz * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    NA_CK(cudaMemsetAsync(d_adjc + nnz, 0, 4 * sizeof(uint32_t), st));
    NA_CK(cudaMemcpyAsync(d_offc, d_offsets, ((size_t)n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    NA_CK(cudaMemsetAsync(d_offc + n + 1, 0, 4 * sizeof(uint32_t), st));
    NA_CK(cudaMemsetAsync(d_vinfo + n, 0, 4 * sizeof(uint2), st));
    k_na_check_offsets<<<(unsigned)((n + 1 + 255) / 256), 256, 0, st>>>(n, nnz, d_offsets, d_status);
    if (nnz) {
        const unsigned blocks = (unsigned)std::min<uint64_t>((nnz + 255) / 256, 148ull * 8);
        k_na_check_adj<<<blocks, 256, 0, st>>>(n, nnz, d_adjc, d_status);
    }
    k_na_vinfo<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, d_offsets, d_vinfo);
    k_na_tiles<<<1, 1, 0, st>>>(n, d_offsets, d_tiles, d_tile_of, d_status);
    k_na_roots<<<1, 1024, 0, st>>>(n, d_offsets, d_sources, (uint32_t)nsrc, d_roots, d_mult, d_pend, d_status);
    NA_CK(cudaGetLastError());
    NaStatus hs{};
    NA_CK(cudaMemcpyAsync(&hs, d_status, sizeof(hs), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (hs.error)
        return set_error(BCG_ERR_ARG, "invalid input: %s %llu", bad_name(hs.what), hs.index);

    if (!accumulate) NA_CK(cudaMemsetAsync(d_bc, 0, (size_t)n * sizeof(double), st));
    // the caller's accumulators before the sweep: a run whose uint64 path
    // counts overflow is redone with extended-range counts from this copy,
    // as bcg_run does in its automatic mode
    double *d_bc_save = reinterpret_cast<double *>(scr + kOffBcSave);
    NA_CK(cudaMemcpyAsync(d_bc_save, d_bc, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (hs.nroots == 0) {
        NA_CK(cudaStreamSynchronize(st));
        return BCG_OK;
    }
    // the batch width bcg_run picks for a graph whose rows fit its state budget
    const uint32_t S = hs.nroots > 3 ? 6u : (hs.nroots > 1 ? 3u : 1u);
    const uint64_t nbatch = (hs.nroots + S - 1) / S;
    const uint32_t nhub_alloc = hs.nhub ? hs.nhub : 1u;
    NA_CK(cudaMemsetAsync(d_tmark, 0, (size_t)(hs.ntiles ? hs.ntiles : 1u) * sizeof(uint32_t), st));
    NA_CK(cudaMemsetAsync(scr + kOffHubCnt, 0, (size_t)nhub_alloc * sizeof(unsigned int), st));

    BatchArgs a{};
    a.n = n;
    a.offs = d_offc;
    a.adj = d_adjc;
    a.vinfo = d_vinfo;
    a.tiles = d_tiles;
    a.ntiles = hs.ntiles;
    a.tile_of = d_tile_of;
    a.tmark = d_tmark;
    a.lists = reinterpret_cast<uint32_t *>(scr + kOffLists);
    a.list_cap = (unsigned long long)S * ((unsigned long long)n + hs.ntiles);
    a.lbase = reinterpret_cast<uint32_t *>(scr + kOffLbase);
    a.lcnt = reinterpret_cast<uint32_t *>(scr + kOffLcnt);
    a.ulist = reinterpret_cast<uint32_t *>(scr + kOffUlist);
    a.rows = scr + kOffRows;
    a.bc = d_bc;
    a.roots = d_roots;
    a.mult = d_mult;
    a.pend = d_pend;
    a.nbatch = (uint32_t)nbatch;  // <= 65536 / 6 + 1: one launch stays under the 65535-batch tile-key limit
    a.hub_acc = reinterpret_cast<unsigned long long *>(scr + kOffHubAcc);
    a.hub_cnt = reinterpret_cast<unsigned int *>(scr + kOffHubCnt);
    a.ctrl = d_ctrl;
    a.rstat = reinterpret_cast<RootStat *>(scr + kOffRstat);
    a.nnz = nnz;
    a.push_pull_ratio = 0.2f;
    if (const char *e = getenv("BCG_PUSH_PULL_RATIO")) a.push_pull_ratio = (float)atof(e);
    a.mark_ratio = 8;
    if (const char *e = getenv("BCG_CHILD_MARK_RATIO")) a.mark_ratio = (uint32_t)std::min(strtoul(e, nullptr, 10), 1024ul);
    a.directed = 0;
    for (int pass = 0; pass < 2; ++pass) {
        const bool ext = pass == 1;
        if (ext) {
            // overflow: restore the accumulators and clear the scratch the
            // aborted sweep left behind (control block, tile marks, hub
            // arrival counters), then run extended counts
            NA_CK(cudaMemcpyAsync(d_bc, d_bc_save, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
            NA_CK(cudaMemsetAsync(d_ctrl, 0, sizeof(Ctrl), st));
            NA_CK(cudaMemsetAsync(d_tmark, 0, (size_t)(hs.ntiles ? hs.ntiles : 1u) * sizeof(uint32_t), st));
            NA_CK(cudaMemsetAsync(scr + kOffHubCnt, 0, (size_t)nhub_alloc * sizeof(unsigned int), st));
        }
        int grid = 0;
        rc = launch_sweep((int)S, a, st, &grid, ext);
        if (rc) return rc;
        int flags[2] = {0, 0};  // Ctrl::error, Ctrl::overflow
        NA_CK(cudaMemcpyAsync(flags, &d_ctrl->error, sizeof(flags), cudaMemcpyDeviceToHost, st));
        NA_CK(cudaStreamSynchronize(st));
        if (flags[1] || flags[0] == BCG_ERR_OVERFLOW) {
            if (!ext) continue;
            return set_error(BCG_ERR_OVERFLOW, "a shortest-path count exceeded the extended range");
        }
        if (flags[0])
            return set_error(flags[0], "device reported error %d (%s)", flags[0],
                             flags[0] == BCG_ERR_TIMEOUT ? "a bounded wait gave up" : "level limit exceeded");
        return BCG_OK;
    }
    return BCG_OK;
}
