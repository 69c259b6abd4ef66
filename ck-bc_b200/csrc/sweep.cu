// Multi-source Brandes sweep kernel (sm_100a).
//
// One cooperative, persistent launch runs every batch of S BFS roots:
//   init      rows of all vertices reset, roots at level 0 with sigma 1
//             (setcuda + set_mlp_cuda, cuda_kernels.cu:689-703, 1100-1119)
//   forward   one sweep per BFS level, push (top-down from the level-d
//             vertices) or pull (bottom-up into the unvisited vertices),
//             chosen per level from the frontier/unvisited edge counts; sigma is
//             summed exactly in uint64 (scan_col_csc_cuda_mono + scan_col_mono2,
//             cuda_kernels.cu:471-541, 835-918, which push only and keep uint32
//             sigma)
//   backward  one sweep per level d = D..1, each level-d vertex pulls
//             X(w) = (1 + delta_w) / sigma_w from its level-(d+1) neighbours:
//             delta_v = reach_v + sigma_v * sum X(w), then X(v) replaces sigma_v
//             in place and bc[v] += mult * delta_v (scan_frt_mono +
//             update_bc, cuda_kernels.cu:263-277, 546-599, which push float32
//             atomics)
//   end       bc[root] += pendant_sources * (W - 2) (the source term of
//             update_bc, cuda_kernels.cu:269-271, with W from
//             pre_update_bc_cuda's reduction, cuda_kernels.cu:312-336)
// Grid-wide barriers between sweeps are software barriers whose waits give up
// after Ctrl::wait_ns, set an error code and let every CTA return.
//
// State.  One row per vertex holds the S levels and the S values (RowGeom):
// a 32-byte row for S = 3, so one gathered sector answers both "is this
// neighbour at the wanted level" and "what is its value" for all slots.  With
// S = 3 the rows of a 1.5M-vertex graph take 47 MB and stay in the 126 MB L2
// while the adjacency streams past with an evict-first policy.  A neighbour's
// row is gathered with one 32-byte load per lane (two for S = 6): a scattered
// load costs the L1 one pass per distinct line it touches, so one 32-byte
// access per row halves those passes against two 16-byte ones.
//
// Work decomposition.  Vertices are cut into static tiles of <= 32
// consecutive vertices and <= kTileEdges (512) adjacency entries; a vertex
// with more entries is split into kTileEdges-entry chunks ("hub" chunks).
// One warp works on one tile at a time with no CTA-wide synchronisation: lane
// j owns vertex j, every active vertex's edges are cut into segments of
// kItems (4) edges aligned to the vertex's first edge, and the lanes take one
// segment each per round (32 segments a round).  Each warp pipelines its
// tiles: while it works on one tile, the next tile's adjacency range, own
// rows, degree/reach words and row starts are already being copied into the
// other half of its shared buffers by four 1-D bulk asynchronous copies
// (cp.async.bulk, completion on an mbarrier), and the descriptors of the two
// tiles after it are in registers.  A tile then costs one dependent round
// trip per round (the row gathers) instead of more for its own data.  Push
// and backward sweeps walk only the tiles on the level's list (tiles holding
// a vertex first reached at that level, for any slot; a sparse push splits
// each tile over kPushSplit warps); pull sweeps walk the tiles that still
// hold an unvisited vertex (all tiles in the first pull of a batch).
//
// Deterministic sums.  A vertex's sum over its neighbours (sigma of parents
// in a pull, X of children in the backward pass) is formed in a fixed order:
// each lane adds its segment's terms in adjacency order; the vertex's own
// lane folds its segment partials left to right after every round; a
// one-vertex tile sums lane-wise over the rounds and then over the lanes in
// a fixed butterfly; a hub's chunk totals are stored in one slot per chunk
// and added in chunk order by the chunk that arrives last.  The segments of
// a vertex depend on that vertex alone, and no floating-point atomic ever
// races another (the one such add, into bc, is made once per vertex per
// sweep, and sweeps are ordered by the grid barrier), so a run's results are
// bitwise reproducible and a source's contribution does not depend on the
// batch it shares.
//
// Child marks.  A backward sweep at level d reads every edge of every vertex
// of level d to find its children at level d + 1.  When level d + 1 holds far
// fewer pair-edges than level d (the last levels of a small-diameter graph),
// most vertices of level d have no child at all.  So the backward sweep of
// such a small level d + 1 also marks the parents it sees (level d in the same
// slot) with an atomic AND on the parent row's mark bits, and the sweep at
// level d then reads the edges of marked vertices only.  An unmarked vertex
// has no child in any of its slots: its sums are zero either way, so the
// results are bitwise the same.  Undirected graphs only (a directed graph's
// adjacency does not list the parents).
//
// Memory coherence.  The L1 caches of the SMs are not coherent with each
// other: a plain load can hit a line this SM cached in an earlier sweep or
// batch after another SM rewrote it in L2.  Everything that other SMs rewrite
// during a launch (state rows, level lists, the unvisited ring, bc, hub
// slots, tile marks) is therefore read with L2 loads (.cg, volatile or atomic)
// or copied by the bulk-copy engine, which reads L2.
#include <cstdio>

#include "bcg.h"
#include "bcg_common.hpp"
#include "engine.cuh"
#include "ext64.cuh"

namespace bcg {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long vload64(const unsigned long long *p) {
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

__device__ __forceinline__ uint32_t vload32(const uint32_t *p) {
    return *reinterpret_cast<const volatile uint32_t *>(p);
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// L2 policy for streamed data: evicted before the state rows.
__device__ __forceinline__ unsigned long long evict_first_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ unsigned long long evict_normal_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// ---- mbarrier + bulk copy (one 1-D async copy per tile adjacency range)
__device__ __forceinline__ void mbar_init(unsigned long long *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Copies [src, src + bytes) to dst (both 16-byte aligned, bytes a nonzero
// multiple of 16), completing `bytes` of transfer on the barrier at shared
// address bar.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, unsigned bar,
                                          unsigned long long pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(bar), "l"(pol)
        : "memory");
}
// Bounded wait for phase `parity` of the barrier; false when wait_ns ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity, unsigned long long wait_ns) {
    const unsigned b = smem_addr(bar);
    unsigned long long t0 = 0;
    for (uint32_t spins = 0;; ++spins) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(b), "r"(parity)
            : "memory");
        if (done) return true;
        if (spins == 0) t0 = global_ns();
        else if ((spins & 15u) == 0 && global_ns() - t0 > wait_ns) return false;
    }
}

// ---- loads of state rows into registers (rows are 16, 32 or 64 bytes, aligned)
template <int NW>
__device__ __forceinline__ void ld_row(const unsigned char *row, uint32_t (&w)[NW]) {
    if (NW == 4) {
        asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]) : "l"(row));
    } else {
#pragma unroll
        for (int h = 0; h < NW / 8; ++h)
            asm volatile("ld.global.cg.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(w[8 * h]), "=r"(w[8 * h + 1]), "=r"(w[8 * h + 2]), "=r"(w[8 * h + 3]), "=r"(w[8 * h + 4]),
                           "=r"(w[8 * h + 5]), "=r"(w[8 * h + 6]), "=r"(w[8 * h + 7])
                         : "l"(row + 32 * h));
    }
}
// The level block (first 8 or 16 bytes) of a row.
template <int NL>
__device__ __forceinline__ void ld_lvl(const unsigned char *row, uint32_t (&w)[NL]) {
    if (NL == 2)
        asm volatile("ld.global.cg.v2.u32 {%0,%1}, [%2];" : "=r"(w[0]), "=r"(w[1]) : "l"(row));
    else
        asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]) : "l"(row));
}

// Software grid barrier (all CTAs co-resident: cooperative launch).  One
// atomic per CTA on a monotone arrival counter: the k-th barrier of the
// launch is complete once the counter reaches k * nblocks, so nothing is
// reset between barriers.  Thread 0 also reads the error and overflow flags
// once, after every CTA has arrived, and hands the verdict to its CTA through
// shared memory.  Returns false when any CTA recorded an error or an overflow,
// in which case the caller returns.  The fence before the arrival and the
// acquire loads and fence after the wait order every write before the
// barrier (any CTA) before every read after it.  Data that other SMs rewrite
// between sweeps (state rows, level lists, the unvisited ring, bc, hub
// slots) is also always read with L2-coherent loads (.cg), never through a
// possibly stale L1 line.  A barrier does not hold the other CTAs back
// afterwards: the first CTA out may already work on the next sweep while the
// last one still reads the counters of the previous one.  So every value read
// after a barrier is one the next sweep does not write (the per-sweep counter
// rings of Ctrl, the level lists, each cleared two sweeps ahead).
__device__ bool grid_sync(Ctrl *c, unsigned int nblocks, unsigned long long wait_ns) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned long long arrived = atomicAdd(&c->bar_arrived, 1ull) + 1ull;
        const unsigned long long target = (arrived + nblocks - 1) / nblocks * nblocks;
        const volatile int *err = &c->error;
        if (arrived != target) {
            unsigned long long t0 = global_ns();
            unsigned int spins = 0;
            while (ld_acquire64(&c->bar_arrived) < target) {
                if ((++spins & 255u) == 0) {
                    if (*err) break;
                    if (global_ns() - t0 > wait_ns) {
                        atomicCAS(&c->error, 0, BCG_ERR_TIMEOUT);
                        break;
                    }
                }
                __nanosleep(32);
            }
        }
        // with the arrival fences of the other CTAs, this fence makes their
        // writes before the barrier visible to this CTA's reads after it
        __threadfence();
        ok = (*err == 0) && (*reinterpret_cast<volatile int *>(&c->overflow) == 0);
    }
    __syncthreads();
    return ok != 0;
}

// ---- state-row field access (row words: levels in halfwords, then values)
__device__ __forceinline__ uint16_t w_lvl(const uint32_t *w, int k) {
    return (uint16_t)(w[k >> 1] >> ((k & 1) * 16));
}
template <int S>
__device__ __forceinline__ unsigned long long w_val(const uint32_t *w, int k) {
    constexpr int b = RowGeom<S>::kValWord;
    return (unsigned long long)w[b + 2 * k] | ((unsigned long long)w[b + 2 * k + 1] << 32);
}
template <int S>
__device__ __forceinline__ unsigned char *row_of(const BatchArgs &a, uint32_t v) {
    return a.rows + (size_t)v * RowGeom<S>::kBytes;
}
__device__ __forceinline__ uint16_t *lvl_at(unsigned char *row, int k) {
    return reinterpret_cast<uint16_t *>(row) + k;
}
template <int S>
__device__ __forceinline__ unsigned long long *val_at(unsigned char *row, int k) {
    return reinterpret_cast<unsigned long long *>(row + RowGeom<S>::kLvlBytes) + k;
}

// Adjacency entries a tile buffer holds: the range [e0, e1) widened to
// 16-byte boundaries on both sides (<= 3 entries each).
constexpr int kAdjBuf = kTileEdges + 8;

static_assert((kAdjBuf * 4) % 16 == 0, "tile buffers keep 16-byte alignment");

// Per-warp scratch.
template <int S>
struct WarpSmem {
    alignas(128) uint32_t adjs[2][kAdjBuf];  // tile adjacency, double-buffered (bulk-copy targets)
    alignas(16) uint4 rows[2][kTileVerts * RowGeom<S>::kVec];  // the tile's own state rows (bulk-copy targets)
    alignas(16) uint2 vbuf[2][kTileVerts + 2];   // their {degree, reach} words, from an even vertex on
    alignas(16) uint32_t obuf[2][kTileVerts + 8];  // their row starts, from a multiple-of-4 vertex on
    unsigned long long mbar[2];              // completion of the four copies of buffer b
    uint4 vmeta[kTileVerts];                 // {first segment, edge start in adjs, edges, active slots}
    unsigned long long part[32][S];          // the round's segment partial sums, by lane
    unsigned char sown[kTileEdges / kItems + kTileVerts];  // vertex of each segment of the tile
    uint32_t app[2 * 32];   // buffered appends to the next level's list
    uint32_t uapp[2 * 32];  // buffered appends to the unvisited-tile ring
    uint32_t napp, nuapp;
    unsigned long long acc[kTileVerts][S];   // per-vertex sums of the tile
    unsigned long long own[kTileVerts][S];   // push: sigma of the frontier vertex's active slots
    // per-warp discovery totals of the sweep (LaneCounts layout)
    unsigned long long cnt[2 + 3 * S];
};

// Levels whose backward sweep may mark parents (a per-CTA bit each).
constexpr uint32_t kMarkLevels = 2048;

template <int S>
struct Smem {
    WarpSmem<S> w[SweepGeom<S>::kWarps];
    // per-CTA counters of the current sweep
    unsigned long long c_disc, c_pf;
    unsigned long long c_vis[S], c_w[S], c_mc[S];
    // batch constants
    uint32_t roots[S];
    double mult[S];
    uint32_t next;  // work items drawn by this CTA's warps in the current sweep
    uint32_t mlev[kMarkLevels / 32];  // levels whose backward sweep marks parents
};

template <int S>
size_t smem_bytes() { return sizeof(Smem<S>); }

// A tile descriptor held one 32-bit word per lane (lanes 0..7), so a warp's
// pipeline of drawn tiles costs one register per tile; unpacked by shuffles
// when the tile comes up.
__device__ __forceinline__ uint32_t tile_word(const Tile *tiles, uint32_t ti) {
    const unsigned lane = threadIdx.x & 31;
    return lane < 8 ? reinterpret_cast<const uint32_t *>(tiles + ti)[lane] : 0u;
}
__device__ __forceinline__ Tile tile_unpack(uint32_t tw) {
    Tile T;
    T.v0 = __shfl_sync(0xffffffffu, tw, 0);
    T.v1 = __shfl_sync(0xffffffffu, tw, 1);
    T.e0 = __shfl_sync(0xffffffffu, tw, 2);
    T.e1 = __shfl_sync(0xffffffffu, tw, 3);
    T.hub = (int32_t)__shfl_sync(0xffffffffu, tw, 4);
    T.nchunks = __shfl_sync(0xffffffffu, tw, 5);
    T.hslot = __shfl_sync(0xffffffffu, tw, 6);
    T.hchunk = __shfl_sync(0xffffffffu, tw, 7);
    return T;
}

// Parameters of one sweep, identical in every warp.
struct SweepCtx {
    int mode;
    uint32_t b;          // batch
    uint32_t d, D;
    uint32_t key_next;   // tile mark of (batch, level d+1)
    uint32_t lb_next;    // list start of level d+1
    uint32_t next_lvl;   // d + 1 (index into lcnt)
    uint32_t split;      // warps per tile (push sweeps over short lists)
    unsigned long long ubase;  // ring position of this sweep's first unvisited-tile append
    bool mark;           // backward: mark the parents (level d - 1) of level d's vertices
    bool filt;           // backward: level d + 1 marked its parents; read marked vertices only
};


__device__ __forceinline__ uint32_t tile_key(uint32_t b, uint32_t level) {
    return ((b & 0xFFFFu) << 16) | (level + 1u);
}

__device__ __forceinline__ void set_error(Ctrl *c, int code) { atomicCAS(&c->error, 0, code); }

// Appends one sweep-trace record (CTA 0, thread 0, right after a barrier).
__device__ __forceinline__ void trace(const BatchArgs &a, uint32_t b, uint32_t kind, uint32_t level,
                                      uint32_t nwork, unsigned long long disc) {
    if (!a.trace || blockIdx.x != 0 || threadIdx.x != 0) return;
    const unsigned int i = *a.trace_cnt;
    if (i >= a.trace_cap) return;
    TraceRec r;
    r.t_ns = global_ns();
    r.batch = b;
    r.kind = kind;
    r.level = level;
    r.nwork = nwork;
    r.disc = disc;
    a.trace[i] = r;
    *a.trace_cnt = i + 1;
}

// Writes the warp's buffered level-list appends to the global list.
template <int S>
__device__ __forceinline__ void flush_level(const BatchArgs &a, WarpSmem<S> &ws, uint32_t cnt, const SweepCtx &x) {
    const unsigned lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(a.lcnt + x.next_lvl, cnt);
    base = __shfl_sync(0xffffffffu, base, 0);
    if ((unsigned long long)x.lb_next + base + cnt > a.list_cap) {
        if (lane == 0) set_error(a.ctrl, BCG_ERR_OOM);
    } else {
        for (uint32_t i = lane; i < cnt; i += 32) a.lists[x.lb_next + base + i] = ws.app[i];
    }
    __syncwarp();
}

// Writes the warp's buffered unvisited-tile appends to the ring: the sweep's
// appends occupy ring positions x.ubase, x.ubase + 1, ... (its counter
// uadd[d % 4] hands them out).
template <int S>
__device__ __forceinline__ void flush_unvisited(const BatchArgs &a, WarpSmem<S> &ws, uint32_t cnt, const SweepCtx &x) {
    const unsigned lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&a.ctrl->uadd[x.d & 3], (unsigned long long)cnt);
    base = __shfl_sync(0xffffffffu, base, 0) + x.ubase;
    const unsigned long long ring = 2ull * a.ntiles;
    for (uint32_t i = lane; i < cnt; i += 32) a.ulist[(base + i) % ring] = ws.uapp[i];
    __syncwarp();
}

// Appends tile t (kNoTile: nothing) of this lane to level d+1's list.  All
// 32 lanes must call it together.  Hubs (kHubFlag) expand to all chunks.
template <int S>
__device__ __forceinline__ void append_level(const BatchArgs &a, WarpSmem<S> &ws, uint32_t t, const SweepCtx &x) {
    const unsigned lane = threadIdx.x & 31;
    if (t != kNoTile && (t & kHubFlag)) {
        const uint32_t t0 = t & ~kHubFlag;
        const uint32_t nch = a.tiles[t0].nchunks;
        const uint32_t base = atomicAdd(a.lcnt + x.next_lvl, nch);
        if ((unsigned long long)x.lb_next + base + nch > a.list_cap) {
            set_error(a.ctrl, BCG_ERR_OOM);
        } else {
            for (uint32_t c = 0; c < nch; ++c) a.lists[x.lb_next + base + c] = t0 + c;
        }
        t = kNoTile;
    }
    const unsigned want = __ballot_sync(0xffffffffu, t != kNoTile);
    if (!want) return;
    uint32_t cnt = ws.napp;
    if (t != kNoTile) ws.app[cnt + __popc(want & ((1u << lane) - 1u))] = t;
    cnt += __popc(want);
    __syncwarp();
    if (cnt >= 32) {
        flush_level<S>(a, ws, cnt, x);
        cnt = 0;
    }
    if (lane == 0) ws.napp = cnt;
    __syncwarp();
}

// Appends tile t (kNoTile: nothing; kHubFlag: all chunks) to the ring of tiles
// that still hold unvisited vertices.  All 32 lanes call it together.
template <int S>
__device__ __forceinline__ void append_unvisited(const BatchArgs &a, WarpSmem<S> &ws, uint32_t t, const SweepCtx &x) {
    const unsigned lane = threadIdx.x & 31;
    if (t != kNoTile && (t & kHubFlag)) {
        const uint32_t t0 = t & ~kHubFlag;
        const uint32_t nch = a.tiles[t0].nchunks;
        const unsigned long long base = x.ubase + atomicAdd(&a.ctrl->uadd[x.d & 3], (unsigned long long)nch);
        const unsigned long long ring = 2ull * a.ntiles;
        for (uint32_t c = 0; c < nch; ++c) a.ulist[(base + c) % ring] = t0 + c;
        t = kNoTile;
    }
    const unsigned want = __ballot_sync(0xffffffffu, t != kNoTile);
    if (!want) return;
    uint32_t cnt = ws.nuapp;
    if (t != kNoTile) ws.uapp[cnt + __popc(want & ((1u << lane) - 1u))] = t;
    cnt += __popc(want);
    __syncwarp();
    if (cnt >= 32) {
        flush_unvisited<S>(a, ws, cnt, x);
        cnt = 0;
    }
    if (lane == 0) ws.nuapp = cnt;
    __syncwarp();
}

// Claims the tile of a vertex reached at level d+1 for the next list: returns
// the tile to append (with kHubFlag for hubs) or kNoTile if already listed.
__device__ __forceinline__ uint32_t claim_tile(const BatchArgs &a, uint32_t w, uint32_t key) {
    const uint32_t tf = a.tile_of[w];
    const uint32_t t = tf & ~kHubFlag;
    if (vload32(a.tmark + t) == key) return kNoTile;
    if (atomicExch(a.tmark + t, key) == key) return kNoTile;
    return tf;
}

// Discovery counters of one lane over one tile: (vertex, slot) pairs
// discovered, their degrees, and per slot the count, sum of (1 + reach) and
// sum of (deg + 2 reach).  32-bit: a lane discovers at most 8 * S pairs per tile.
template <int S>
struct LaneCounts {
    uint32_t disc = 0, pf = 0;
    uint32_t vis[S] = {}, w[S] = {}, mc[S] = {};
    __device__ __forceinline__ void add(int k, uint2 info) {
        ++disc;
        pf += info.x;
        ++vis[k];
        w[k] += 1u + info.y;
        mc[k] += info.x + 2u * info.y;
    }
};

// Warp sum of 32-bit values without overflow (16-bit halves reduced apart).
__device__ __forceinline__ unsigned long long warp_sum32(uint32_t x) {
    return (unsigned long long)__reduce_add_sync(0xffffffffu, x & 0xFFFFu) +
           ((unsigned long long)__reduce_add_sync(0xffffffffu, x >> 16) << 16);
}

// Adds the warp's tile counters to its per-warp totals (all lanes call it).
template <int S>
__device__ __forceinline__ void flush_counts(WarpSmem<S> &ws, const LaneCounts<S> &c) {
    if (!__any_sync(0xffffffffu, c.disc != 0)) return;
    const unsigned long long disc = warp_sum32(c.disc), pf = warp_sum32(c.pf);
    unsigned long long vis[S], w[S], mc[S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        vis[k] = warp_sum32(c.vis[k]);
        w[k] = warp_sum32(c.w[k]);
        mc[k] = warp_sum32(c.mc[k]);
    }
    if ((threadIdx.x & 31) == 0) {
        ws.cnt[0] += disc;
        ws.cnt[1] += pf;
#pragma unroll
        for (int k = 0; k < S; ++k) {
            ws.cnt[2 + k] += vis[k];
            ws.cnt[2 + S + k] += w[k];
            ws.cnt[2 + 2 * S + k] += mc[k];
        }
    }
    __syncwarp();
}

// A wrapped uint64 sum: flag it (a plain store keeps the unrolled sum sites
// small); every CTA leaves at the next grid barrier, and the host fails the
// run or redoes it with extended counts.
__device__ __forceinline__ void flag_overflow(Ctrl *c) { c->overflow = 1; }

// Value arithmetic of a sweep.  Forward sweeps sum sigma values, backward
// sweeps sum X = (1 + delta) / sigma values; with EXT both are extended-range
// numbers (ext64.cuh), otherwise sigma is an exact uint64 (a wrapped sum sets
// the overflow flag) and X a double.  vsum(x, y) adds y after x.
template <bool EXT, int MODE>
__device__ __forceinline__ unsigned long long vsum(unsigned long long x, unsigned long long y, const BatchArgs &a) {
    if (EXT) return ext_add(x, y);
    if (MODE == kBwd)
        return (unsigned long long)__double_as_longlong(__longlong_as_double((long long)x) +
                                                        __longlong_as_double((long long)y));
    const unsigned long long t = x + y;
    if (t < y) flag_overflow(a.ctrl);
    return t;
}

// *p += y atomically in global memory (push sweeps: integer sigma, or the
// extended form as a compare-and-swap retry loop; each failed attempt means
// another thread's add went through, so the loop always ends).  Integer and
// extended sums of exact counts do not depend on the order of the adds.
// Returns the value before the add: 0 only for the first add to a vertex not
// reached before (every sigma added is at least 1; a wrapped sum sets the
// overflow flag, and the run is then redone with extended counts).
template <bool EXT>
__device__ __forceinline__ unsigned long long sigma_add_old(unsigned long long *p, unsigned long long y,
                                                            const BatchArgs &a) {
    if (EXT) {
        unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(p), seen;
        do {
            seen = old;
            old = atomicCAS(p, seen, ext_add(seen, y));
        } while (old != seen);
        return seen;
    }
    const unsigned long long old = atomicAdd(p, y);
    if (old + y < y) flag_overflow(a.ctrl);
    return old;
}

// One tile (or one part of a split tile), processed by one warp.  The tile's
// adjacency (copied from entry T.e0 & ~3 on), own rows, degree/reach words
// and row starts are in buffer `buf` of the warp's scratch (tile_fetch).
//
// Work split.  Every active vertex's edges are cut into segments of kItems
// edges aligned to the vertex's first edge; each lane takes one segment per
// round (its vertex from a per-tile segment map).  A vertex's segments
// depend on the vertex alone, not on which other vertices are active.  A
// lane adds its segment's terms in adjacency order, and the segment partials
// of a vertex are
// folded left to right in segment order by the vertex's own lane after every
// round (in a one-vertex tile: lane-wise over the rounds, then over the lanes
// by a fixed butterfly): the same bits whatever the batch's other slots did.
template <int S, int MODE, bool EXT>
__device__ void warp_tile(const BatchArgs &a, Smem<S> &sm, WarpSmem<S> &ws, uint32_t ti, const Tile &T,
                          uint32_t part, const SweepCtx &x, int buf) {
    constexpr int NW = RowGeom<S>::kWords;
    constexpr int NV = RowGeom<S>::kVec;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t d = x.d;
    const uint16_t dl = (uint16_t)d;
    const bool hub = T.hub >= 0;
    const uint32_t nv = T.v1 - T.v0;
    const uint32_t *adjs = ws.adjs[buf];
    const uint32_t ab = T.e0 & ~3u;
    // the lane's own row, as copied with the tile (levels, and sigma of the
    // slots whose level is d); read again from the buffer where needed
    auto own_row = [&](uint32_t (&ow)[NW]) {
#pragma unroll
        for (int h = 0; h < NV; ++h) {
            const uint4 t = ws.rows[buf][lane * NV + h];
            ow[4 * h] = t.x; ow[4 * h + 1] = t.y; ow[4 * h + 2] = t.z; ow[4 * h + 3] = t.w;
        }
    };
    // the lane's degree/reach word and row start, as copied with the tile
    uint2 vi = make_uint2(0u, 0u);
    uint32_t ob = 0;
    if (lane < nv) {
        vi = ws.vbuf[buf][(T.v0 & 1u) + lane];
        ob = ws.obuf[buf][(T.v0 & 3u) + lane];
    }
    // ---- phase 1: the lane's vertex
    uint32_t m = 0, dg = 0;
    if (lane < nv) {
        uint32_t ow[NW];
        own_row(ow);
#pragma unroll
        for (int k = 0; k < S; ++k) {
            const uint16_t L = w_lvl(ow, k);
            if (MODE == kFwdPull) m |= (uint32_t)(L == kUnvisited) << k;
            else m |= (uint32_t)(L == dl) << k;
        }
        if (MODE == kFwdPull && vi.x == 0) m = 0;  // no edge: cannot be reached
        const uint32_t eb = hub ? T.e0 : ob;
        uint32_t ee = ob + vi.x;
        if (hub && T.e1 < ee) ee = T.e1;
        if (ee < eb) ee = eb;
        if (m) dg = ee - eb;
        if (MODE == kBwd) {
            // a vertex with no child in any slot reads no edge (the deepest
            // level has none), unless its sweep marks parents
            const uint32_t mk = ~(ow[RowGeom<S>::kMarkWord] >> RowGeom<S>::kMarkShift) & ((1u << S) - 1u);
            if (!x.mark && (d == x.D || (x.filt && !(m & mk)))) dg = 0;
        }
        ws.vmeta[lane].y = eb - ab;
        ws.vmeta[lane].z = dg;
        if (MODE == kFwdPush) {
#pragma unroll
            for (int k = 0; k < S; ++k) ws.own[lane][k] = ((m >> k) & 1u) ? w_val<S>(ow, k) : 0ull;
        }
        ws.vmeta[lane].w = m;
    }
    if (hub && !__shfl_sync(0xffffffffu, m, 0)) return;  // same decision in every chunk
    // segment prefix
    const uint32_t nseg = (dg + kItems - 1) / kItems;
    uint32_t incl = nseg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (lane < nv) ws.vmeta[lane].x = incl - nseg;
    // segment -> vertex map (one-vertex tiles need none)
    if (nv > 1)
        for (uint32_t p = incl - nseg; p < incl; ++p) ws.sown[p] = (unsigned char)lane;
    __syncwarp();

    // ---- phase 2: segments [s0, s1) of this part, one per lane per round
    uint32_t s0 = 0, s1 = total;
    if (MODE == kFwdPush && x.split > 1) {
        s0 = (uint32_t)(((unsigned long long)total * part) / x.split);
        s1 = (uint32_t)(((unsigned long long)total * (part + 1)) / x.split);
    }
    constexpr uint32_t kSkipItem = 0xFFFFFFFFu;
    // one-vertex tiles keep their partials in registers, summed round by round
    const bool solo = (nv == 1);
    unsigned long long ls[S];
#pragma unroll
    for (int k = 0; k < S; ++k) ls[k] = 0ull;
    // the lane's own vertex: its segments and the running fold of their sums
    const uint32_t myp0 = incl - nseg, myp1 = incl;
    if (MODE == kFwdPush) {
        // Pushes add integers with atomics, so their order is free: the part's
        // (segment, edge) pairs are spread over all lanes, K = ceil(pairs /
        // 32) <= kItems consecutive pairs per lane and round, so a sparse part
        // keeps every lane busy with one edge instead of a few lanes with a
        // whole segment each.
        constexpr int NL = RowGeom<S>::kLvlBytes / 4;
        const uint32_t np = (uint32_t)kItems * (s1 - s0);
        const uint32_t K = min((uint32_t)kItems, (np + 31u) / 32u);
        for (uint32_t p0 = 0; p0 < np; p0 += 32u * K) {
            uint32_t uu[kItems], jq[kItems];
#pragma unroll
            for (int q = 0; q < kItems; ++q) {
                uu[q] = kSkipItem;
                jq[q] = 0;
                const uint32_t pp = p0 + lane * K + (uint32_t)q;
                if ((uint32_t)q < K && pp < np) {
                    const uint32_t seg = s0 + pp / kItems;
                    const uint32_t j = solo ? 0u : ws.sown[seg];
                    const uint4 vm = ws.vmeta[j];
                    const uint32_t rr = (seg - vm.x) * kItems + pp % kItems;
                    if (rr < vm.z && vm.w) {
                        uu[q] = adjs[vm.y + rr];
                        jq[q] = j;
                    }
                }
            }
            // the targets' level blocks, then the sigma adds (the first add to
            // a vertex claims it)
            LaneCounts<S> lc;
            uint32_t lw[kItems][NL];
#pragma unroll
            for (int q = 0; q < kItems; ++q)
                if (uu[q] != kSkipItem) ld_lvl<NL>(row_of<S>(a, uu[q]), lw[q]);
#pragma unroll
            for (int q = 0; q < kItems; ++q) {
                uint32_t app = kNoTile;
                if (uu[q] != kSkipItem) {
                    const uint32_t wv = uu[q], jm = ws.vmeta[jq[q]].w;
                    unsigned char *wrow = row_of<S>(a, wv);
                    bool claimed_any = false;
#pragma unroll
                    for (int k = 0; k < S; ++k) {
                        if (!((jm >> k) & 1u)) continue;
                        const uint16_t L = w_lvl(lw[q], k);
                        // unvisited, or reached at d + 1 in this sweep: a DAG
                        // edge either way (levels only move from unvisited to
                        // d + 1 during a push); the add that finds sigma still
                        // 0 is the first, and its lane claims the vertex
                        if (L != (uint16_t)(d + 1) && L != kUnvisited) continue;
                        if (sigma_add_old<EXT>(val_at<S>(wrow, k), ws.own[jq[q]][k], a) == 0ull) {
                            *lvl_at(wrow, k) = (uint16_t)(d + 1);
                            lc.add(k, a.vinfo[wv]);
                            claimed_any = true;
                        }
                    }
                    if (claimed_any) app = claim_tile(a, wv, x.key_next);
                }
                append_level<S>(a, ws, app, x);
            }
            flush_counts<S>(ws, lc);
        }
    }
    // (push parts were done above)
    for (uint32_t r0 = s0; MODE != kFwdPush && r0 < s1; r0 += 32) {
        const uint32_t seg = r0 + lane;
        const bool has = seg < s1;
        uint32_t j = 0, cnt = 0, e0 = 0, jm = 0;
        if (has) {
            j = solo ? 0u : ws.sown[seg];
            const uint4 vm = ws.vmeta[j];
            const uint32_t rr = (seg - vm.x) * kItems;
            cnt = min((uint32_t)kItems, vm.z - rr);
            e0 = vm.y + rr;
            jm = vm.w;
        }
        uint32_t uu[kItems];
#pragma unroll
        for (int q = 0; q < kItems; ++q) uu[q] = ((uint32_t)q < cnt && jm) ? adjs[e0 + q] : kSkipItem;
        {
            // gather the neighbours' rows (kHalf at a time: all 8 for rows of
            // up to 32 bytes, 4 for 64-byte rows) and sum the matching values
            // in adjacency order
            constexpr int kHalf = (NW <= 8) ? kItems : kItems / 2;
            const uint16_t want = (MODE == kFwdPull) ? dl : (uint16_t)(d + 1);
            const uint16_t par = (uint16_t)(d - 1);  // parents, in a marking backward sweep
            bool ovf = false;  // a wrapped uint64 sum (flagged once per round)
            auto add = [&](unsigned long long x, unsigned long long y) -> unsigned long long {
                if (EXT) return ext_add(x, y);
                if (MODE == kBwd)
                    return (unsigned long long)__double_as_longlong(__longlong_as_double((long long)x) +
                                                                    __longlong_as_double((long long)y));
                const unsigned long long t = x + y;
                ovf |= t < y;
                return t;
            };
            unsigned long long run[S];
#pragma unroll
            for (int k = 0; k < S; ++k) run[k] = 0ull;
#pragma unroll
            for (int h0 = 0; h0 < kItems; h0 += kHalf) {
                uint32_t wr[kHalf][NW];
#pragma unroll
                for (int q = 0; q < kHalf; ++q)
                    if (uu[h0 + q] != kSkipItem) ld_row<NW>(row_of<S>(a, uu[h0 + q]), wr[q]);
#pragma unroll
                for (int q = 0; q < kHalf; ++q) {
                    if (uu[h0 + q] == kSkipItem) continue;
#pragma unroll
                    for (int k = 0; k < S; ++k) {
                        if (!((jm >> k) & 1u) || w_lvl(wr[q], k) != want) continue;
                        run[k] = add(run[k], w_val<S>(wr[q], k));
                    }
                    if (MODE == kBwd && x.mark) {
                        // the neighbour is a parent in the slots where it sits
                        // one level up; mark the slots it does not show marked yet
                        uint32_t pm = 0;
#pragma unroll
                        for (int k = 0; k < S; ++k)
                            pm |= (uint32_t)(((jm >> k) & 1u) && w_lvl(wr[q], k) == par) << k;
                        pm &= wr[q][RowGeom<S>::kMarkWord] >> RowGeom<S>::kMarkShift;
                        if (pm)
                            atomicAnd(reinterpret_cast<unsigned int *>(row_of<S>(a, uu[h0 + q])) +
                                          RowGeom<S>::kMarkWord,
                                      ~(pm << RowGeom<S>::kMarkShift));
                    }
                }
            }
            if (!EXT && MODE != kBwd && ovf) flag_overflow(a.ctrl);
            if (solo) {
#pragma unroll
                for (int k = 0; k < S; ++k) ls[k] = vsum<EXT, MODE>(ls[k], run[k], a);
            } else {
                if (has) {
#pragma unroll
                    for (int k = 0; k < S; ++k) ws.part[lane][k] = run[k];
                }
                __syncwarp();
                // each vertex's lane folds in its segments of this round, in order
                const uint32_t q0 = max(myp0, r0), q1 = min(myp1, r0 + 32u);
                for (uint32_t q = q0; q < q1; ++q) {
#pragma unroll
                    for (int k = 0; k < S; ++k) ls[k] = vsum<EXT, MODE>(ls[k], ws.part[q - r0][k], a);
                }
                __syncwarp();
            }
        }
    }
    __syncwarp();
    if (MODE == kFwdPush) return;

    // ---- each vertex's total over its segments, in segment order
    if (solo) {
        // lane l held segments l, l + 32, ... (rounds in order); the lanes'
        // sums meet in a fixed butterfly, every lane ending with the total
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
#pragma unroll
            for (int k = 0; k < S; ++k) ls[k] = vsum<EXT, MODE>(ls[k], __shfl_xor_sync(0xffffffffu, ls[k], o), a);
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < S; ++k) ws.acc[0][k] = ls[k];
        }
    } else if (lane < nv) {
#pragma unroll
        for (int k = 0; k < S; ++k) ws.acc[lane][k] = ls[k];
    }
    __syncwarp();

    // ---- hub chunks: each chunk stores its total in its own slot; the chunk
    // that arrives last adds the slots in chunk order and finishes the vertex
    if (hub) {
        unsigned long long *slot0 = a.hub_acc + (size_t)(T.hslot - T.hchunk) * S;
        uint32_t last = 0;
        if (lane == 0) {
            // one thread stores the chunk's slot, fences and arrives (a release)
#pragma unroll
            for (int k = 0; k < S; ++k) __stcg(slot0 + (size_t)T.hchunk * S + k, ws.acc[0][k]);
            __threadfence();
            last = (atomicAdd(a.hub_cnt + T.hub, 1u) == T.nchunks - 1);
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (!last) return;
        __threadfence();
        if (lane < (unsigned)S) {
            unsigned long long s = __ldcg(slot0 + lane);
            for (uint32_t c = 1; c < T.nchunks; ++c) s = vsum<EXT, MODE>(s, __ldcg(slot0 + (size_t)c * S + lane), a);
            ws.acc[0][lane] = s;
        }
        if (lane == 0) atomicExch(a.hub_cnt + T.hub, 0u);
        __syncwarp();
    }

    // ---- phase 3: finish the tile's vertices
    uint32_t nd = 0, left = 0;
    LaneCounts<S> cnt;
    if (lane < nv && m) {
        const uint32_t v = T.v0 + lane;
        unsigned char *vrow = row_of<S>(a, v);
        if (MODE == kFwdPull) {
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (!((m >> k) & 1u)) continue;
                const unsigned long long s = ws.acc[lane][k];
                if (!s) {
                    ++left;
                    continue;
                }
                *lvl_at(vrow, k) = (uint16_t)(d + 1);
                *val_at<S>(vrow, k) = s;
                ++nd;
                cnt.add(k, vi);
            }
        } else {
            double add = 0.0;
            const double reach = (double)vi.y;
            uint32_t ow[NW];
            own_row(ow);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (!((m >> k) & 1u)) continue;
                double delta;
                const unsigned long long sgv = w_val<S>(ow, k);
                if (EXT) {
                    // sigma * sum X is a dependency count (in double range)
                    // even where sigma and X are not
                    delta = reach + ext_to_double(ext_mul(sgv, ws.acc[lane][k]));
                    *val_at<S>(vrow, k) = ext_div(1.0 + delta, sgv);
                } else {
                    const double sig = (double)sgv;
                    const double acc = __longlong_as_double((long long)ws.acc[lane][k]);
                    delta = reach + sig * acc;
                    const double xo = (1.0 + delta) / sig;
                    *val_at<S>(vrow, k) = (unsigned long long)__double_as_longlong(xo);
                }
                if (d > 0) {
                    // served waves keep each slot's dependencies apart (added
                    // to the requests in slot order at the batch's end)
                    if (a.slot_delta) a.slot_delta[(size_t)k * a.n + v] = delta;
                    else add += sm.mult[k] * delta;
                }
                if (a.dbg_delta) a.dbg_delta[((size_t)x.b * S + k) * a.n + v] = delta;
            }
            if (d > 0 && !a.slot_delta) {
                // one add per vertex per sweep (one warp finishes a vertex), and
                // sweeps are ordered by the grid barrier: the adds reach bc[v]
                // in sweep order, the same bits as a load-add-store, without
                // waiting for the load
                atomicAdd(a.bc + (a.ext ? a.ext[v] : v), add);
            }
        }
    }
    if (MODE == kFwdPull) {
        flush_counts<S>(ws, cnt);
        // a pull sweep visits every listed tile once, so no mark is needed; a
        // hub is listed by its finishing chunk (first chunk | kHubFlag expands it)
        const uint32_t me = hub ? a.tile_of[T.v0] : ti;
        const bool any = __any_sync(0xffffffffu, nd > 0);
        append_level<S>(a, ws, (any && lane == 0) ? me : kNoTile, x);
        const bool keep = __any_sync(0xffffffffu, left > 0);
        append_unvisited<S>(a, ws, (keep && lane == 0) ? me : kNoTile, x);
    }
}

// Starts the copy of tile T's data into buffer `buf` of the warp and its
// lanes' registers: the adjacency range (one bulk copy by lane 0) and, per
// lane, the row, degree/reach word and row start of vertex T.v0 + lane.
// Four 1-D bulk copies, issued by lane 0 and completing on the buffer's
// mbarrier: the adjacency range [e0, e1) from e0 & ~3 on (up to 3 entries
// either side: the adjacency has a 4-entry tail pad), the rows of [v0, v1),
// their {degree, reach} words from v0 & ~1 on and their row starts from
// v0 & ~3 on (vinfo and offs have 4 entries of tail padding).  Every source
// and destination is 16-byte aligned and every size a multiple of 16.
template <int S>
__device__ __forceinline__ void tile_fetch(const BatchArgs &a, WarpSmem<S> &ws, int buf, uint32_t tw,
                                           unsigned long long pol) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t v0 = __shfl_sync(0xffffffffu, tw, 0), v1 = __shfl_sync(0xffffffffu, tw, 1);
    const uint32_t e0 = __shfl_sync(0xffffffffu, tw, 2), e1 = __shfl_sync(0xffffffffu, tw, 3);
    __syncwarp();  // every lane is done with the buffer's previous tile
    if (lane == 0) {
        const uint32_t ab = e0 & ~3u, ae = (e1 + 3u) & ~3u;
        const uint32_t vb = v0 & ~1u, ve = (v1 + 1u) & ~1u;
        const uint32_t obb = v0 & ~3u, obe = (v1 + 3u) & ~3u;
        const uint32_t abytes = (ae - ab) * 4u;
        const uint32_t rbytes = (v1 - v0) * (uint32_t)RowGeom<S>::kBytes;
        const uint32_t vbytes = (ve - vb) * 8u;
        const uint32_t obytes = (obe - obb) * 4u;
        const unsigned b = smem_addr(&ws.mbar[buf]);
        // rows were written by other CTAs' generic stores before the last
        // grid barrier: make them visible to the async proxy, and order this
        // warp's reads of the buffer before its refill
        asm volatile("fence.proxy.async.global;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b),
                     "r"(abytes + rbytes + vbytes + obytes)
                     : "memory");
        if (abytes) bulk_copy(ws.adjs[buf], a.adj + ab, abytes, b, pol);
        bulk_copy(ws.rows[buf], row_of<S>(a, v0), rbytes, b, evict_normal_policy());
        bulk_copy(ws.vbuf[buf], a.vinfo + vb, vbytes, b, evict_normal_policy());
        bulk_copy(ws.obuf[buf], a.offs + obb, obytes, b, evict_normal_policy());
    }
}

// Runs one sweep: the grid walks the work items, item i being
// list[(start + i) % ring] (or tile i when list is null); with x.split > 1
// each item is cut into x.split parts handed to different warps.  CTA b owns
// items b, b + G, b + 2G, ... (G CTAs: every CTA gets a slice of every region
// of the list), and its warps take them one at a time from a shared counter
// (sm.next, zeroed before the sweep), so a warp that drew cheap tiles keeps
// working instead of waiting at the sweep's barrier.
// With no list and a range table, item i is tile ranges[r].x + (i - ranges[r].y)
// for the last range r with ranges[r].y <= i (nranges ranges, increasing .y).
// Each warp keeps a pipeline of drawn items: the tile being worked on, the
// next one (its adjacency, rows, degree words and row starts in flight to the
// other buffer), the one after (descriptor loaded) and one more (list entry
// loaded).
// pstate holds the warp's buffer phases (bits 0, 1) and next buffer (bit 2)
// across sweeps.  A copy that does not arrive within wait_ns sets
// BCG_ERR_TIMEOUT and ends the warp's part of the sweep.
template <int S, bool EXT>
__device__ __forceinline__ void run_sweep(const BatchArgs &a, Smem<S> &sm, const SweepCtx &x, const uint32_t *list,
                                          unsigned long long start, uint32_t nwork, unsigned long long ring,
                                          uint32_t &pstate, unsigned long long wait_ns,
                                          const uint2 *ranges = nullptr, uint32_t nranges = 0) {
    const unsigned wid = threadIdx.x >> 5;
    WarpSmem<S> &ws = sm.w[wid];
    if ((threadIdx.x & 31) == 0) {
        ws.napp = 0;
        ws.nuapp = 0;
#pragma unroll
        for (int q = 0; q < 2 + 3 * S; ++q) ws.cnt[q] = 0ull;
    }
    __syncwarp();
    // item numbers fit 32 bits: a sweep's work list holds at most 2^31 tiles
    const uint32_t nitems = nwork * x.split;
    auto item_tile = [&](uint32_t it) -> uint32_t {
        const uint32_t i = it / x.split;
        if (list) return __ldcg(list + (start + i) % ring);
        if (!ranges) return i;
        uint32_t lo = 0, hi = nranges;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (ranges[mid].y <= i) lo = mid; else hi = mid;
        }
        const uint2 r = ranges[lo];
        return r.x + (i - r.y);
    };
    const unsigned long long G = gridDim.x;
    auto grab = [&]() -> uint32_t {
        uint32_t c = 0;
        if ((threadIdx.x & 31) == 0) c = atomicAdd(&sm.next, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        const unsigned long long it = blockIdx.x + (unsigned long long)c * G;
        return it < nitems ? (uint32_t)it : nitems;
    };
    const unsigned long long pol = evict_first_policy();
    uint32_t itA = grab();
    if (itA < nitems) {
        int buf = (pstate >> 2) & 1;
        uint32_t tiA = item_tile(itA);
        uint32_t twA = tile_word(a.tiles, tiA);
        uint32_t itB = grab();
        uint32_t tiB = (itB < nitems) ? item_tile(itB) : 0u;
        tile_fetch<S>(a, ws, buf, twA, pol);
        uint32_t twB = (itB < nitems) ? tile_word(a.tiles, tiB) : 0u;
        uint32_t itC = (itB < nitems) ? grab() : nitems;
        uint32_t tiC = (itC < nitems) ? item_tile(itC) : 0u;
        for (;;) {
            if (itB < nitems) tile_fetch<S>(a, ws, buf ^ 1, twB, pol);
            const uint32_t twC = (itC < nitems) ? tile_word(a.tiles, tiC) : 0u;
            const uint32_t itD = (itC < nitems) ? grab() : nitems;
            const uint32_t tiD = (itD < nitems) ? item_tile(itD) : 0u;
            const bool got = mbar_wait(&ws.mbar[buf], (pstate >> buf) & 1u, wait_ns);
            pstate ^= 1u << buf;
            if (!__all_sync(0xffffffffu, got)) {
                // a copy that never arrived: record it, give the copy still in
                // flight one more bounded wait, and leave the sweep
                if ((threadIdx.x & 31) == 0) set_error(a.ctrl, BCG_ERR_TIMEOUT);
                if (itB < nitems) {
                    mbar_wait(&ws.mbar[buf ^ 1], (pstate >> (buf ^ 1)) & 1u, wait_ns);
                    pstate ^= 1u << (buf ^ 1);
                }
                __syncwarp();
                pstate = (pstate & 3u) | ((uint32_t)buf << 2);
                break;
            }
            const Tile TA = tile_unpack(twA);
            const uint32_t part = itA % x.split;
            if (x.mode == kFwdPush) warp_tile<S, kFwdPush, EXT>(a, sm, ws, tiA, TA, part, x, buf);
            else if (x.mode == kFwdPull) warp_tile<S, kFwdPull, EXT>(a, sm, ws, tiA, TA, 0, x, buf);
            else warp_tile<S, kBwd, EXT>(a, sm, ws, tiA, TA, 0, x, buf);
            __syncwarp();
            buf ^= 1;
            if (itB >= nitems) {
                pstate = (pstate & 3u) | ((uint32_t)buf << 2);
                break;
            }
            itA = itB; tiA = tiB; twA = twB;
            itB = itC; tiB = tiC; twB = twC;
            itC = itD; tiC = tiD;
        }
    }
    if (x.mode != kBwd) {
        const uint32_t cnt = ws.napp;
        if (cnt) flush_level<S>(a, ws, cnt, x);
        const uint32_t ucnt = ws.nuapp;
        if (ucnt) flush_unvisited<S>(a, ws, ucnt, x);
        // per-warp discovery totals into the CTA's counters
        if ((threadIdx.x & 31) == 0 && ws.cnt[0]) {
            atomicAdd(&sm.c_disc, ws.cnt[0]);
            atomicAdd(&sm.c_pf, ws.cnt[1]);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                atomicAdd(&sm.c_vis[k], ws.cnt[2 + k]);
                atomicAdd(&sm.c_w[k], ws.cnt[2 + S + k]);
                atomicAdd(&sm.c_mc[k], ws.cnt[2 + 2 * S + k]);
            }
        }
    }
}

template <int S, bool EXT>
__global__ void __launch_bounds__(SweepGeom<S>::kThreads, 1) bc_sweep_kernel(BatchArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Smem<S> &sm = *reinterpret_cast<Smem<S> *>(smem_raw);
    constexpr int R = RowGeom<S>::kBytes;
    Ctrl *c = a.ctrl;
    const unsigned int nblk = gridDim.x;
    const unsigned long long wait_ns = c->wait_ns ? c->wait_ns : kDefaultWaitNs;
    const unsigned long long ring = 2ull * a.ntiles;
    const uint32_t total_warps = gridDim.x * SweepGeom<S>::kWarps;
    {
        WarpSmem<S> &ws = sm.w[threadIdx.x >> 5];
        if ((threadIdx.x & 31) == 0) {
            mbar_init(&ws.mbar[0]);
            mbar_init(&ws.mbar[1]);
            mbar_init_fence();
        }
        __syncwarp();
    }
    uint32_t pstate = 0;  // this warp's tile-buffer phases and next buffer

    const bool packed = a.xbeg != nullptr;
    for (uint32_t b = 0; b < a.nbatch; ++b) {
        if (threadIdx.x < S) {
            sm.roots[threadIdx.x] = packed ? kNoRoot : a.roots[(size_t)b * S + threadIdx.x];
            sm.mult[threadIdx.x] = packed ? 1.0 : a.mult[(size_t)b * S + threadIdx.x];
        }
        for (uint32_t i = threadIdx.x; i < kMarkLevels / 32; i += blockDim.x) sm.mlev[i] = 0;
        __syncthreads();
        // frontier / unvisited pair-edge counts of level 0 (same in every CTA)
        unsigned long long pf_cur = 0, pu_cur = 0;
        if (packed) {
            pf_cur = a.xpf[b];
            pu_cur = a.xpu[b];
        } else {
            unsigned int valid = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const uint32_t r = sm.roots[k];
                if (r == kNoRoot) continue;
                ++valid;
                pf_cur += a.vinfo[r].x;
            }
            pu_cur = (unsigned long long)valid * a.nnz - pf_cur;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            for (int s = 0; s < 4; ++s) { c->disc[s] = 0; c->pf[s] = 0; c->uadd[s] = 0; }
            for (int k = 0; k < 8; ++k) { c->visited[k] = 0; c->wsum[k] = 0; c->mc2[k] = 0; }
            a.lbase[0] = 0;
            a.lcnt[1] = 0;
            uint32_t n0 = 0;
            const uint32_t key0 = tile_key(b, 0);
            for (int k = 0; k < S; ++k) {
                const uint32_t r = sm.roots[k];
                if (r == kNoRoot) continue;
                const uint2 ri = a.vinfo[r];
                c->visited[k] = 1;
                c->wsum[k] = 1ull + ri.y;
                c->mc2[k] = (unsigned long long)ri.x + 2ull * ri.y;
                const uint32_t tf = a.tile_of[r];
                const uint32_t t = tf & ~kHubFlag;
                if (vload32(a.tmark + t) == key0) continue;
                a.tmark[t] = key0;
                const uint32_t nch = (tf & kHubFlag) ? a.tiles[t].nchunks : 1u;
                for (uint32_t q = 0; q < nch; ++q) a.lists[n0++] = t + q;
            }
            a.lcnt[0] = n0;
        }
        // reset the rows the batch can reach (every row; in a packed batch the
        // vertices of its tile ranges, i.e. of the components of its roots);
        // single-root slots: roots at level 0 with sigma 1
        auto reset_rows = [&](size_t v_begin, size_t v_end) {
            for (size_t v = v_begin + (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < v_end;
                 v += (size_t)gridDim.x * blockDim.x) {
                constexpr int VW = RowGeom<S>::kValWord;
                uint32_t w[R / 4];
#pragma unroll
                for (int q = 0; q < VW; ++q) w[q] = 0xFFFFFFFFu;  // all levels unvisited
#pragma unroll
                for (int q = VW; q < R / 4; ++q) w[q] = 0u;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    if (sm.roots[k] != (uint32_t)v) continue;
                    w[k >> 1] &= ~(0xFFFFu << ((k & 1) * 16));  // level 0
                    w[VW + 2 * k] = EXT ? 0u : 1u;               // sigma 1
                    w[VW + 2 * k + 1] = EXT ? (uint32_t)(kExtOne >> 32) : 0u;
                }
                uint4 *p = reinterpret_cast<uint4 *>(a.rows + v * R);
#pragma unroll
                for (int h = 0; h < R / 16; ++h)
                    p[h] = make_uint4(w[4 * h], w[4 * h + 1], w[4 * h + 2], w[4 * h + 3]);
            }
        };
        if (!packed) {
            reset_rows(0, a.n);
        } else {
            const uint32_t q0 = a.xrbeg[b], q1 = a.xrbeg[b + 1];
            for (uint32_t q = q0; q < q1; ++q) {
                const uint2 rg = a.xrange[q];
                const uint32_t len = ((q + 1 < q1) ? a.xrange[q + 1].y : a.xtiles[b]) - rg.y;
                if (len) reset_rows(a.tiles[rg.x].v0, a.tiles[rg.x + len - 1].v1);
            }
        }
        if (!grid_sync(c, nblk, wait_ns)) return;
        if (packed) {
            // seed the batch's roots once every row is reset: level 0 and
            // sigma 1 in the root's slot, the slot counters, and the root's
            // tile (all chunks for a hub) on level 0's list
            const uint32_t key0 = tile_key(b, 0);
            const uint32_t r0 = a.xbeg[b], r1 = a.xbeg[b + 1];
            for (uint32_t i = r0 + blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += gridDim.x * blockDim.x) {
                const uint32_t r = a.xroots[i];
                const int k = a.xslot[i];
                unsigned char *row = row_of<S>(a, r);
                *lvl_at(row, k) = 0;
                *val_at<S>(row, k) = EXT ? kExtOne : 1ull;
                const uint2 ri = a.vinfo[r];
                atomicAdd(&c->visited[k], 1ull);
                atomicAdd(&c->wsum[k], 1ull + ri.y);
                atomicAdd(&c->mc2[k], (unsigned long long)ri.x + 2ull * ri.y);
                const uint32_t tf = a.tile_of[r];
                const uint32_t t = tf & ~kHubFlag;
                if (atomicExch(a.tmark + t, key0) == key0) continue;
                const uint32_t nch = (tf & kHubFlag) ? a.tiles[t].nchunks : 1u;
                const uint32_t base = atomicAdd(a.lcnt, nch);
                for (uint32_t q = 0; q < nch; ++q) a.lists[base + q] = t + q;
            }
            if (!grid_sync(c, nblk, wait_ns)) return;
        }
        trace(a, b, 0, 0, 0, 0);

        // ---- forward sweeps
        uint32_t d = 0;
        bool uall = true;              // no pull sweep yet: every tile may hold unvisited vertices
        unsigned long long ustart = 0; // ring position / length of the unvisited-tile list
        uint32_t ulen = 0;
        // ring position of the next pull's appends: every CTA advances it by
        // the appends of each pull sweep, read from that sweep's own counter
        // after its barrier (a shared write position would race with CTAs
        // that already append in the next sweep)
        unsigned long long ucur = 0;
        // level d's list: loaded together with the sweep counters right after
        // each barrier (one round trip per sweep)
        uint32_t lb = vload32(a.lbase), lc = vload32(a.lcnt);
        for (;;) {
            SweepCtx x;
            x.b = b;
            x.mode = (!a.directed && (double)pf_cur >= (double)a.push_pull_ratio * (double)pu_cur) ? kFwdPull
                                                                                                    : kFwdPush;
            x.d = d;
            x.D = 0;
            x.lb_next = lb + lc;
            x.next_lvl = d + 1;
            x.key_next = tile_key(b, d + 1);
            x.split = (x.mode == kFwdPush && lc * 2 < total_warps) ? kPushSplit : 1;
            x.ubase = ucur;
            x.mark = x.filt = false;
            if (threadIdx.x == 0) {
                sm.next = 0;
                sm.c_disc = 0; sm.c_pf = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) { sm.c_vis[k] = 0; sm.c_w[k] = 0; sm.c_mc[k] = 0; }
                if (blockIdx.x == 0) {
                    a.lbase[d + 1] = x.lb_next;
                    a.lcnt[d + 2] = 0;
                    c->disc[(d + 2) & 3] = 0;
                    c->pf[(d + 2) & 3] = 0;
                    c->uadd[(d + 2) & 3] = 0;
                }
            }
            __syncthreads();
            uint32_t walked;
            if (x.mode == kFwdPull) {
                walked = uall ? (packed ? a.xtiles[b] : a.ntiles) : ulen;
                const bool ranged = uall && packed;
                run_sweep<S, EXT>(a, sm, x, uall ? nullptr : a.ulist, ustart, walked, ring, pstate, wait_ns,
                                  ranged ? a.xrange + a.xrbeg[b] : nullptr, ranged ? a.xrbeg[b + 1] - a.xrbeg[b] : 0u);
            } else {
                walked = lc;
                run_sweep<S, EXT>(a, sm, x, a.lists + lb, 0, lc, 0xFFFFFFFFull, pstate, wait_ns);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const int slot = d & 3;
                if (sm.c_disc) {
                    atomicAdd(&c->disc[slot], sm.c_disc);
                    atomicAdd(&c->pf[slot], sm.c_pf);
                }
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    if (!sm.c_vis[k]) continue;
                    atomicAdd(&c->visited[k], sm.c_vis[k]);
                    atomicAdd(&c->wsum[k], sm.c_w[k]);
                    atomicAdd(&c->mc2[k], sm.c_mc[k]);
                }
            }
            if (!grid_sync(c, nblk, wait_ns)) return;
            const unsigned long long disc = vload64(&c->disc[d & 3]);
            const unsigned long long pfn = vload64(&c->pf[d & 3]);
            const unsigned long long uadded = vload64(&c->uadd[d & 3]);
            lb = vload32(a.lbase + d + 1);
            lc = vload32(a.lcnt + d + 1);
            trace(a, b, x.mode == kFwdPull ? 2u : 1u, d, walked, disc);
            if (x.mode == kFwdPull) {
                ustart = ucur;
                ulen = (uint32_t)uadded;
                ucur += uadded;
                uall = false;
            }
            if (disc == 0) break;
            // level d + 1 marks its parents in the backward pass when it holds
            // far fewer pair-edges than level d (the same decision in every CTA)
            if (threadIdx.x == 0 && !a.directed && d + 1 >= 2 && d + 1 < kMarkLevels &&
                pfn * a.mark_ratio < pf_cur)
                sm.mlev[(d + 1) >> 5] |= 1u << ((d + 1) & 31);
            ++d;
            if (d > kMaxLevel) {
                if (blockIdx.x == 0 && threadIdx.x == 0) set_error(c, BCG_ERR_DEPTH);
                return;
            }
            pu_cur = pu_cur > pfn ? pu_cur - pfn : 0;
            pf_cur = pfn;
        }
        const uint32_t D = d;

        if (a.dbg_level || a.dbg_sigma) {
            // debug or level-export run: copy every slot's levels (and sigma)
            // out before the backward pass overwrites sigma
            for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < a.n;
                 v += (size_t)gridDim.x * blockDim.x) {
                unsigned char *row = a.rows + v * R;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    const uint16_t L = __ldcg(lvl_at(row, k));
                    const size_t o = ((size_t)b * S + k) * a.n + v;  // slot k of batch b
                    if (a.dbg_level) a.dbg_level[o] = (L == kUnvisited) ? -1 : (int32_t)L;
                    if (a.dbg_sigma) a.dbg_sigma[o] = (L == kUnvisited) ? 0ull : __ldcg(val_at<S>(row, k));
                }
            }
            if (!grid_sync(c, nblk, wait_ns)) return;
        }

        // ---- backward sweeps over the level lists
        const int lowest = a.dbg_delta ? 0 : 1;
        // the level lists are final: each level's list position is loaded one
        // sweep ahead
        uint32_t blb = vload32(a.lbase + D), blc = vload32(a.lcnt + D);
        for (int dd = (int)D; dd >= lowest; --dd) {
            SweepCtx x;
            x.b = b;
            x.mode = kBwd;
            x.d = (uint32_t)dd;
            x.D = D;
            x.key_next = 0;
            x.lb_next = 0;
            x.next_lvl = 0;
            x.split = 1;
            auto marks_parents = [&](uint32_t e) {
                return e < kMarkLevels && ((sm.mlev[e >> 5] >> (e & 31)) & 1u);
            };
            x.mark = marks_parents((uint32_t)dd);
            x.filt = !x.mark && dd >= 1 && marks_parents((uint32_t)dd + 1);
            const uint32_t lb = blb, lc = blc;
            if (dd > lowest) {
                blb = vload32(a.lbase + dd - 1);
                blc = vload32(a.lcnt + dd - 1);
            }
            if (threadIdx.x == 0) sm.next = 0;
            __syncthreads();
            run_sweep<S, EXT>(a, sm, x, a.lists + lb, 0, lc, 0xFFFFFFFFull, pstate, wait_ns);
            if (!grid_sync(c, nblk, wait_ns)) return;
            trace(a, b, 3u, (uint32_t)dd, lc, (x.mark ? 1u : 0u) | (x.filt ? 2u : 0u));
        }

        // ---- served waves: each slot's dependencies into the buffer of the
        // request that owns the slot's source, slots in order (so a request's
        // sources reach its buffer in source order however they were packed)
        if (a.slot_delta) {
            const uint32_t q0 = a.xrbeg[b], q1 = a.xrbeg[b + 1];
            for (uint32_t q = q0; q < q1; ++q) {
                const uint2 rg = a.xrange[q];
                const uint32_t len = ((q + 1 < q1) ? a.xrange[q + 1].y : a.xtiles[b]) - rg.y;
                if (!len) continue;
                const SlotOut o = a.xout[q];
                const size_t v0 = a.tiles[rg.x].v0, v1 = a.tiles[rg.x + len - 1].v1;
                for (size_t v = v0 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < v1;
                     v += (size_t)gridDim.x * blockDim.x) {
                    const unsigned char *row = a.rows + v * R;
#pragma unroll
                    for (int k = 0; k < S; ++k) {
                        const uint16_t L = __ldcg(reinterpret_cast<const unsigned short *>(row) + k);
                        if (L == kUnvisited || L == 0 || !o.out[k]) continue;
                        double *op = o.out[k] + (v - o.base);
                        __stcg(op, __ldcg(op) + __ldcg(a.slot_delta + (size_t)k * a.n + v));
                    }
                }
            }
            if (!grid_sync(c, nblk, wait_ns)) return;
        }

        // ---- source term and per-root statistics
        if (blockIdx.x == 0 && threadIdx.x < S) {
            const int k = threadIdx.x;
            const uint32_t r = sm.roots[k];
            if (r != kNoRoot || packed) {
                const size_t idx = (size_t)b * S + k;
                const unsigned long long W = vload64(&c->wsum[k]);
                const uint32_t p = packed ? 0u : a.pend[idx];
                if (p && W >= 2) {
                    double *bp = a.bc + (a.ext ? a.ext[r] : r);
                    __stcg(bp, __ldcg(bp) + (double)p * (double)(W - 2));
                }
                a.rstat[idx].visited = vload64(&c->visited[k]);
                a.rstat[idx].wsum = W;
                a.rstat[idx].mc2 = vload64(&c->mc2[k]);
                a.rstat[idx].depth = D;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host-side launch helpers.
// ---------------------------------------------------------------------------

template <int S, bool EXT>
static int launch_impl(const BatchArgs &a, cudaStream_t st, int *grid_out) {
    const size_t smem = smem_bytes<S>();
    cudaError_t e = cudaFuncSetAttribute(bc_sweep_kernel<S, EXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return set_error(BCG_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bc_sweep_kernel<S, EXT>, SweepGeom<S>::kThreads, smem);
    if (e != cudaSuccess) return set_error(BCG_ERR_CUDA, "occupancy query: %s", cudaGetErrorString(e));
    if (per_sm < 1) return set_error(BCG_ERR_CUDA, "sweep kernel cannot be resident (smem %zu)", smem);
    int grid = nsm * per_sm;
    if (grid_out) *grid_out = grid;
    BatchArgs args = a;
    void *params[] = {&args};
    e = cudaLaunchCooperativeKernel((const void *)bc_sweep_kernel<S, EXT>, dim3(grid), dim3(SweepGeom<S>::kThreads), params, smem,
                                    st);
    if (e != cudaSuccess)
        return set_error(e == cudaErrorNoKernelImageForDevice ? BCG_ERR_NOGPU : BCG_ERR_CUDA,
                         "sweep kernel launch: %s", cudaGetErrorString(e));
    return BCG_OK;
}

int launch_sweep(int S, const BatchArgs &a, cudaStream_t st, int *grid_out, bool ext) {
    switch (S) {
        case 1: return ext ? launch_impl<1, true>(a, st, grid_out) : launch_impl<1, false>(a, st, grid_out);
        case 3: return ext ? launch_impl<3, true>(a, st, grid_out) : launch_impl<3, false>(a, st, grid_out);
        case 6: return ext ? launch_impl<6, true>(a, st, grid_out) : launch_impl<6, false>(a, st, grid_out);
        default: return set_error(BCG_ERR_ARG, "batch width %d not in {1,3,6}", S);
    }
}

}  // namespace bcg
