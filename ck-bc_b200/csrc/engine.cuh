// Device-side definitions shared by the engine's CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bcg {

// Sweep kernel geometry (one CTA per SM).  Each lane keeps the rows of a
// whole segment (kItems gathers of up to 32 bytes) in registers; 512 threads
// leave 128 registers per thread, which widths 1 and 3 fit, and width 6 runs
// with 384 threads (168 registers).
template <int S>
struct SweepGeom {
    static constexpr int kThreads = (S == 6) ? 384 : 512;
    static constexpr int kWarps = kThreads / 32;  // independent tile workers per CTA
};
constexpr int kTileVerts = 32;           // max vertices per tile (one per lane)
#ifndef BCG_TILE_EDGES
#define BCG_TILE_EDGES 512
#endif
constexpr int kTileEdges = BCG_TILE_EDGES;  // max adjacency entries per tile
constexpr int kItems = 4;                   // edges of a segment: one lane's share of a round
constexpr int kRoundEdges = 32 * kItems;    // a warp takes a tile's edges in rounds of this many
static_assert(kTileEdges % kRoundEdges == 0, "a tile holds whole rounds");
constexpr int kPushSplit = 8;            // sparse push sweeps: warps per tile
constexpr uint16_t kUnvisited = 0xFFFFu;
constexpr uint32_t kMaxLevel = 0xFFFDu;  // deepest level a 16-bit level can hold
constexpr uint32_t kNoRoot = 0xFFFFFFFFu;
constexpr uint32_t kNoTile = 0xFFFFFFFFu;
constexpr uint32_t kHubFlag = 0x80000000u;  // tile_of[v] flag: v is split into chunks
constexpr unsigned long long kDefaultWaitNs = 20ull * 1000 * 1000 * 1000;  // 20 s

// Per-vertex state row of a batch of S slots (S in {1, 3, 6}): a level block
// of S 16-bit levels padded to 8 bytes (16 for S = 6), then S 64-bit values:
// 16, 32 or 64 bytes, i.e. half of, one or two 32-byte sectors.  The value of
// a slot is sigma during the forward pass and (1 + delta) / sigma after the
// vertex's backward step.  The padding of the level block holds the child
// marks: bit k (from kMarkShift on in word kMarkWord) is cleared once a
// vertex of level L + 1 in slot k has found the vertex, at level L in slot
// k, as its parent (the batch reset sets the whole block to ones).
template <int S>
struct RowGeom {
    static_assert(S == 1 || S == 3 || S == 6, "batch width must be 1, 3 or 6");
    static constexpr int kLvlBytes = (S <= 4) ? 8 : 16;
    static constexpr int kBytes = kLvlBytes + 8 * S;
    static constexpr int kWords = kBytes / 4;
    static constexpr int kVec = kBytes / 16;
    static constexpr int kValWord = kLvlBytes / 4;  // first word of the values
    // the level block's free halfwords: word 1's upper half (S = 1, 3) or
    // word 3 (S = 6, the levels of slots 6 and 7 that do not exist)
    static constexpr int kMarkWord = (S <= 4) ? 1 : 3;
    static constexpr int kMarkShift = (S <= 4) ? 16 : 0;
    static_assert(16 * S <= 32 * kMarkWord + kMarkShift && 32 * kMarkWord + kMarkShift + S <= 8 * kLvlBytes,
                  "marks lie between the levels and the values");
};

__host__ __device__ constexpr int row_bytes(int S) { return ((S <= 4) ? 8 : 16) + 8 * S; }

// One unit of sweep work: vertices [v0, v1) with all their edges, or one
// chunk [e0, e1) of the adjacency of a single high-degree vertex (hub >= 0).
// The chunks of a hub are consecutive tiles; chunk c of a hub has its own
// accumulator slot hslot (the hub's chunks use slots hslot - c .. hslot - c +
// nchunks - 1), so the chunk totals can be added in chunk order.
struct Tile {
    uint32_t v0, v1;
    uint32_t e0, e1;
    int32_t hub;       // hub index, -1 for an ordinary tile
    uint32_t nchunks;  // chunks of this hub (1 for ordinary tiles)
    uint32_t hslot;    // hub chunks: accumulator slot of this chunk (0 otherwise)
    uint32_t hchunk;   // hub chunks: index c of this chunk within its hub (0 otherwise)
};

// Sweep modes.
enum : int { kFwdPush = 0, kFwdPull = 1, kBwd = 2 };

// Control block of one kernel launch (zeroed by the host before the launch).
struct Ctrl {
    unsigned long long bar_arrived;  // grid barrier arrivals since the launch (monotone)
    int error;      // BCG_ERR_* code set by the device, 0 = fine
    int overflow;   // a uint64 sigma sum wrapped
    unsigned long long wait_ns;  // bound of every device-side wait
    // ring of per-sweep counters, indexed by sweep % 4: a sweep adds only to
    // its own entry, and the entry is cleared two sweeps ahead, so a value
    // read after the sweep's barrier cannot change while a faster CTA is
    // already in the next sweep
    unsigned long long disc[4];  // (vertex, slot) pairs discovered in the sweep
    unsigned long long pf[4];    // sum of degrees over those pairs
    unsigned long long uadd[4];  // tiles the sweep (a pull) appended to the unvisited-tile ring
    // per-slot accumulators of the current batch
    unsigned long long visited[8];
    unsigned long long wsum[8];  // sum of (1 + reach) over visited vertices
    unsigned long long mc2[8];   // sum of (deg + 2 reach) over visited vertices
};

// One record of the optional sweep trace (written by CTA 0 after each grid
// barrier when BatchArgs::trace is set).
struct TraceRec {
    unsigned long long t_ns;   // %globaltimer when the phase ended
    unsigned int batch;
    unsigned int kind;         // 0 init, 1 push, 2 pull, 3 backward
    unsigned int level;
    unsigned int nwork;        // tiles walked
    unsigned long long disc;   // (vertex, slot) pairs discovered (forward)
};

// Per-root result of a batch.
struct RootStat {
    unsigned long long visited;
    unsigned long long wsum;
    unsigned long long mc2;
    unsigned int depth;
    unsigned int pad;
};

// Where the dependencies of one graph's slots in one packed batch go (served
// waves): slot k's delta of vertex v is added to out[k][v - base] (nullptr:
// slot k holds no root of that graph in that batch).
struct SlotOut {
    double *out[6];
    uint32_t base;
    uint32_t pad;
};

struct BatchArgs {
    uint32_t n;             // vertices with state rows a sweep may touch (the tiles' range)
    const uint32_t *offs;   // CSR row starts (n+1); pruned lists start here too
    const uint32_t *adj;    // adjacency (pruned lists compacted to the front)
    const uint2 *vinfo;     // per vertex {deg in the pruned graph, reach}
    const Tile *tiles;
    uint32_t ntiles;
    const uint32_t *tile_of;  // per vertex: its tile (first chunk | kHubFlag for hubs)
    uint32_t *tmark;        // per tile: (batch, level) key of its last list append
    uint32_t *lists;        // per-level lists of active tiles, back to back
    unsigned long long list_cap;
    uint32_t *lbase;        // kMaxLevel + 3: start of level d's list
    uint32_t *lcnt;         // kMaxLevel + 3: length of level d's list
    uint32_t *ulist;        // ring of 2 * ntiles: tiles that still hold unvisited vertices
    unsigned char *rows;    // n state rows of row_bytes(S)
    double *bc;             // n accumulators
    const uint32_t *ext;    // vertex v's bc is bc[ext[v]] (nullptr: bc[v])
    const uint32_t *roots;  // nbatch * S, kNoRoot = empty slot
    const double *mult;     // nbatch * S weight of each root's dependencies
    const uint32_t *pend;   // nbatch * S pendant sources folded into the root
    uint32_t nbatch;
    unsigned long long *hub_acc;  // (hub chunks) * S: one slot per chunk
    unsigned int *hub_cnt;        // nhub: chunks of the hub finished in the current sweep
    Ctrl *ctrl;
    RootStat *rstat;        // nbatch * S
    unsigned long long nnz; // adjacency entries of the pruned graph
    float push_pull_ratio;  // pull when frontier pair-edges >= ratio * unvisited pair-edges
    uint32_t mark_ratio;    // a level marks its parents in the backward pass when its
                            // pair-edges * mark_ratio < the level above's (0: never)
    int directed;           // 1: adjacency is not symmetric, pull is not allowed
    // debug outputs (nullptr otherwise): slot k of batch b, vertex v at
    // [(b * S + k) * n + v]; levels and sigma are copied after the forward
    // pass, delta is written by the backward pass (which then runs down to
    // level 0)
    int32_t *dbg_level;
    unsigned long long *dbg_sigma;
    double *dbg_delta;
    // optional sweep trace (nullptr = off); trace_cnt counts records written
    TraceRec *trace;
    unsigned int trace_cap;
    unsigned int *trace_cnt;
    // Component-packed batches (xbeg == nullptr: one root per slot, given by
    // roots / mult / pend).  Batch b runs roots xroots[xbeg[b] .. xbeg[b+1]),
    // root i in slot xslot[i]; roots that share a slot lie in different
    // connected components, so their searches never meet.  Every such root has
    // weight 1 and no pendant sources; the per-slot counters add up over its
    // roots.  xpu[b] = sum over the batch's roots of the adjacency entries of
    // their components minus their own degrees (level 0's unvisited
    // pair-edges).  The tiles of those components are the ranges
    // xrange[xrbeg[b] .. xrbeg[b+1]) ({first tile, tiles before this range});
    // xtiles[b] is their total: the first pull of the batch walks only them.
    const uint32_t *xbeg;
    const uint32_t *xroots;
    const unsigned char *xslot;
    const unsigned long long *xpf;   // per batch: sum of the roots' degrees
    const unsigned long long *xpu;
    const uint32_t *xtiles;
    const uint32_t *xrbeg;
    const uint2 *xrange;
    // served waves: the backward pass keeps each slot's dependencies in
    // slot_delta[k * n + v], and at the batch's end xout[q] routes the slots
    // of range q into the requests' buffers; nullptr: dependencies go to bc
    const SlotOut *xout;
    double *slot_delta;
};

}  // namespace bcg
