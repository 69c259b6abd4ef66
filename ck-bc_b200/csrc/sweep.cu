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
// Values rotate over three arrays by level mod 3.  The neighbours of a vertex
// at level L sit at levels L-1, L and L+1 only, so in the array of level L+1
// the only non-zero entries a level-L vertex can see are its children's, and
// in the array of level L the only non-zero entries an unvisited vertex can
// see during the level-L pull are its parents'.  Pull and backward sweeps
// therefore sum the neighbour's whole value row without reading its levels:
// one gather of S*8 bytes per edge for all S slots.  Push sweeps read the
// neighbour's 16-bit level row to claim it.
//
// Work decomposition.  Vertices are cut into static tiles of <= 32
// consecutive vertices and <= 256 adjacency entries; a vertex with more than
// 256 neighbours is split into 256-entry chunks whose partial sums meet in
// hub_acc (the last chunk to arrive finishes the vertex).  Every warp works
// on one tile at a time with no CTA-wide synchronisation: lane j owns vertex j
// of the tile, the tile's edges are cut into contiguous runs of 8 per lane
// (merge-path over the warp's exclusive scan of active degrees).
// Push and backward sweeps walk only the tiles on the level's list (tiles
// holding a vertex first reached at that level, for any slot); pull sweeps walk
// the tiles that still hold an unvisited vertex (all tiles in the first pull of
// a batch).  Both lists are written through warp-buffered appends.
#include <cstdio>

#include "bcg.h"
#include "bcg_common.hpp"
#include "engine.cuh"

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

// L2 policy for streamed data: evicted before the per-vertex rows.
__device__ __forceinline__ unsigned long long evict_first_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// Streaming read of the adjacency (read-only for the whole launch).
__device__ __forceinline__ uint32_t ld_adj(const uint32_t *p, unsigned long long pol) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

// Software grid barrier (all CTAs co-resident: cooperative launch).  Returns
// false when any CTA recorded an error, in which case the caller returns.
__device__ bool grid_sync(Ctrl *c, unsigned int nblocks, unsigned long long wait_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *genp = &c->bar_gen;
        unsigned int gen = *genp;
        __threadfence();
        unsigned int arrived = atomicAdd(&c->bar_count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&c->bar_count, 0u);
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            unsigned long long t0 = global_ns();
            unsigned int spins = 0;
            while (*genp == gen) {
                if ((++spins & 255u) == 0) {
                    if (*reinterpret_cast<volatile int *>(&c->error)) break;
                    if (global_ns() - t0 > wait_ns) {
                        atomicCAS(&c->error, 0, BCG_ERR_TIMEOUT);
                        break;
                    }
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *reinterpret_cast<volatile int *>(&c->error) == 0;
}

template <int S>
__device__ __forceinline__ void load_row(const uint16_t *base, uint32_t v, uint16_t (&r)[S]) {
    const uint16_t *p = base + (size_t)v * S;
    if constexpr (S == 1) {
        r[0] = p[0];
    } else if constexpr (S == 2) {
        uint32_t x = *reinterpret_cast<const uint32_t *>(p);
        r[0] = (uint16_t)x;
        r[1] = (uint16_t)(x >> 16);
    } else if constexpr (S == 4) {
        uint2 x = *reinterpret_cast<const uint2 *>(p);
        r[0] = (uint16_t)x.x; r[1] = (uint16_t)(x.x >> 16);
        r[2] = (uint16_t)x.y; r[3] = (uint16_t)(x.y >> 16);
    } else {
        uint4 x = *reinterpret_cast<const uint4 *>(p);
        r[0] = (uint16_t)x.x; r[1] = (uint16_t)(x.x >> 16);
        r[2] = (uint16_t)x.y; r[3] = (uint16_t)(x.y >> 16);
        r[4] = (uint16_t)x.z; r[5] = (uint16_t)(x.z >> 16);
        r[6] = (uint16_t)x.w; r[7] = (uint16_t)(x.w >> 16);
    }
}

template <int S>
__device__ __forceinline__ void store_row(uint16_t *base, uint32_t v, const uint16_t (&r)[S]) {
    uint16_t *p = base + (size_t)v * S;
    if constexpr (S == 1) {
        p[0] = r[0];
    } else if constexpr (S == 2) {
        *reinterpret_cast<uint32_t *>(p) = (uint32_t)r[0] | ((uint32_t)r[1] << 16);
    } else if constexpr (S == 4) {
        *reinterpret_cast<uint2 *>(p) = make_uint2((uint32_t)r[0] | ((uint32_t)r[1] << 16),
                                                  (uint32_t)r[2] | ((uint32_t)r[3] << 16));
    } else {
        *reinterpret_cast<uint4 *>(p) = make_uint4((uint32_t)r[0] | ((uint32_t)r[1] << 16),
                                                  (uint32_t)r[2] | ((uint32_t)r[3] << 16),
                                                  (uint32_t)r[4] | ((uint32_t)r[5] << 16),
                                                  (uint32_t)r[6] | ((uint32_t)r[7] << 16));
    }
}

// Gathers the S 64-bit values of vertex v from one value array (one 128- or
// 256-bit load per 32 bytes of row).
template <int S>
__device__ __forceinline__ void load_vals(const unsigned long long *arr, uint32_t v, unsigned long long (&x)[S]) {
    const unsigned long long *p = arr + (size_t)v * S;
    if constexpr (S == 1) {
        x[0] = p[0];
    } else if constexpr (S == 2) {
        const ulonglong2 t = *reinterpret_cast<const ulonglong2 *>(p);
        x[0] = t.x; x[1] = t.y;
    } else {
#pragma unroll
        for (int h = 0; h < S; h += 4)
            asm volatile("ld.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                         : "=l"(x[h]), "=l"(x[h + 1]), "=l"(x[h + 2]), "=l"(x[h + 3])
                         : "l"(p + h));
    }
}

// Per-warp scratch.
template <int S>
struct WarpSmem {
    uint32_t pre[kTileVerts + 1];
    uint32_t eb[kTileVerts];
    uint32_t mask[kTileVerts];
    uint32_t app[2 * 32];   // buffered appends to the next level's list
    uint32_t uapp[2 * 32];  // buffered appends to the unvisited-tile ring
    uint32_t napp, nuapp;
    unsigned long long acc[kTileVerts][S];
    unsigned long long own[kTileVerts][S];
};

template <int S>
struct Smem {
    WarpSmem<S> w[kWarps];
    // per-CTA counters of the current sweep
    unsigned long long c_disc, c_pf;
    unsigned long long c_vis[S], c_w[S], c_mc[S];
    // batch constants
    uint32_t roots[S];
    double mult[S];
};

template <int S>
size_t smem_bytes() { return sizeof(Smem<S>); }

// Parameters of one sweep, identical in every warp.
struct SweepCtx {
    int mode;
    uint32_t d, D;
    uint32_t key_next;   // tile mark of (batch, level d+1)
    uint32_t lb_next;    // list start of level d+1
    uint32_t next_lvl;   // d + 1 (index into lcnt)
    const unsigned long long *src;  // value array read by the sweep's edges
    unsigned long long *own;        // value array of level d (own sigma / X)
    unsigned long long *dst;        // value array of level d+1 (push / pull)
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

// Writes the warp's buffered unvisited-tile appends to the ring.
template <int S>
__device__ __forceinline__ void flush_unvisited(const BatchArgs &a, WarpSmem<S> &ws, uint32_t cnt) {
    const unsigned lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&a.ctrl->uctr, (unsigned long long)cnt);
    base = __shfl_sync(0xffffffffu, base, 0);
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
__device__ __forceinline__ void append_unvisited(const BatchArgs &a, WarpSmem<S> &ws, uint32_t t) {
    const unsigned lane = threadIdx.x & 31;
    if (t != kNoTile && (t & kHubFlag)) {
        const uint32_t t0 = t & ~kHubFlag;
        const uint32_t nch = a.tiles[t0].nchunks;
        const unsigned long long base = atomicAdd(&a.ctrl->uctr, (unsigned long long)nch);
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
        flush_unvisited<S>(a, ws, cnt);
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

template <int S>
__device__ __forceinline__ void flush_run(const BatchArgs &a, WarpSmem<S> &ws, int mode, uint32_t j,
                                          unsigned long long (&run)[S]) {
#pragma unroll
    for (int k = 0; k < S; ++k) {
        if (!run[k]) continue;
        if (mode == kFwdPull) {
            const unsigned long long old = atomicAdd(&ws.acc[j][k], run[k]);
            if (old + run[k] < run[k]) a.ctrl->overflow = 1;
        } else {
            atomicAdd(reinterpret_cast<double *>(&ws.acc[j][k]), __longlong_as_double((long long)run[k]));
        }
        run[k] = 0ull;
    }
}

// One tile, processed by one warp.
template <int S, int MODE>
__device__ void warp_tile(const BatchArgs &a, Smem<S> &sm, WarpSmem<S> &ws, uint32_t ti, const SweepCtx &x) {
    const unsigned lane = threadIdx.x & 31;
    constexpr int mode = MODE;
    const uint32_t d = x.d;
    const uint16_t dl = (uint16_t)d;
    const Tile T = a.tiles[ti];
    const bool hub = T.hub >= 0;
    const uint32_t nv = T.v1 - T.v0;
    uint32_t deg_act = 0, m = 0;
    uint2 vi = make_uint2(0, 0);
    // ---- phase 1: activity of the tile's vertices
    if (lane < nv) {
        const uint32_t v = T.v0 + lane;
        uint16_t l[S];
        load_row<S>(a.lvl, v, l);
#pragma unroll
        for (int k = 0; k < S; ++k) {
            if (mode == kFwdPull) m |= (uint32_t)(l[k] == kUnvisited) << k;
            else m |= (uint32_t)(l[k] == dl) << k;
        }
        if (m) {
            vi = a.vinfo[v];
            if (mode == kFwdPull && vi.x == 0) m = 0;  // no edge: cannot be reached
        }
        if (m) {
            const uint32_t ob = a.offs[v];
            const uint32_t eb = hub ? T.e0 : ob;
            uint32_t ee = ob + vi.x;
            if (hub && T.e1 < ee) ee = T.e1;
            if (ee < eb) ee = eb;
            deg_act = ee - eb;
            if (mode == kBwd && d == x.D) deg_act = 0;
            ws.eb[lane] = eb;
#pragma unroll
            for (int k = 0; k < S; ++k) ws.acc[lane][k] = 0ull;
            if (mode != kFwdPull) {
                unsigned long long o[S];
                load_vals<S>(x.own, v, o);
#pragma unroll
                for (int k = 0; k < S; ++k) ws.own[lane][k] = ((m >> k) & 1u) ? o[k] : 0ull;
            }
        }
        ws.mask[lane] = m;
    }
    if (hub && !__shfl_sync(0xffffffffu, m, 0)) return;  // same decision in every chunk
    uint32_t incl = deg_act;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (lane < nv) ws.pre[lane] = incl - deg_act;
    if (lane == 0) ws.pre[nv] = total;
    __syncwarp();

    // ---- phase 2: edges, a contiguous run of <= kItems per lane
    if (total) {
        const uint32_t i0 = lane * kItems;
        const uint32_t i1 = min(total, i0 + kItems);
        uint32_t j = 0;
        if (i0 < i1) {
            uint32_t lo = 0, hi = nv;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (ws.pre[mid] <= i0) lo = mid; else hi = mid;
            }
            j = lo;
        }
        // edges per lane in flight, bounded by the registers their rows need
        // (S 16-bit levels for push, S 64-bit values for pull / backward)
        constexpr int QB = (MODE == kFwdPush) ? ((S >= 8) ? 2 : kSub) : ((S >= 8) ? 1 : (S >= 4) ? 2 : kSub);
        const unsigned long long pol = evict_first_policy();
        unsigned long long run[S];
#pragma unroll
        for (int k = 0; k < S; ++k) run[k] = 0ull;
        uint32_t runj = j;
#pragma unroll
        for (int sub = 0; sub < kItems / QB; ++sub) {
            uint32_t jj[QB], uu[QB];
#pragma unroll
            for (int q = 0; q < QB; ++q) {
                const uint32_t i = i0 + sub * QB + q;
                if (i < i1) {
                    while (i >= ws.pre[j + 1]) ++j;
                    jj[q] = j;
                    uu[q] = ld_adj(a.adj + ws.eb[j] + (i - ws.pre[j]), pol);
                }
            }
            if (mode == kFwdPush) {
                uint16_t ul[QB][S];
#pragma unroll
                for (int q = 0; q < QB; ++q)
                    if (i0 + sub * QB + q < i1) load_row<S>(a.lvl, uu[q], ul[q]);
#pragma unroll
                for (int q = 0; q < QB; ++q) {
                    uint32_t app = kNoTile;
                    if (i0 + sub * QB + q < i1) {
                        const uint32_t jm = ws.mask[jj[q]];
                        const uint32_t w = uu[q];
                        bool claimed_any = false;
#pragma unroll
                        for (int k = 0; k < S; ++k) {
                            if (!((jm >> k) & 1u)) continue;
                            const uint16_t L = ul[q][k];
                            bool take = (L == (uint16_t)(d + 1));
                            if (L == kUnvisited) {
                                const uint16_t old =
                                    atomicCAS(reinterpret_cast<unsigned short *>(a.lvl) + (size_t)w * S + k,
                                              (unsigned short)kUnvisited, (unsigned short)(d + 1));
                                if (old == kUnvisited) {
                                    const uint2 wi = a.vinfo[w];
                                    atomicAdd(&sm.c_disc, 1ull);
                                    atomicAdd(&sm.c_pf, (unsigned long long)wi.x);
                                    atomicAdd(&sm.c_vis[k], 1ull);
                                    atomicAdd(&sm.c_w[k], 1ull + wi.y);
                                    atomicAdd(&sm.c_mc[k], (unsigned long long)wi.x + 2ull * wi.y);
                                    take = true;
                                    claimed_any = true;
                                } else {
                                    take = (old == (uint16_t)(d + 1));
                                }
                            }
                            if (take) {
                                const unsigned long long s = ws.own[jj[q]][k];
                                const unsigned long long old = atomicAdd(x.dst + (size_t)w * S + k, s);
                                if (old + s < s) a.ctrl->overflow = 1;
                            }
                        }
                        if (claimed_any) app = claim_tile(a, w, x.key_next);
                    }
                    append_level<S>(a, ws, app, x);
                }
            } else {
                unsigned long long xv[QB][S];
#pragma unroll
                for (int q = 0; q < QB; ++q)
                    if (i0 + sub * QB + q < i1) load_vals<S>(x.src, uu[q], xv[q]);
#pragma unroll
                for (int q = 0; q < QB; ++q) {
                    if (i0 + sub * QB + q >= i1) continue;
                    if (jj[q] != runj) {
                        flush_run<S>(a, ws, mode, runj, run);
                        runj = jj[q];
                    }
                    const uint32_t jm = ws.mask[jj[q]];
#pragma unroll
                    for (int k = 0; k < S; ++k) {
                        if (!((jm >> k) & 1u)) continue;
                        if (mode == kFwdPull) {
                            const unsigned long long t = run[k] + xv[q][k];
                            if (t < xv[q][k]) a.ctrl->overflow = 1;
                            run[k] = t;
                        } else {
                            const double t = __longlong_as_double((long long)run[k]) +
                                             __longlong_as_double((long long)xv[q][k]);
                            run[k] = (unsigned long long)__double_as_longlong(t);
                        }
                    }
                }
            }
        }
        if (mode != kFwdPush && i0 < i1) flush_run<S>(a, ws, mode, runj, run);
    }
    __syncwarp();
    if (mode == kFwdPush) return;

    // ---- hub chunks meet in hub_acc; the last chunk to arrive finishes the vertex
    if (hub) {
        const uint32_t hm = ws.mask[0];
        unsigned long long *hacc = a.hub_acc + (size_t)T.hub * S;
        if (lane < (unsigned)S && ((hm >> lane) & 1u)) {
            const unsigned long long xa = ws.acc[0][lane];
            if (mode == kFwdPull) {
                const unsigned long long old = atomicAdd(hacc + lane, xa);
                if (old + xa < xa) a.ctrl->overflow = 1;
            } else {
                atomicAdd(reinterpret_cast<double *>(hacc + lane), __longlong_as_double((long long)xa));
            }
        }
        __threadfence();
        __syncwarp();
        uint32_t last = 0;
        if (lane == 0) last = (atomicAdd(a.hub_cnt + T.hub, 1u) == T.nchunks - 1);
        last = __shfl_sync(0xffffffffu, last, 0);
        if (!last) return;
        __threadfence();
        if (lane < (unsigned)S) ws.acc[0][lane] = atomicExch(hacc + lane, 0ull);
        if (lane == 0) atomicExch(a.hub_cnt + T.hub, 0u);
        __syncwarp();
    }

    // ---- phase 3: finish the tile's vertices
    uint32_t nd = 0, left = 0;
    if (lane < nv && m) {
        const uint32_t v = T.v0 + lane;
        if (mode == kFwdPull) {
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (!((m >> k) & 1u)) continue;
                const unsigned long long s = ws.acc[lane][k];
                if (!s) {
                    ++left;
                    continue;
                }
                a.lvl[(size_t)v * S + k] = (uint16_t)(d + 1);
                x.dst[(size_t)v * S + k] = s;
                ++nd;
                atomicAdd(&sm.c_vis[k], 1ull);
                atomicAdd(&sm.c_w[k], 1ull + vi.y);
                atomicAdd(&sm.c_mc[k], (unsigned long long)vi.x + 2ull * vi.y);
            }
            if (nd) {
                atomicAdd(&sm.c_disc, (unsigned long long)nd);
                atomicAdd(&sm.c_pf, (unsigned long long)nd * vi.x);
            }
        } else {
            double add = 0.0;
            const double reach = (double)vi.y;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (!((m >> k) & 1u)) continue;
                const double sig = (double)ws.own[lane][k];
                const double acc = __longlong_as_double((long long)ws.acc[lane][k]);
                const double delta = reach + sig * acc;
                const double xo = (1.0 + delta) / sig;
                x.own[(size_t)v * S + k] = (unsigned long long)__double_as_longlong(xo);
                if (d > 0) add += sm.mult[k] * delta;
                if (a.dbg_delta) a.dbg_delta[v] = delta;
            }
            if (d > 0) a.bc[v] += add;
        }
    }
    if (mode == kFwdPull) {
        // a pull sweep visits every listed tile once, so no mark is needed; a
        // hub is listed by its finishing chunk (first chunk | kHubFlag expands it)
        const uint32_t me = hub ? a.tile_of[T.v0] : ti;
        const bool any = __any_sync(0xffffffffu, nd > 0);
        append_level<S>(a, ws, (any && lane == 0) ? me : kNoTile, x);
        const bool keep = __any_sync(0xffffffffu, left > 0);
        append_unvisited<S>(a, ws, (keep && lane == 0) ? me : kNoTile);
    }
}

// Runs one sweep: every warp of the grid walks its share of the work items,
// item i being list[i % ring] (or tile i when list is null).
template <int S>
__device__ void run_sweep(const BatchArgs &a, Smem<S> &sm, const SweepCtx &x, const uint32_t *list,
                          unsigned long long start, uint32_t nwork, unsigned long long ring) {
    const unsigned wid = threadIdx.x >> 5;
    WarpSmem<S> &ws = sm.w[wid];
    const uint32_t gw = blockIdx.x * kWarps + wid;
    const uint32_t nw = gridDim.x * kWarps;
    if ((threadIdx.x & 31) == 0) { ws.napp = 0; ws.nuapp = 0; }
    __syncwarp();
    for (uint32_t i = gw; i < nwork; i += nw) {
        const uint32_t ti = list ? list[(start + i) % ring] : i;
        if (x.mode == kFwdPush) warp_tile<S, kFwdPush>(a, sm, ws, ti, x);
        else if (x.mode == kFwdPull) warp_tile<S, kFwdPull>(a, sm, ws, ti, x);
        else warp_tile<S, kBwd>(a, sm, ws, ti, x);
        __syncwarp();
    }
    if (x.mode != kBwd) {
        const uint32_t cnt = ws.napp;
        if (cnt) flush_level<S>(a, ws, cnt, x);
        const uint32_t ucnt = ws.nuapp;
        if (ucnt) flush_unvisited<S>(a, ws, ucnt);
    }
}

// CTAs per SM the register allocation is sized for (2: 64 registers/thread).
#ifndef BCG_MIN_BLOCKS
#define BCG_MIN_BLOCKS 2
#endif

template <int S>
__global__ void __launch_bounds__(kThreads, BCG_MIN_BLOCKS) bc_sweep_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<S> &sm = *reinterpret_cast<Smem<S> *>(smem_raw);
    Ctrl *c = a.ctrl;
    const unsigned int nblk = gridDim.x;
    const unsigned long long wait_ns = c->wait_ns ? c->wait_ns : kDefaultWaitNs;
    const size_t plane = (size_t)a.n * S;  // distance between the three value arrays
    const unsigned long long ring = 2ull * a.ntiles;

    for (uint32_t b = 0; b < a.nbatch; ++b) {
        if (threadIdx.x < S) {
            sm.roots[threadIdx.x] = a.roots[(size_t)b * S + threadIdx.x];
            sm.mult[threadIdx.x] = a.mult[(size_t)b * S + threadIdx.x];
        }
        __syncthreads();
        // frontier / unvisited pair-edge counts of level 0 (same in every CTA)
        unsigned long long pf_cur = 0, pu_cur = 0;
        {
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
            for (int s = 0; s < 4; ++s) { c->disc[s] = 0; c->pf[s] = 0; }
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
                if (a.tmark[t] == key0) continue;
                a.tmark[t] = key0;
                const uint32_t nch = (tf & kHubFlag) ? a.tiles[t].nchunks : 1u;
                for (uint32_t q = 0; q < nch; ++q) a.lists[n0++] = t + q;
            }
            a.lcnt[0] = n0;
        }
        // reset every row; roots at level 0 with sigma 1 (array 0)
        for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < a.n;
             v += (size_t)gridDim.x * blockDim.x) {
            uint16_t l[S];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const bool r = (sm.roots[k] == (uint32_t)v);
                l[k] = r ? (uint16_t)0 : kUnvisited;
                a.val[v * S + k] = r ? 1ull : 0ull;
                a.val[plane + v * S + k] = 0ull;
                a.val[2 * plane + v * S + k] = 0ull;
            }
            store_row<S>(a.lvl, (uint32_t)v, l);
        }
        if (!grid_sync(c, nblk, wait_ns)) return;
        trace(a, b, 0, 0, 0, 0);

        // ---- forward sweeps
        uint32_t d = 0;
        bool uall = true;              // no pull sweep yet: every tile may hold unvisited vertices
        unsigned long long ustart = 0; // ring position / length of the unvisited-tile list
        uint32_t ulen = 0;
        for (;;) {
            SweepCtx x;
            x.mode = (!a.directed && (double)pf_cur >= (double)a.push_pull_ratio * (double)pu_cur) ? kFwdPull
                                                                                                    : kFwdPush;
            x.d = d;
            x.D = 0;
            const uint32_t lb = vload32(a.lbase + d);
            const uint32_t lc = vload32(a.lcnt + d);
            x.lb_next = lb + lc;
            x.next_lvl = d + 1;
            x.key_next = tile_key(b, d + 1);
            x.own = a.val + (size_t)(d % 3) * plane;
            x.src = x.own;
            x.dst = a.val + (size_t)((d + 1) % 3) * plane;
            const unsigned long long ubefore = vload64(&c->uctr);
            if (threadIdx.x == 0) {
                sm.c_disc = 0; sm.c_pf = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) { sm.c_vis[k] = 0; sm.c_w[k] = 0; sm.c_mc[k] = 0; }
                if (blockIdx.x == 0) {
                    a.lbase[d + 1] = x.lb_next;
                    a.lcnt[d + 2] = 0;
                    c->disc[(d + 2) & 3] = 0;
                    c->pf[(d + 2) & 3] = 0;
                }
            }
            __syncthreads();
            uint32_t walked;
            if (x.mode == kFwdPull) {
                walked = uall ? a.ntiles : ulen;
                run_sweep<S>(a, sm, x, uall ? nullptr : a.ulist, ustart, walked, ring);
            } else {
                walked = lc;
                run_sweep<S>(a, sm, x, a.lists + lb, 0, lc, 0xFFFFFFFFull);
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
            trace(a, b, x.mode == kFwdPull ? 2u : 1u, d, walked, disc);
            if (x.mode == kFwdPull) {
                const unsigned long long uafter = vload64(&c->uctr);
                ustart = ubefore;
                ulen = (uint32_t)(uafter - ubefore);
                uall = false;
            }
            if (disc == 0) break;
            ++d;
            if (d > kMaxLevel) {
                if (blockIdx.x == 0 && threadIdx.x == 0) set_error(c, BCG_ERR_DEPTH);
                return;
            }
            pu_cur = pu_cur > pfn ? pu_cur - pfn : 0;
            pf_cur = pfn;
        }
        const uint32_t D = d;

        if (a.dbg_sigma) {
            for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < a.n;
                 v += (size_t)gridDim.x * blockDim.x) {
                const uint16_t L = a.lvl[v * S];
                a.dbg_sigma[v] = (L == kUnvisited) ? 0ull : a.val[(size_t)(L % 3) * plane + v * S];
            }
            if (!grid_sync(c, nblk, wait_ns)) return;
        }

        // ---- backward sweeps over the level lists
        const int lowest = a.dbg_delta ? 0 : 1;
        for (int dd = (int)D; dd >= lowest; --dd) {
            SweepCtx x;
            x.mode = kBwd;
            x.d = (uint32_t)dd;
            x.D = D;
            x.key_next = 0;
            x.lb_next = 0;
            x.next_lvl = 0;
            x.own = a.val + (size_t)(dd % 3) * plane;
            x.src = a.val + (size_t)((dd + 1) % 3) * plane;
            x.dst = nullptr;
            const uint32_t lb = vload32(a.lbase + dd);
            const uint32_t lc = vload32(a.lcnt + dd);
            run_sweep<S>(a, sm, x, a.lists + lb, 0, lc, 0xFFFFFFFFull);
            if (!grid_sync(c, nblk, wait_ns)) return;
            trace(a, b, 3u, (uint32_t)dd, lc, 0);
        }

        // ---- source term and per-root statistics
        if (blockIdx.x == 0 && threadIdx.x < S) {
            const int k = threadIdx.x;
            const uint32_t r = sm.roots[k];
            if (r != kNoRoot) {
                const size_t idx = (size_t)b * S + k;
                const unsigned long long W = vload64(&c->wsum[k]);
                const uint32_t p = a.pend[idx];
                if (p && W >= 2) a.bc[r] += (double)p * (double)(W - 2);
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

template <int S>
static int launch_impl(const BatchArgs &a, cudaStream_t st, int *grid_out) {
    const size_t smem = smem_bytes<S>();
    cudaError_t e = cudaFuncSetAttribute(bc_sweep_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return set_error(BCG_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bc_sweep_kernel<S>, kThreads, smem);
    if (e != cudaSuccess) return set_error(BCG_ERR_CUDA, "occupancy query: %s", cudaGetErrorString(e));
    if (per_sm < 1) return set_error(BCG_ERR_CUDA, "sweep kernel cannot be resident (smem %zu)", smem);
    int grid = nsm * per_sm;
    if (grid_out) *grid_out = grid;
    BatchArgs args = a;
    void *params[] = {&args};
    e = cudaLaunchCooperativeKernel((const void *)bc_sweep_kernel<S>, dim3(grid), dim3(kThreads), params, smem, st);
    if (e != cudaSuccess)
        return set_error(e == cudaErrorNoKernelImageForDevice ? BCG_ERR_NOGPU : BCG_ERR_CUDA,
                         "sweep kernel launch: %s", cudaGetErrorString(e));
    return BCG_OK;
}

int launch_sweep(int S, const BatchArgs &a, cudaStream_t st, int *grid_out) {
    switch (S) {
        case 1: return launch_impl<1>(a, st, grid_out);
        case 2: return launch_impl<2>(a, st, grid_out);
        case 4: return launch_impl<4>(a, st, grid_out);
        case 8: return launch_impl<8>(a, st, grid_out);
        default: return set_error(BCG_ERR_ARG, "batch width %d not in {1,2,4,8}", S);
    }
}

}  // namespace bcg
