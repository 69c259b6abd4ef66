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
// Data layout (HBM, L2-resident for the target sizes): per vertex a row of S
// 16-bit levels (lvl[v*S + k]) and a row of S 64-bit values (val[v*S + k]);
// slot k belongs to the k-th root of the batch.  Sweeps walk static tiles of
// consecutive vertices (<= kTileEdges adjacency entries, <= kTileVerts
// vertices), handed out through a monotone ticket counter; vertices with more
// than kTileEdges neighbours are split into chunks whose partial sums meet in
// hub_acc, the last chunk to arrive finishing the vertex.
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
                __nanosleep(64);
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

template <int S>
struct Smem {
    uint32_t pre[kTileVerts + 1];
    uint32_t eb[kTileVerts];
    uint32_t mask[kTileVerts];
    unsigned long long acc[kTileVerts][S];
    unsigned long long own[kTileVerts][S];
    uint32_t warp_tot[kThreads / 32];
    unsigned long long ticket;
    int last;
    // per-CTA counters of the current sweep
    unsigned long long c_disc, c_pf;
    unsigned long long c_vis[S], c_w[S], c_mc[S];
    // batch constants
    uint32_t roots[S];
    double mult[S];
};

template <int S>
size_t smem_bytes() { return sizeof(Smem<S>); }

// Exclusive scan of one value per thread over the CTA; returns the total.
template <int S>
__device__ __forceinline__ uint32_t block_exclusive_scan(Smem<S> &sm, uint32_t x, uint32_t &excl) {
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    if (lane == 31) sm.warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < kThreads / 32 ? sm.warp_tot[lane] : 0;
        uint32_t ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= (unsigned)o) ti += y;
        }
        if (lane < kThreads / 32) sm.warp_tot[lane] = ti - t;  // exclusive warp offsets
        if (lane == kThreads / 32 - 1) sm.pre[kTileVerts] = ti;  // total (scratch slot)
    }
    __syncthreads();
    excl = sm.warp_tot[wid] + incl - x;
    return sm.pre[kTileVerts];
}

// Processes one tile in the given mode at level d (D = deepest level, used by
// the backward pass).
template <int S>
__device__ void process_tile(const BatchArgs &a, Smem<S> &sm, const Tile &T, int mode, uint32_t d,
                             uint32_t D) {
    const uint32_t tid = threadIdx.x;
    const bool hub = T.hub >= 0;
    const uint32_t nv = T.v1 - T.v0;
    uint32_t deg_act = 0;
    uint2 vi = make_uint2(0, 0);
    uint32_t m = 0;
    const uint16_t dl = (uint16_t)d;
    // ---- phase 1: activity of each vertex of the tile
    if (tid < nv) {
        const uint32_t v = T.v0 + tid;
        uint16_t l[S];
        load_row<S>(a.lvl, v, l);
#pragma unroll
        for (int k = 0; k < S; ++k) {
            if (mode == kFwdPull) m |= (uint32_t)(l[k] == kUnvisited) << k;
            else m |= (uint32_t)(l[k] == dl) << k;
        }
        vi = a.vinfo[v];
        const uint32_t ob = a.offs[v];
        uint32_t eb = hub ? T.e0 : ob;
        uint32_t ee = ob + vi.x;
        if (hub && T.e1 < ee) ee = T.e1;
        if (ee < eb) ee = eb;
        deg_act = m ? ee - eb : 0;
        if (mode == kBwd && d == D) deg_act = 0;
        sm.mask[tid] = m;
        sm.eb[tid] = eb;
#pragma unroll
        for (int k = 0; k < S; ++k) sm.acc[tid][k] = 0ull;
        if (mode != kFwdPull && m) {
#pragma unroll
            for (int k = 0; k < S; ++k)
                sm.own[tid][k] = ((m >> k) & 1u) ? a.val[(size_t)v * S + k] : 0ull;
        }
    }
    uint32_t excl;
    const uint32_t total = block_exclusive_scan<S>(sm, tid < nv ? deg_act : 0u, excl);
    if (tid < nv) sm.pre[tid] = excl;
    if (tid == 0) sm.pre[nv] = total;
    __syncthreads();

    // ---- phase 2: edges, a contiguous run of <= kItems per thread
    if (total) {
        const uint32_t per = (total + kThreads - 1) / kThreads;
        const uint32_t i0 = tid * per;
        const uint32_t i1 = min(total, i0 + per);
        if (i0 < i1) {
            // first local vertex j with pre[j] <= i0 < pre[j+1]
            uint32_t lo = 0, hi = nv;
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (sm.pre[mid] <= i0) lo = mid; else hi = mid;
            }
            uint32_t j = lo;
            uint32_t jj[kItems], uu[kItems];
#pragma unroll
            for (int q = 0; q < kItems; ++q) {
                const uint32_t i = i0 + q;
                if (i < i1) {
                    while (i >= sm.pre[j + 1]) ++j;
                    jj[q] = j;
                    uu[q] = __ldg(a.adj + sm.eb[j] + (i - sm.pre[j]));
                }
            }
            uint16_t ul[kItems][S];
#pragma unroll
            for (int q = 0; q < kItems; ++q)
                if (i0 + q < i1) load_row<S>(a.lvl, uu[q], ul[q]);

            if (mode == kFwdPush) {
#pragma unroll
                for (int q = 0; q < kItems; ++q) {
                    if (i0 + q >= i1) continue;
                    const uint32_t jm = sm.mask[jj[q]];
                    const uint32_t w = uu[q];
#pragma unroll
                    for (int k = 0; k < S; ++k) {
                        if (!((jm >> k) & 1u)) continue;
                        uint16_t L = ul[q][k];
                        bool take = (L == (uint16_t)(d + 1));
                        if (L == kUnvisited) {
                            uint16_t old = atomicCAS(reinterpret_cast<unsigned short *>(a.lvl) +
                                                         (size_t)w * S + k,
                                                     (unsigned short)kUnvisited, (unsigned short)(d + 1));
                            if (old == kUnvisited) {
                                const uint2 wi = a.vinfo[w];
                                atomicAdd(&sm.c_disc, 1ull);
                                atomicAdd(&sm.c_pf, (unsigned long long)wi.x);
                                atomicAdd(&sm.c_vis[k], 1ull);
                                atomicAdd(&sm.c_w[k], 1ull + wi.y);
                                atomicAdd(&sm.c_mc[k], (unsigned long long)wi.x + 2ull * wi.y);
                                take = true;
                            } else {
                                take = (old == (uint16_t)(d + 1));
                            }
                        }
                        if (take) {
                            const unsigned long long s = sm.own[jj[q]][k];
                            unsigned long long old = atomicAdd(a.val + (size_t)w * S + k, s);
                            if (old + s < s) a.ctrl->overflow = 1;
                        }
                    }
                }
            } else {
                const uint16_t want = (mode == kFwdPull) ? dl : (uint16_t)(d + 1);
                unsigned long long run[S];
#pragma unroll
                for (int k = 0; k < S; ++k) run[k] = 0ull;
                uint32_t runj = jj[0];
#pragma unroll
                for (int q = 0; q < kItems; ++q) {
                    if (i0 + q >= i1) continue;
                    if (jj[q] != runj) {
#pragma unroll
                        for (int k = 0; k < S; ++k) {
                            if (!run[k]) continue;
                            if (mode == kFwdPull) {
                                unsigned long long old = atomicAdd(&sm.acc[runj][k], run[k]);
                                if (old + run[k] < run[k]) a.ctrl->overflow = 1;
                            } else {
                                atomicAdd(reinterpret_cast<double *>(&sm.acc[runj][k]),
                                          __longlong_as_double((long long)run[k]));
                            }
                            run[k] = 0ull;
                        }
                        runj = jj[q];
                    }
                    const uint32_t jm = sm.mask[jj[q]];
                    const uint32_t w = uu[q];
#pragma unroll
                    for (int k = 0; k < S; ++k) {
                        if (((jm >> k) & 1u) && ul[q][k] == want) {
                            const unsigned long long x = a.val[(size_t)w * S + k];
                            if (mode == kFwdPull) {
                                unsigned long long t = run[k] + x;
                                if (t < x) a.ctrl->overflow = 1;
                                run[k] = t;
                            } else {
                                double t = __longlong_as_double((long long)run[k]) +
                                           __longlong_as_double((long long)x);
                                run[k] = (unsigned long long)__double_as_longlong(t);
                            }
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    if (!run[k]) continue;
                    if (mode == kFwdPull) {
                        unsigned long long old = atomicAdd(&sm.acc[runj][k], run[k]);
                        if (old + run[k] < run[k]) a.ctrl->overflow = 1;
                    } else {
                        atomicAdd(reinterpret_cast<double *>(&sm.acc[runj][k]),
                                  __longlong_as_double((long long)run[k]));
                    }
                }
            }
        }
    }
    __syncthreads();
    if (mode == kFwdPush) return;

    // ---- hub chunks: meet in hub_acc; the last chunk finishes the vertex
    if (hub) {
        const uint32_t hm = sm.mask[0];
        if (!hm) return;  // same decision in every chunk of this hub
        unsigned long long *hacc = a.hub_acc + (size_t)T.hub * S;
        if (tid < S && ((hm >> tid) & 1u)) {
            const unsigned long long x = sm.acc[0][tid];
            if (mode == kFwdPull) {
                unsigned long long old = atomicAdd(hacc + tid, x);
                if (old + x < x) a.ctrl->overflow = 1;
            } else {
                atomicAdd(reinterpret_cast<double *>(hacc + tid), __longlong_as_double((long long)x));
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            unsigned int old = atomicAdd(a.hub_cnt + T.hub, 1u);
            sm.last = (old == T.nchunks - 1);
        }
        __syncthreads();
        if (!sm.last) return;
        __threadfence();
        if (tid < S) sm.acc[0][tid] = atomicExch(hacc + tid, 0ull);
        if (tid == 0) atomicExch(a.hub_cnt + T.hub, 0u);
        __syncthreads();
    }

    // ---- phase 3: finish the tile's vertices
    if (tid < nv && m) {
        const uint32_t v = T.v0 + tid;
        if (mode == kFwdPull) {
            uint32_t nd = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (!((m >> k) & 1u)) continue;
                const unsigned long long s = sm.acc[tid][k];
                if (!s) continue;
                a.lvl[(size_t)v * S + k] = (uint16_t)(d + 1);
                a.val[(size_t)v * S + k] = s;
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
                const double sig = (double)sm.own[tid][k];
                const double acc = __longlong_as_double((long long)sm.acc[tid][k]);
                const double delta = reach + sig * acc;
                const double x = (1.0 + delta) / sig;
                a.val[(size_t)v * S + k] = (unsigned long long)__double_as_longlong(x);
                if (d > 0) add += sm.mult[k] * delta;
                if (a.dbg_delta) a.dbg_delta[v] = delta;
            }
            if (d > 0) a.bc[v] += add;
        }
    }
    __syncthreads();
}

template <int S>
__device__ void run_sweep(const BatchArgs &a, Smem<S> &sm, int mode, uint32_t d, uint32_t D,
                          unsigned long long &base) {
    for (;;) {
        if (threadIdx.x == 0) sm.ticket = atomicAdd(&a.ctrl->ticket, 1ull);
        __syncthreads();
        const long long ti = (long long)(sm.ticket - base);
        __syncthreads();
        if (ti >= (long long)a.ntiles) break;
        const Tile T = a.tiles[ti];
        process_tile<S>(a, sm, T, mode, d, D);
    }
    base += a.ntiles + gridDim.x;
}

template <int S>
__global__ void __launch_bounds__(kThreads, 2) bc_sweep_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<S> &sm = *reinterpret_cast<Smem<S> *>(smem_raw);
    Ctrl *c = a.ctrl;
    const unsigned int nblk = gridDim.x;
    const unsigned long long wait_ns = c->wait_ns ? c->wait_ns : kDefaultWaitNs;
    unsigned long long base = 0;

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
            c->depth = 0;
            for (int k = 0; k < S; ++k) {
                const uint32_t r = sm.roots[k];
                if (r == kNoRoot) continue;
                const uint2 ri = a.vinfo[r];
                c->visited[k] = 1;
                c->wsum[k] = 1ull + ri.y;
                c->mc2[k] = (unsigned long long)ri.x + 2ull * ri.y;
            }
        }
        // reset every row; roots at level 0 with sigma 1
        for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < a.n;
             v += (size_t)gridDim.x * blockDim.x) {
            uint16_t l[S];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const bool r = (sm.roots[k] == (uint32_t)v);
                l[k] = r ? (uint16_t)0 : kUnvisited;
                a.val[v * S + k] = r ? 1ull : 0ull;
            }
            store_row<S>(a.lvl, (uint32_t)v, l);
        }
        if (!grid_sync(c, nblk, wait_ns)) return;

        // ---- forward sweeps
        uint32_t d = 0;
        for (;;) {
            const int mode = (!a.directed && (double)pf_cur >= (double)a.push_pull_ratio * (double)pu_cur)
                                 ? kFwdPull : kFwdPush;
            if (threadIdx.x == 0) {
                sm.c_disc = 0; sm.c_pf = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) { sm.c_vis[k] = 0; sm.c_w[k] = 0; sm.c_mc[k] = 0; }
            }
            __syncthreads();
            run_sweep<S>(a, sm, mode, d, 0, base);
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
                if (blockIdx.x == 0) { c->disc[(d + 2) & 3] = 0; c->pf[(d + 2) & 3] = 0; }
            }
            // every CTA learns which slots discovered something at level d+1
            if (!grid_sync(c, nblk, wait_ns)) return;
            const unsigned long long disc = vload64(&c->disc[d & 3]);
            const unsigned long long pfn = vload64(&c->pf[d & 3]);
            if (disc == 0) break;
            ++d;
            if (d > kMaxLevel) {
                if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(&c->error, 0, BCG_ERR_DEPTH);
                return;
            }
            pu_cur = pu_cur > pfn ? pu_cur - pfn : 0;
            pf_cur = pfn;
        }
        const uint32_t D = d;

        if (a.dbg_sigma) {
            for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < a.n;
                 v += (size_t)gridDim.x * blockDim.x)
                a.dbg_sigma[v] = a.val[v * S];
            if (!grid_sync(c, nblk, wait_ns)) return;
        }

        // ---- backward sweeps
        const int lowest = a.dbg_delta ? 0 : 1;
        for (int dd = (int)D; dd >= lowest; --dd) {
            run_sweep<S>(a, sm, kBwd, (uint32_t)dd, D, base);
            if (!grid_sync(c, nblk, wait_ns)) return;
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
