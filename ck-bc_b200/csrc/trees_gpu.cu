// Iterated pendant-tree folding on the device (BCG_PRUNE_TREES).  The
// reference folds one layer of degree-1 vertices on the host
// (degree_reduction, bc2d.c:314-419, then init_bc_1degree / init_delta,
// bc2d.c:455-465, cuda_kernels.cu:1083-1098); here whole trees hanging off
// the graph's 2-core are folded, and the betweenness of the tree vertices
// is computed in closed form.
//
// Peeling runs in rounds.  Round r removes every vertex whose degree among
// the vertices not yet removed is 1; its one remaining neighbour becomes its
// parent, and a neighbour whose degree drops to 1 joins round r + 1.  Two
// degree-1 vertices adjacent to each other (the last edge of a tree) are
// resolved by id: the smaller stays.  So the removed vertices form trees
// rooted at the kept vertices (their anchors), children are removed in
// earlier rounds than their parents, and a component that is a tree keeps
// one vertex.  Subtree sizes are summed as vertices are removed (a vertex's
// children are all gone by then); anchors follow the rounds backwards.
//
// Exactness (ordered pairs (s, t), s a requested source):
//   - A path between two vertices of one tree, or between a tree vertex and
//     anything outside its tree, is unique inside the tree and enters the
//     core only through the anchor.  So a tree vertex v lies on the path of
//     (s, t) exactly when s and t sit in different branches at v (its child
//     subtrees and "the rest of the component"), and
//       bc[v] += sum over branches B at v of (sources in B) * (n_comp - 1 - |B|).
//   - An anchor a gets the same terms for its child subtrees; pairs with the
//     source outside its tree are counted by the core search.
//   - The core is searched from every anchor a that is requested or holds
//     requested sources in its tree, with weight mult(a) = [a in S] +
//     (sources in T_a), and every core vertex weighs 1 + reach (its tree's
//     size - 1) as a target (the engine's reach weights, init_delta).
// Every term is an integer below 2^53, so the device adds them with 64-bit
// integer atomics: the result does not depend on the order of the adds.
//
// The kept graph is renumbered so that the vertices that keep an edge come
// first (in their original order), by a device scan; its lists stay sorted.
// Components (for n_comp) are labelled by a union-find over the kept graph
// (roots hooked smaller-under-larger, so every component's root is its
// smallest internal id) and extended to the tree vertices through their
// anchors.
#include <algorithm>
#include <vector>

#include "bcg_common.hpp"
#include "engine_internal.hpp"

namespace bcg {

namespace {

constexpr uint32_t kKept = 0xFFFFFFFFu;  // rem[v] of a vertex that is not peeled

#define CKT(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_error(e_ == cudaErrorMemoryAllocation ? BCG_ERR_OOM : BCG_ERR_CUDA, "%s failed: %s", \
                             #call, cudaGetErrorString(e_));                                       \
    } while (0)

inline unsigned nblocks(uint64_t work, unsigned per) { return (unsigned)std::max<uint64_t>(1, (work + per - 1) / per); }

// ---- exclusive scan of uint32 counts (every partial sum fits 32 bits)
constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(kScanBlock) k_scan_block(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                           uint32_t *__restrict__ bsum, uint64_t len) {
    __shared__ uint32_t wsum[kScanBlock / 32];
    const uint64_t i = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t x = i < len ? in[i] : 0u;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = wsum[lane];
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= (unsigned)o) wi += y;
        }
        wsum[lane] = wi - w;
        if (lane == 31) bsum[blockIdx.x] = wi;
    }
    __syncthreads();
    if (i < len) out[i] = wsum[wid] + incl - x;
}

__global__ void k_scan_add(uint32_t *__restrict__ out, const uint32_t *__restrict__ boff, uint64_t len) {
    const uint64_t i = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < len) out[i] += boff[blockIdx.x];
}

// out[i] = in[0] + ... + in[i-1] (in and out may be the same array).
int scan_exclusive(const uint32_t *d_in, uint32_t *d_out, uint64_t len, cudaStream_t st) {
    if (len == 0) return BCG_OK;
    const uint64_t nb = (len + kScanBlock - 1) / kScanBlock;
    uint32_t *bsum = nullptr;
    CKT(cudaMalloc(&bsum, nb * sizeof(uint32_t)));
    k_scan_block<<<(unsigned)nb, kScanBlock, 0, st>>>(d_in, d_out, bsum, len);
    int rc = BCG_OK;
    if (cudaGetLastError() != cudaSuccess) rc = set_error(BCG_ERR_CUDA, "scan launch failed");
    if (!rc && nb > 1) {
        rc = scan_exclusive(bsum, bsum, nb, st);
        if (!rc) {
            k_scan_add<<<(unsigned)nb, kScanBlock, 0, st>>>(d_out, bsum, len);
            if (cudaGetLastError() != cudaSuccess) rc = set_error(BCG_ERR_CUDA, "scan launch failed");
        }
    }
    cudaStreamSynchronize(st);
    cudaFree(bsum);
    return rc;
}

// ---- peeling
__global__ void k_tp_init(uint32_t n, const uint32_t *__restrict__ offs, uint32_t *__restrict__ deg,
                          uint32_t *__restrict__ rem, uint32_t *__restrict__ parent, uint32_t *__restrict__ sz,
                          uint32_t *__restrict__ anchor, uint32_t *__restrict__ front, uint32_t *__restrict__ nfront) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint32_t d = offs[v + 1] - offs[v];
    deg[v] = d;
    rem[v] = kKept;
    parent[v] = kNoRoot;
    sz[v] = 1;
    anchor[v] = v;
    if (d == 1) front[atomicAdd(nfront, 1u)] = v;
}

// Round r, first half: every frontier vertex finds its remaining neighbour
// (nothing is removed yet, so all decisions see the state at the round's start).
__global__ void k_tp_decide(uint32_t nf, const uint32_t *__restrict__ front, const uint32_t *__restrict__ offs,
                            const uint32_t *__restrict__ adj, const uint32_t *__restrict__ deg,
                            const uint32_t *__restrict__ rem, uint32_t *__restrict__ cand) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const uint32_t v = front[i];
    uint32_t p = kNoRoot;
    if (deg[v] == 1) {
        for (uint32_t e = offs[v]; e < offs[v + 1]; ++e) {
            const uint32_t u = adj[e];
            if (rem[u] == kKept) {
                p = u;
                break;
            }
        }
        // the last edge of a tree: both ends have degree 1; the smaller id stays
        if (p != kNoRoot && deg[p] == 1 && v < p) p = kNoRoot;
    }
    cand[i] = p;
}

// Round r, second half: remove the decided vertices.
__global__ void k_tp_apply(uint32_t nf, const uint32_t *__restrict__ front, const uint32_t *__restrict__ cand,
                           uint32_t round, uint32_t *__restrict__ deg, uint32_t *__restrict__ rem,
                           uint32_t *__restrict__ parent, uint32_t *__restrict__ sz, uint32_t *__restrict__ next,
                           uint32_t *__restrict__ nnext, uint32_t *__restrict__ order, uint32_t *__restrict__ norder) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const uint32_t p = cand[i];
    if (p == kNoRoot) return;
    const uint32_t v = front[i];
    rem[v] = round;
    parent[v] = p;
    atomicAdd(sz + p, sz[v]);  // v's children left in earlier rounds: sz[v] is final
    order[atomicAdd(norder, 1u)] = v;
    if (atomicSub(deg + p, 1u) == 2u) next[atomicAdd(nnext, 1u)] = p;
}

__global__ void k_tp_anchor(uint32_t cnt, const uint32_t *__restrict__ ord, const uint32_t *__restrict__ parent,
                            const uint32_t *__restrict__ rem, uint32_t *__restrict__ anchor) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const uint32_t v = ord[i];
    const uint32_t p = parent[v];
    anchor[v] = rem[p] == kKept ? p : anchor[p];  // p left in a later round: its anchor is set
}

// Degree of each kept vertex among the kept vertices (one warp per vertex).
__global__ void k_tp_cdeg(uint32_t n, const uint32_t *__restrict__ offs, const uint32_t *__restrict__ adj,
                          const uint32_t *__restrict__ rem, uint32_t *__restrict__ cdeg) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (w >= n) return;
    const uint32_t v = (uint32_t)w;
    uint32_t c = 0;
    if (rem[v] == kKept)
        for (uint32_t e = offs[v] + lane; e < offs[v + 1]; e += 32) c += rem[adj[e]] == kKept;
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) cdeg[v] = c;
}

__global__ void k_tp_flag(uint32_t n, const uint32_t *__restrict__ cdeg, uint32_t *__restrict__ flag) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) flag[v] = cdeg[v] > 0;
}

// Internal numbering: vertices with kept edges first, then the rest, each in
// the caller's order (live[v] = live vertices before v).
__global__ void k_tp_number(uint32_t n, uint32_t nlive, const uint32_t *__restrict__ cdeg,
                            const uint32_t *__restrict__ live, uint32_t *__restrict__ intl, uint32_t *__restrict__ ext) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint32_t i = cdeg[v] ? live[v] : nlive + (v - live[v]);
    intl[v] = i;
    ext[i] = v;
}

__global__ void k_tp_len(uint32_t n, const uint32_t *__restrict__ ext, const uint32_t *__restrict__ cdeg,
                         uint32_t *__restrict__ len) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = cdeg[ext[i]];
    if (i == n) len[n] = 0;
}

// The kept lists in internal ids (one warp per live vertex; order kept, and
// the numbering is monotone on live vertices, so lists stay sorted).
__global__ void k_tp_fill(uint32_t nlive, const uint32_t *__restrict__ ext, const uint32_t *__restrict__ offs,
                          const uint32_t *__restrict__ adj, const uint32_t *__restrict__ rem,
                          const uint32_t *__restrict__ intl, const uint32_t *__restrict__ offs2,
                          uint32_t *__restrict__ adj2) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (w >= nlive) return;
    const uint32_t v = ext[w];
    uint32_t out = offs2[w];
    for (uint32_t b = offs[v]; b < offs[v + 1]; b += 32) {
        const uint32_t e = b + lane;
        uint32_t u = 0;
        bool keep = false;
        if (e < offs[v + 1]) {
            u = adj[e];
            keep = rem[u] == kKept;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) adj2[out + __popc(bal & ((1u << lane) - 1u))] = intl[u];
        out += __popc(bal);
    }
}

// Degree/reach words in internal ids: kept vertices weigh 1 + (tree size - 1).
__global__ void k_tp_vinfo(uint32_t n, const uint32_t *__restrict__ ext, const uint32_t *__restrict__ cdeg,
                           const uint32_t *__restrict__ rem, const uint32_t *__restrict__ sz, uint2 *__restrict__ vi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t v = ext[i];
    vi[i] = make_uint2(cdeg[v], rem[v] == kKept ? sz[v] - 1u : 0u);
}

// ---- union-find over the kept graph (internal ids).  root[x] <= x always,
// so path halving with plain stores only ever lowers a value.
__device__ __forceinline__ uint32_t uf_find(uint32_t *root, uint32_t v) {
    volatile uint32_t *r = root;
    uint32_t cur = r[v];
    if (cur == v) return v;
    uint32_t prev = v, next;
    while (cur > (next = r[cur])) {
        r[prev] = next;
        prev = cur;
        cur = next;
    }
    return cur;
}

__global__ void k_uf_init(uint32_t n, uint32_t *__restrict__ root) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) root[v] = v;
}

// One warp per live vertex hooks it to its larger neighbours.
__global__ void k_uf_link(uint32_t nlive, const uint32_t *__restrict__ offs2, const uint32_t *__restrict__ adj2,
                          uint32_t *root) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (w >= nlive) return;
    const uint32_t v = (uint32_t)w;
    for (uint32_t e = offs2[v] + lane; e < offs2[v + 1]; e += 32) {
        const uint32_t u = adj2[e];
        if (u <= v) continue;  // each edge once
        uint32_t a = uf_find(root, v), b = uf_find(root, u);
        while (a != b) {
            if (a < b) { const uint32_t t = a; a = b; b = t; }  // hook the larger root a under b
            const uint32_t old = atomicCAS(root + a, a, b);
            if (old == a) break;
            a = uf_find(root, old);
            b = uf_find(root, b);
        }
    }
}

// After linking every root is final.  The walk here stores nothing on the
// way (a path-halving store from one thread could land on root[v] after v's
// own thread wrote the final root and put back an interior ancestor), so
// root[v] is written once, by v's thread, with its root; a concurrent walk
// that reads it sees either v's old parent or the root, both on v's path.
__global__ void k_uf_flatten(uint32_t n, uint32_t *root) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    volatile uint32_t *r = root;
    uint32_t cur = v, next;
    while ((next = r[cur]) != cur) cur = next;
    root[v] = cur;
}

// Component of every vertex (its anchor's root, an internal id) and the
// vertex count of every component.
__global__ void k_tp_comp(uint32_t n, const uint32_t *__restrict__ anchor, const uint32_t *__restrict__ intl,
                          const uint32_t *__restrict__ root, uint32_t *__restrict__ comp,
                          unsigned long long *__restrict__ comp_n) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint32_t c = root[intl[anchor[v]]];
    comp[v] = c;
    atomicAdd(comp_n + c, 1ull);
}

__global__ void k_check_ids(uint64_t nnz, uint32_t n, const uint32_t *__restrict__ adj, unsigned long long *bad) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (uint64_t)gridDim.x * blockDim.x)
        if (adj[e] >= n) atomicMin(bad, (unsigned long long)e);
}

// ---- per-run tree terms
__global__ void k_tt_count(uint64_t k, const uint32_t *__restrict__ src, uint32_t *__restrict__ cnt) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) atomicAdd(cnt + src[i], 1u);
}

__global__ void k_tt_init(uint32_t n, const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ comp,
                          unsigned long long *__restrict__ sub, unsigned long long *__restrict__ csrc) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const uint32_t c = cnt[v];
    sub[v] = c;
    if (c) atomicAdd(csrc + comp[v], (unsigned long long)c);
}

__global__ void k_tt_sub(uint32_t cnt, const uint32_t *__restrict__ ord, const uint32_t *__restrict__ parent,
                         unsigned long long *sub) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const uint32_t v = ord[i];
    atomicAdd(sub + parent[v], sub[v]);  // v's subtree finished in earlier rounds
}

__global__ void k_tt_acc(uint32_t cnt, const uint32_t *__restrict__ ord, const uint32_t *__restrict__ parent,
                         const uint32_t *__restrict__ sz, const uint32_t *__restrict__ comp,
                         const unsigned long long *__restrict__ comp_n, const unsigned long long *__restrict__ sub,
                         const unsigned long long *__restrict__ csrc, unsigned long long *acc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const uint32_t v = ord[i];
    const uint32_t c = comp[v];
    const unsigned long long nc = comp_n[c], s = sub[v], z = sz[v];
    // v's subtree is a branch at its parent; the rest of the component is a branch at v
    if (s) atomicAdd(acc + parent[v], s * (nc - 1ull - z));
    const unsigned long long rest = csrc[c] - s;
    if (rest && z > 1) atomicAdd(acc + v, rest * (z - 1ull));
}

__global__ void k_tt_add(uint32_t n, const unsigned long long *__restrict__ acc, double *__restrict__ bc) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n && acc[v]) bc[v] += (double)acc[v];
}

}  // namespace

void tree_free(bcg_graph *g) {
    TreeDev &t = g->tdev;
    cudaFree(t.parent); cudaFree(t.sz); cudaFree(t.comp); cudaFree(t.comp_n); cudaFree(t.order);
    cudaFree(t.cnt); cudaFree(t.sub); cudaFree(t.csrc); cudaFree(t.acc); cudaFree(t.src);
    t = TreeDev{};
}

int prepare_trees(bcg_graph *g, const uint32_t *d_offs0, const uint32_t *d_adj0, uint64_t nnz, bool check_ids,
                  std::vector<uint32_t> &h_offs2) {
    const uint32_t n = g->n;
    cudaStream_t st = 0;
    TreeDev &t = g->tdev;
    uint32_t *deg = nullptr, *rem = nullptr, *anchor = nullptr, *cand = nullptr, *fa = nullptr, *fb = nullptr,
             *ctr = nullptr, *cdeg = nullptr, *tmp = nullptr, *intl = nullptr, *root = nullptr;
    unsigned long long *bad = nullptr;
    auto cleanup = [&]() {
        cudaFree(deg); cudaFree(rem); cudaFree(anchor); cudaFree(cand); cudaFree(fa); cudaFree(fb);
        cudaFree(ctr); cudaFree(cdeg); cudaFree(tmp); cudaFree(intl); cudaFree(root); cudaFree(bad);
    };
    struct Guard { decltype(cleanup) &f; ~Guard() { f(); } } guard{cleanup};
    const size_t nb = (size_t)n * sizeof(uint32_t);
    if (check_ids && nnz) {
        CKT(cudaMalloc(&bad, sizeof(unsigned long long)));
        CKT(cudaMemset(bad, 0xFF, sizeof(unsigned long long)));
        k_check_ids<<<148 * 8, 256, 0, st>>>(nnz, n, d_adj0, bad);
        unsigned long long hb = 0;
        CKT(cudaMemcpy(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost));
        if (hb != ~0ull) return set_error(BCG_ERR_ARG, "adj[%llu] >= n", hb);
    }
    CKT(cudaMalloc(&deg, nb));
    CKT(cudaMalloc(&rem, nb));
    CKT(cudaMalloc(&anchor, nb));
    CKT(cudaMalloc(&cand, nb));
    CKT(cudaMalloc(&fa, nb));
    CKT(cudaMalloc(&fb, nb));
    CKT(cudaMalloc(&ctr, 4 * sizeof(uint32_t)));
    CKT(cudaMalloc(&t.parent, nb));
    CKT(cudaMalloc(&t.sz, nb));
    CKT(cudaMalloc(&t.order, nb));
    CKT(cudaMemset(ctr, 0, 4 * sizeof(uint32_t)));
    // ctr[0]: frontier of the next round, ctr[1]: vertices removed so far
    k_tp_init<<<nblocks(n, 256), 256, 0, st>>>(n, d_offs0, deg, rem, t.parent, t.sz, anchor, fa, ctr);
    CKT(cudaGetLastError());
    uint32_t hc[2] = {0, 0};
    CKT(cudaMemcpy(hc, ctr, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    uint32_t nf = hc[0];
    t.round_off.assign(1, 0);
    for (uint32_t round = 0; nf; ++round) {
        CKT(cudaMemset(ctr, 0, sizeof(uint32_t)));
        k_tp_decide<<<nblocks(nf, 256), 256, 0, st>>>(nf, fa, d_offs0, d_adj0, deg, rem, cand);
        k_tp_apply<<<nblocks(nf, 256), 256, 0, st>>>(nf, fa, cand, round, deg, rem, t.parent, t.sz, fb, ctr, t.order,
                                                     ctr + 1);
        CKT(cudaGetLastError());
        CKT(cudaMemcpy(hc, ctr, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        t.round_off.push_back(hc[1]);
        nf = hc[0];
        std::swap(fa, fb);
    }
    t.npeeled = t.round_off.back();
    for (size_t r = t.round_off.size() - 1; r-- > 0;) {
        const uint32_t o = t.round_off[r], c = t.round_off[r + 1] - o;
        if (c) k_tp_anchor<<<nblocks(c, 256), 256, 0, st>>>(c, t.order + o, t.parent, rem, anchor);
    }
    CKT(cudaGetLastError());
    // the kept graph, renumbered
    CKT(cudaMalloc(&cdeg, nb));
    CKT(cudaMalloc(&tmp, nb + 4 * sizeof(uint32_t)));
    CKT(cudaMalloc(&intl, nb));
    CKT(cudaMalloc(&g->d_ext, nb));
    k_tp_cdeg<<<nblocks((uint64_t)n * 32, 256), 256, 0, st>>>(n, d_offs0, d_adj0, rem, cdeg);
    k_tp_flag<<<nblocks(n, 256), 256, 0, st>>>(n, cdeg, tmp);
    CKT(cudaGetLastError());
    CKT(cudaMemset(tmp + n, 0, sizeof(uint32_t)));
    int rc = scan_exclusive(tmp, tmp, (uint64_t)n + 1, st);
    if (rc) return rc;
    uint32_t nlive = 0;
    CKT(cudaMemcpy(&nlive, tmp + n, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    k_tp_number<<<nblocks(n, 256), 256, 0, st>>>(n, nlive, cdeg, tmp, intl, g->d_ext);
    k_tp_len<<<nblocks((uint64_t)n + 1, 256), 256, 0, st>>>(n, g->d_ext, cdeg, tmp);
    CKT(cudaGetLastError());
    // offsets with 4 entries of tail padding (the sweep reads 16-byte pieces)
    CKT(cudaMalloc(&g->d_offs, ((size_t)n + 1 + 4) * sizeof(uint32_t)));
    CKT(cudaMemset(g->d_offs + n + 1, 0, 4 * sizeof(uint32_t)));
    rc = scan_exclusive(tmp, g->d_offs, (uint64_t)n + 1, st);
    if (rc) return rc;
    h_offs2.resize((size_t)n + 1);
    CKT(cudaMemcpy(h_offs2.data(), g->d_offs, ((size_t)n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    const uint64_t nnz2 = h_offs2[n];
    CKT(cudaMalloc(&g->d_adj, (nnz2 + 4) * sizeof(uint32_t)));
    CKT(cudaMemset(g->d_adj + nnz2, 0, 4 * sizeof(uint32_t)));
    if (nlive)
        k_tp_fill<<<nblocks((uint64_t)nlive * 32, 256), 256, 0, st>>>(nlive, g->d_ext, d_offs0, d_adj0, rem, intl,
                                                                      g->d_offs, g->d_adj);
    CKT(cudaGetLastError());
    // degree/reach words (internal ids), kept for create_common's buffer
    CKT(cudaMalloc(&g->d_vinfo_trees, (size_t)n * sizeof(uint2)));
    k_tp_vinfo<<<nblocks(n, 256), 256, 0, st>>>(n, g->d_ext, cdeg, rem, t.sz, g->d_vinfo_trees);
    // components
    CKT(cudaMalloc(&root, nb));
    CKT(cudaMalloc(&t.comp, nb));
    CKT(cudaMalloc(&t.comp_n, (size_t)n * sizeof(unsigned long long)));
    CKT(cudaMemset(t.comp_n, 0, (size_t)n * sizeof(unsigned long long)));
    k_uf_init<<<nblocks(n, 256), 256, 0, st>>>(n, root);
    if (nlive) k_uf_link<<<nblocks((uint64_t)nlive * 32, 256), 256, 0, st>>>(nlive, g->d_offs, g->d_adj, root);
    k_uf_flatten<<<nblocks(n, 256), 256, 0, st>>>(n, root);
    k_tp_comp<<<nblocks(n, 256), 256, 0, st>>>(n, anchor, intl, root, t.comp, t.comp_n);
    CKT(cudaGetLastError());
    // per-run scratch of the tree terms
    CKT(cudaMalloc(&t.cnt, nb));
    CKT(cudaMalloc(&t.sub, (size_t)n * sizeof(unsigned long long)));
    CKT(cudaMalloc(&t.csrc, (size_t)n * sizeof(unsigned long long)));
    CKT(cudaMalloc(&t.acc, (size_t)n * sizeof(unsigned long long)));
    // host copies the source planning needs
    g->h_anchor.resize(n);
    g->h_cdeg.resize(n);
    g->h_intl.resize(n);
    g->h_sz.resize(n);
    CKT(cudaMemcpy(g->h_anchor.data(), anchor, nb, cudaMemcpyDeviceToHost));
    CKT(cudaMemcpy(g->h_cdeg.data(), cdeg, nb, cudaMemcpyDeviceToHost));
    CKT(cudaMemcpy(g->h_intl.data(), intl, nb, cudaMemcpyDeviceToHost));
    CKT(cudaMemcpy(g->h_sz.data(), t.sz, nb, cudaMemcpyDeviceToHost));
    g->tile_n = nlive ? nlive : 1;
    g->npruned = t.npeeled;
    return BCG_OK;
}

int tree_terms(bcg_graph *g, const std::vector<uint32_t> &src, cudaStream_t st) {
    TreeDev &t = g->tdev;
    const uint32_t n = g->n;
    if (src.empty()) return BCG_OK;
    if (t.src_cap < src.size()) {
        cudaFree(t.src);
        t.src = nullptr;
        t.src_cap = 0;
        CKT(cudaMalloc(&t.src, src.size() * sizeof(uint32_t)));
        t.src_cap = src.size();
    }
    CKT(cudaMemcpyAsync(t.src, src.data(), src.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CKT(cudaMemsetAsync(t.cnt, 0, (size_t)n * sizeof(uint32_t), st));
    CKT(cudaMemsetAsync(t.csrc, 0, (size_t)n * sizeof(unsigned long long), st));
    CKT(cudaMemsetAsync(t.acc, 0, (size_t)n * sizeof(unsigned long long), st));
    k_tt_count<<<nblocks(src.size(), 256), 256, 0, st>>>(src.size(), t.src, t.cnt);
    k_tt_init<<<nblocks(n, 256), 256, 0, st>>>(n, t.cnt, t.comp, t.sub, t.csrc);
    for (size_t r = 0; r + 1 < t.round_off.size(); ++r) {
        const uint32_t o = t.round_off[r], c = t.round_off[r + 1] - o;
        if (c) k_tt_sub<<<nblocks(c, 256), 256, 0, st>>>(c, t.order + o, t.parent, t.sub);
    }
    if (t.npeeled)
        k_tt_acc<<<nblocks(t.npeeled, 256), 256, 0, st>>>(t.npeeled, t.order, t.parent, t.sz, t.comp, t.comp_n, t.sub,
                                                          t.csrc, t.acc);
    k_tt_add<<<nblocks(n, 256), 256, 0, st>>>(n, t.acc, g->d_bc);
    CKT(cudaGetLastError());
    return BCG_OK;
}

}  // namespace bcg
