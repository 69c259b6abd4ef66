// Iterated pendant-tree folding on the device (BCG_PRUNE_TREES).  The
// reference folds one layer of degree-1 vertices on the host
// (degree_reduction, bc2d.c:314-419, then init_bc_1degree / init_delta,
// bc2d.c:455-465, cuda_kernels.cu:1083-1098); here whole trees hanging off
// the graph's 2-core are folded, and the betweenness of the tree vertices
// is computed in closed form.  BCG_PRUNE_DEGREE1 is the same machinery
// stopped after the first round: exactly the reference's one layer (the
// same vertices fold into the same anchors, by the same pair rule), with the
// kept graph renumbered like the trees mode's.
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
// The argument needs only that every removed subtree hangs from the kept
// graph by one edge, so it holds when peeling stops after any round.
// Every term is an integer below 2^53, so the device adds them with 64-bit
// integer atomics: the result does not depend on the order of the adds.
//
// The kept graph is renumbered so that the vertices that keep an edge come
// first (in their original order), by a device scan; its lists stay sorted.
// Components (for n_comp) are labelled by a union-find over the kept graph
// (larger roots hooked under smaller ones, so every component's root is its
// smallest internal id; links in the Afforest order, k_uf_link_nth) and
// extended to the tree vertices through their anchors.
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
    CKT(tmp_alloc(&bsum, nb * sizeof(uint32_t), st));
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
    tmp_free(bsum, st);
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
// the numbering is monotone on live vertices, so lists stay sorted).  A
// neighbour u of a live vertex is kept exactly when it is live itself
// (intl[u] < nlive): a kept neighbour has that kept edge, a peeled one has no
// kept edge at all.
__global__ void k_tp_fill(uint32_t nlive, const uint32_t *__restrict__ ext, const uint32_t *__restrict__ offs,
                          const uint32_t *__restrict__ adj, const uint32_t *__restrict__ intl,
                          const uint32_t *__restrict__ offs2, uint32_t *__restrict__ adj2) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (w >= nlive) return;
    const uint32_t v = ext[w];
    uint32_t out = offs2[w];
    for (uint32_t b = offs[v]; b < offs[v + 1]; b += 32) {
        const uint32_t e = b + lane;
        uint32_t iu = nlive;
        if (e < offs[v + 1]) iu = intl[adj[e]];
        const bool keep = iu < nlive;
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) adj2[out + __popc(bal & ((1u << lane) - 1u))] = iu;
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

// Joins the sets of v and u: the larger root is hooked under the smaller
// one by a compare-and-swap (retried from the new roots when another thread
// hooked it first).
__device__ __forceinline__ void uf_link(uint32_t *root, uint32_t v, uint32_t u) {
    uint32_t a = uf_find(root, v), b = uf_find(root, u);
    while (a != b) {
        if (a < b) { const uint32_t t = a; a = b; b = t; }  // hook the larger root a under b
        const uint32_t old = atomicCAS(root + a, a, b);
        if (old == a) break;
        a = uf_find(root, old);
        b = uf_find(root, b);
    }
}

// Components in the manner of Afforest (Sutton, Ben-Nun and Barak, IPDPS
// 2018): every vertex is first linked to its first and its second neighbour
// only, after which most vertices already share the root of the largest
// component; then only the vertices outside it link their remaining
// neighbours.  The lists are symmetric, so an edge with an end outside the
// largest component is linked from that end, and an edge inside it joins
// nothing new.
__global__ void k_uf_link_nth(uint32_t nlive, const uint32_t *__restrict__ offs2, const uint32_t *__restrict__ adj2,
                              uint32_t *root, uint32_t j) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nlive) return;
    const uint32_t e = offs2[v] + j;
    if (e < offs2[v + 1]) uf_link(root, v, adj2[e]);
}

// One warp per live vertex outside the set of root `skip`: links its
// neighbours from the (from)-th on.  (A vertex whose root was rewritten
// meanwhile is simply linked in full.)
__global__ void k_uf_link_rest(uint32_t nlive, const uint32_t *__restrict__ offs2, const uint32_t *__restrict__ adj2,
                               uint32_t *root, uint32_t from, uint32_t skip) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (w >= nlive) return;
    const uint32_t v = (uint32_t)w;
    if (reinterpret_cast<volatile uint32_t *>(root)[v] == skip) return;
    for (uint32_t e = offs2[v] + from + lane; e < offs2[v + 1]; e += 32) uf_link(root, v, adj2[e]);
}

// root[i * nlive / kSamples] for the sampled vertices.
constexpr uint32_t kSamples = 1024;
__global__ void k_uf_sample(uint32_t nlive, const uint32_t *__restrict__ root, uint32_t *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kSamples) out[i] = root[(uint32_t)(((uint64_t)i * nlive) / kSamples)];
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
// (Most vertices share a component: the lanes of a warp that do add once.)
__global__ void k_tp_comp(uint32_t n, const uint32_t *__restrict__ anchor, const uint32_t *__restrict__ intl,
                          const uint32_t *__restrict__ root, uint32_t *__restrict__ comp,
                          unsigned long long *__restrict__ comp_n) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = v < n;
    const uint32_t c = ok ? root[intl[anchor[v]]] : 0u;
    if (ok) comp[v] = c;
    const unsigned active = __ballot_sync(0xffffffffu, ok);
    if (!ok) return;
    const unsigned peers = __match_any_sync(active, c);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(comp_n + c, (unsigned long long)__popc(peers));
}

__global__ void k_check_ids(uint64_t nnz, uint32_t n, const uint32_t *__restrict__ adj, unsigned long long *bad) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (uint64_t)gridDim.x * blockDim.x)
        if (adj[e] >= n) atomicMin(bad, (unsigned long long)e);
}

// What the run planning needs of each source s (ids checked < n on the
// host): its anchor a, and a's kept degree, internal id and tree size.
__global__ void k_src_info(uint64_t k, const uint32_t *__restrict__ src, const uint32_t *__restrict__ anchor,
                           const uint32_t *__restrict__ cdeg, const uint32_t *__restrict__ intl,
                           const uint32_t *__restrict__ sz, uint4 *__restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const uint32_t a = anchor[src[i]];
    out[i] = make_uint4(a, cdeg[a], intl[a], sz[a]);
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
    dev_free(t.parent); dev_free(t.sz); dev_free(t.comp); dev_free(t.comp_n); dev_free(t.order);
    dev_free(t.anchor); dev_free(t.intl); dev_free(t.cdeg);
    dev_free(t.cnt); dev_free(t.sub); dev_free(t.csrc); dev_free(t.acc); dev_free(t.src); dev_free(t.info);
    t = TreeDev{};
}

int prepare_trees(bcg_graph *g, const uint32_t *d_offs0, const uint32_t *d_adj0, uint64_t nnz, bool check_ids,
                  uint32_t max_rounds, std::vector<uint32_t> &h_offs2) {
    const uint32_t n = g->n;
    cudaStream_t st = 0;
    TreeDev &t = g->tdev;
    uint32_t *deg = nullptr, *rem = nullptr, *cand = nullptr, *fa = nullptr, *fb = nullptr, *ctr = nullptr,
             *tmp = nullptr, *root = nullptr;
    unsigned long long *bad = nullptr;
    auto cleanup = [&]() {
        tmp_free(deg, st); tmp_free(rem, st); tmp_free(cand, st); tmp_free(fa, st); tmp_free(fb, st);
        tmp_free(ctr, st); tmp_free(tmp, st); tmp_free(root, st); tmp_free(bad, st);
    };
    struct Guard { decltype(cleanup) &f; ~Guard() { f(); } } guard{cleanup};
    const size_t nb = (size_t)n * sizeof(uint32_t);
    if (check_ids && nnz) {
        CKT(tmp_alloc(&bad, sizeof(unsigned long long), st));
        CKT(cudaMemset(bad, 0xFF, sizeof(unsigned long long)));
        k_check_ids<<<148 * 8, 256, 0, st>>>(nnz, n, d_adj0, bad);
        unsigned long long hb = 0;
        CKT(cudaMemcpy(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost));
        if (hb != ~0ull) return set_error(BCG_ERR_ARG, "adj[%llu] >= n", hb);
    }
    CKT(tmp_alloc(&deg, nb, st));
    CKT(tmp_alloc(&rem, nb, st));
    CKT(dev_alloc(&t.anchor, nb));
    uint32_t *const anchor = t.anchor;
    CKT(tmp_alloc(&cand, nb, st));
    CKT(tmp_alloc(&fa, nb, st));
    CKT(tmp_alloc(&fb, nb, st));
    CKT(tmp_alloc(&ctr, 4 * sizeof(uint32_t), st));
    CKT(dev_alloc(&t.parent, nb));
    CKT(dev_alloc(&t.sz, nb));
    CKT(dev_alloc(&t.order, nb));
    CKT(cudaMemset(ctr, 0, 4 * sizeof(uint32_t)));
    // ctr[0]: frontier of the next round, ctr[1]: vertices removed so far
    k_tp_init<<<nblocks(n, 256), 256, 0, st>>>(n, d_offs0, deg, rem, t.parent, t.sz, anchor, fa, ctr);
    CKT(cudaGetLastError());
    uint32_t hc[2] = {0, 0};
    CKT(cudaMemcpy(hc, ctr, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    uint32_t nf = hc[0];
    t.round_off.assign(1, 0);
    for (uint32_t round = 0; nf && round < max_rounds; ++round) {
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
    CKT(dev_alloc(&t.cdeg, nb));
    CKT(tmp_alloc(&tmp, nb + 4 * sizeof(uint32_t), st));
    CKT(dev_alloc(&t.intl, nb));
    uint32_t *const cdeg = t.cdeg, *const intl = t.intl;
    CKT(dev_alloc(&g->d_ext, nb));
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
    CKT(dev_alloc(&g->d_offs, ((size_t)n + 1 + 4) * sizeof(uint32_t)));
    CKT(cudaMemset(g->d_offs + n + 1, 0, 4 * sizeof(uint32_t)));
    rc = scan_exclusive(tmp, g->d_offs, (uint64_t)n + 1, st);
    if (rc) return rc;
    h_offs2.resize((size_t)n + 1);
    CKT(cudaMemcpy(h_offs2.data(), g->d_offs, ((size_t)n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    const uint64_t nnz2 = h_offs2[n];
    CKT(dev_alloc(&g->d_adj, (nnz2 + 4) * sizeof(uint32_t)));
    CKT(cudaMemset(g->d_adj + nnz2, 0, 4 * sizeof(uint32_t)));
    if (nlive)
        k_tp_fill<<<nblocks((uint64_t)nlive * 32, 256), 256, 0, st>>>(nlive, g->d_ext, d_offs0, d_adj0, intl,
                                                                      g->d_offs, g->d_adj);
    CKT(cudaGetLastError());
    // degree/reach words (internal ids), kept for create_common's buffer
    CKT(dev_alloc(&g->d_vinfo_trees, (size_t)n * sizeof(uint2)));
    k_tp_vinfo<<<nblocks(n, 256), 256, 0, st>>>(n, g->d_ext, cdeg, rem, t.sz, g->d_vinfo_trees);
    // components
    CKT(tmp_alloc(&root, nb, st));
    CKT(dev_alloc(&t.comp, nb));
    CKT(dev_alloc(&t.comp_n, (size_t)n * sizeof(unsigned long long)));
    CKT(cudaMemset(t.comp_n, 0, (size_t)n * sizeof(unsigned long long)));
    k_uf_init<<<nblocks(n, 256), 256, 0, st>>>(n, root);
    if (nlive) {
        for (uint32_t j = 0; j < 2; ++j) {
            k_uf_link_nth<<<nblocks(nlive, 256), 256, 0, st>>>(nlive, g->d_offs, g->d_adj, root, j);
            k_uf_flatten<<<nblocks(nlive, 256), 256, 0, st>>>(nlive, root);
        }
        // the most frequent root among evenly spaced samples
        uint32_t *d_smp = nullptr;
        CKT(tmp_alloc(&d_smp, kSamples * sizeof(uint32_t), st));
        k_uf_sample<<<nblocks(kSamples, 256), 256, 0, st>>>(nlive, root, d_smp);
        std::vector<uint32_t> smp(kSamples);
        const cudaError_t ce = cudaMemcpy(smp.data(), d_smp, kSamples * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        tmp_free(d_smp, st);
        CKT(ce);
        std::sort(smp.begin(), smp.end());
        uint32_t giant = smp[0], best = 0;
        for (size_t i = 0; i < smp.size();) {
            size_t j = i;
            while (j < smp.size() && smp[j] == smp[i]) ++j;
            if (j - i > best) { best = (uint32_t)(j - i); giant = smp[i]; }
            i = j;
        }
        k_uf_link_rest<<<nblocks((uint64_t)nlive * 32, 256), 256, 0, st>>>(nlive, g->d_offs, g->d_adj, root, 2u, giant);
    }
    k_uf_flatten<<<nblocks(n, 256), 256, 0, st>>>(n, root);
    k_tp_comp<<<nblocks(n, 256), 256, 0, st>>>(n, anchor, intl, root, t.comp, t.comp_n);
    CKT(cudaGetLastError());
    // per-run scratch of the tree terms
    CKT(dev_alloc(&t.cnt, nb));
    CKT(dev_alloc(&t.sub, (size_t)n * sizeof(unsigned long long)));
    CKT(dev_alloc(&t.csrc, (size_t)n * sizeof(unsigned long long)));
    CKT(dev_alloc(&t.acc, (size_t)n * sizeof(unsigned long long)));
    g->tile_n = nlive ? nlive : 1;
    g->npruned = t.npeeled;
    return BCG_OK;
}

int tree_source_info(bcg_graph *g, const uint32_t *src, uint64_t k, std::vector<uint4> &info, cudaStream_t st) {
    TreeDev &t = g->tdev;
    t.nsrc = 0;
    info.resize(k);
    if (k == 0) return BCG_OK;
    if (t.src_cap < k) {
        CKT(cudaDeviceSynchronize());  // earlier runs (any stream) are done with the old buffers
        dev_free(t.src);
        dev_free(t.info);
        t.src = nullptr;
        t.info = nullptr;
        t.src_cap = 0;
        CKT(dev_alloc(&t.src, k * sizeof(uint32_t)));
        CKT(dev_alloc(&t.info, k * sizeof(uint4)));
        CKT(cudaDeviceSynchronize());  // ready for stream st
        t.src_cap = k;
    }
    CKT(cudaMemcpyAsync(t.src, src, k * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    k_src_info<<<nblocks(k, 256), 256, 0, st>>>(k, t.src, t.anchor, t.cdeg, t.intl, t.sz, t.info);
    CKT(cudaGetLastError());
    CKT(cudaMemcpyAsync(info.data(), t.info, k * sizeof(uint4), cudaMemcpyDeviceToHost, st));
    CKT(cudaStreamSynchronize(st));
    t.nsrc = k;
    return BCG_OK;
}

int tree_terms(bcg_graph *g, cudaStream_t st, uint64_t *launches) {
    TreeDev &t = g->tdev;
    const uint32_t n = g->n;
    const uint64_t k = t.nsrc;
    *launches = 0;
    if (k == 0) return BCG_OK;
    CKT(cudaMemsetAsync(t.cnt, 0, (size_t)n * sizeof(uint32_t), st));
    CKT(cudaMemsetAsync(t.csrc, 0, (size_t)n * sizeof(unsigned long long), st));
    CKT(cudaMemsetAsync(t.acc, 0, (size_t)n * sizeof(unsigned long long), st));
    k_tt_count<<<nblocks(k, 256), 256, 0, st>>>(k, t.src, t.cnt);
    k_tt_init<<<nblocks(n, 256), 256, 0, st>>>(n, t.cnt, t.comp, t.sub, t.csrc);
    uint64_t nl = 3;  // count, init, add
    for (size_t r = 0; r + 1 < t.round_off.size(); ++r) {
        const uint32_t o = t.round_off[r], c = t.round_off[r + 1] - o;
        if (c) {
            k_tt_sub<<<nblocks(c, 256), 256, 0, st>>>(c, t.order + o, t.parent, t.sub);
            ++nl;
        }
    }
    if (t.npeeled) {
        k_tt_acc<<<nblocks(t.npeeled, 256), 256, 0, st>>>(t.npeeled, t.order, t.parent, t.sz, t.comp, t.comp_n, t.sub,
                                                          t.csrc, t.acc);
        ++nl;
    }
    k_tt_add<<<nblocks(n, 256), 256, 0, st>>>(n, t.acc, g->d_bc);
    CKT(cudaGetLastError());
    *launches = nl;
    return BCG_OK;
}

}  // namespace bcg
