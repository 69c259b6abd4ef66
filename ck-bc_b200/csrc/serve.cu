// Serving form: BC requests against a pool of resident graphs, admitted under
// an HBM budget and run with continuous batching (no counterpart in the
// reference, whose program computes one graph per process).
//
// The pool is uploaded once as one disjoint union whose tiles never cross a
// graph boundary, so each graph owns a contiguous range of tiles.  A request
// asks for the BC of one graph over a list of sources (or all of its
// vertices); its result buffer (one double per vertex of the graph) is
// allocated when it is admitted, FIFO, while the pool plus the admitted
// buffers fit the budget.  Each graph serves its admitted requests in order.
//
// bcg_server_step runs one wave: every graph with an admitted request
// advances its first request by a chunk of up to wave_batches * S sources, all
// of them packed into one persistent launch (component-packed batches: a
// graph's sources fill the S slots of successive batches, graphs share the
// batches; S is 6 while the active graphs' 64-byte state rows fit 64 MB, as
// in bcg_run, else 3).  The first pull of a batch walks only the tile ranges of the
// graphs active in it.  After the launch a drain kernel adds each active
// graph's slice of the union's bc into its request's buffer and clears the
// slice.  A request that arrives while a wave runs joins the next one, so the
// GPU always works on every admitted request at once, and large requests do
// not hold small ones back for longer than one wave.  Every source of a
// request adds the same dependencies alone or in a mix; only the grouping of
// those floating-point sums into waves may differ with the wave width.
#include <algorithm>
#include <deque>
#include <unordered_map>
#include <vector>

#include "bcg_common.hpp"
#include "engine_internal.hpp"

using namespace bcg;

namespace {

struct Req {
    uint32_t graph = 0;
    std::vector<uint32_t> src;  // union ids of the request's non-isolated sources, in order
    size_t next = 0;            // sources already run
    double *d_out = nullptr;    // one accumulator per vertex of the graph (from admission on)
    size_t bytes = 0;
    bool done = false;
};

struct DrainItem {
    double *out;
    uint32_t base;
    uint32_t n;
};

// out[v] += bc[base + v]; bc[base + v] = 0 for every listed graph slice.
__global__ void k_drain(const DrainItem *__restrict__ items, uint32_t nitems, double *__restrict__ bc) {
    for (uint32_t it = blockIdx.y; it < nitems; it += gridDim.y) {
        const DrainItem d = items[it];
        for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < d.n; v += gridDim.x * blockDim.x) {
            double *p = bc + d.base + v;
            d.out[v] += *p;
            *p = 0.0;
        }
    }
}

size_t up16(size_t x) { return (x + 15) & ~size_t(15); }

}  // namespace

struct bcg_server {
    bcg_graph *g = nullptr;
    uint32_t ngraphs = 0;
    std::vector<uint32_t> base, gn, order, hdeg;
    std::vector<uint2> grange;    // per caller graph: its tiles [x, y)
    std::vector<uint64_t> gnnz;
    uint64_t budget = 0, resident = 0, admitted = 0;
    uint32_t width = 6, wave_batches = 64;  // width: the widest a wave may use
    std::unordered_map<uint64_t, Req> reqs;
    uint64_t next_id = 1;
    std::deque<uint64_t> pending;
    std::vector<std::deque<uint64_t>> queue;  // per graph: admitted requests in order
    std::deque<uint64_t> done;                // finished, not yet reported
    // wave schedule: one device region and one pinned staging copy, sized for
    // the largest wave (wave_batches batches, every graph active)
    size_t off_xbeg = 0, off_xroots = 0, off_xslot = 0, off_xpf = 0, off_xpu = 0, off_xtiles = 0, off_xrbeg = 0,
           off_xrange = 0, off_drain = 0, blob_bytes = 0;
    unsigned char *d_blob = nullptr, *h_blob = nullptr;
    RootStat *d_rstat = nullptr;
    cudaStream_t stream = nullptr;
    uint64_t waves = 0;
};

namespace {

#define CKS(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_error(e_ == cudaErrorMemoryAllocation ? BCG_ERR_OOM : BCG_ERR_CUDA, "%s failed: %s", \
                             #call, cudaGetErrorString(e_));                                       \
    } while (0)

// Device bytes the resident pool holds (CSR, per-vertex state of width S,
// tiles and their lists).
uint64_t pool_bytes(const bcg_graph *g, uint32_t S) {
    const uint64_t n = g->n, t = g->ntiles;
    return 4 * (n + 1) + 4 * (g->nnz + 4) + 8 * n /*vinfo*/ + 8 * n /*bc*/ + (uint64_t)row_bytes((int)S) * n +
           32 * t + 4 * n /*tile_of*/ + 4 * t /*tmark*/ + 8 * t /*ring*/ + 4ull * S * (n + t) /*lists*/ +
           8ull * (kMaxLevel + 3);
}

// Admits pending requests, FIFO, while their buffers fit the budget.
int admit(bcg_server *s) {
    while (!s->pending.empty()) {
        Req &r = s->reqs[s->pending.front()];
        if (s->resident + s->admitted + r.bytes > s->budget) break;
        CKS(cudaMallocAsync(reinterpret_cast<void **>(&r.d_out), r.bytes, s->stream));
        CKS(cudaMemsetAsync(r.d_out, 0, r.bytes, s->stream));
        s->admitted += r.bytes;
        s->queue[r.graph].push_back(s->pending.front());
        s->pending.pop_front();
    }
    return BCG_OK;
}

}  // namespace

extern "C" {

int bcg_server_create(uint32_t ngraphs, const uint32_t *const *offsets, const uint32_t *const *adj,
                      const uint32_t *n, uint64_t hbm_budget_bytes, uint32_t wave_batches, bcg_server **out) {
    clear_error();
    if (!out) return set_error(BCG_ERR_ARG, "null output handle");
    *out = nullptr;
    if (wave_batches == 0 || wave_batches > 65535) return set_error(BCG_ERR_ARG, "wave_batches must be 1..65535");
    bcg_server *s = new bcg_server();
    int rc = make_union(ngraphs, offsets, adj, n, false, s->order, s->base, s->hdeg, &s->g);
    if (rc) {
        delete s;
        return rc;
    }
    auto fail = [&](int code) {
        bcg_server_destroy(s);
        return code;
    };
    s->ngraphs = ngraphs;
    s->gn.assign(n, n + ngraphs);
    s->wave_batches = wave_batches;
    s->queue.resize(ngraphs);
    // tiles that never cross a graph boundary: graph g owns tiles [x, y)
    std::vector<uint32_t> breaks(ngraphs);
    for (uint32_t i = 0; i < ngraphs; ++i) breaks[i] = s->base[i];
    std::sort(breaks.begin(), breaks.end());
    s->g->tile_breaks = breaks;
    rc = graph_retile(s->g, s->g->tile_vcap, s->g->tile_ecap, true);
    if (rc) return fail(rc);
    std::vector<uint32_t> tile_of(s->g->n);
    if (cudaMemcpy(tile_of.data(), s->g->d_tile_of, tile_of.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return fail(set_error(BCG_ERR_CUDA, "reading tiles"));
    s->grange.resize(ngraphs);
    s->gnnz.assign(ngraphs, 0);
    for (uint32_t p = 0; p < ngraphs; ++p) {
        const uint32_t gi = s->order[p];
        const uint32_t t0 = tile_of[s->base[gi]] & ~kHubFlag;
        const uint32_t t1 = (p + 1 < ngraphs) ? (tile_of[s->base[s->order[p + 1]]] & ~kHubFlag) : s->g->ntiles;
        s->grange[gi] = make_uint2(t0, t1);
        for (uint32_t v = 0; v < n[gi]; ++v) s->gnnz[gi] += s->hdeg[s->base[gi] + v];
    }
    rc = ensure_state(s->g, s->width);
    if (rc) return fail(rc);
    s->budget = hbm_budget_bytes;
    s->resident = pool_bytes(s->g, s->width);
    if (s->resident > s->budget)
        return fail(set_error(BCG_ERR_OOM, "the resident pool needs %llu bytes, over the %llu-byte budget",
                              (unsigned long long)s->resident, (unsigned long long)s->budget));
    // wave schedule regions
    const size_t W = wave_batches, G = ngraphs, S = s->width, R = W * G * S;
    size_t o = 0;
    s->off_xbeg = o; o += up16((W + 1) * 4);
    s->off_xroots = o; o += up16(R * 4);
    s->off_xslot = o; o += up16(R);
    s->off_xpf = o; o += up16(W * 8);
    s->off_xpu = o; o += up16(W * 8);
    s->off_xtiles = o; o += up16(W * 4);
    s->off_xrbeg = o; o += up16((W + 1) * 4);
    s->off_xrange = o; o += up16(W * G * 8);
    s->off_drain = o; o += up16(G * sizeof(DrainItem));
    s->blob_bytes = o;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_blob, o)) != cudaSuccess || (e = cudaMallocHost(&s->h_blob, o)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_rstat, W * S * sizeof(RootStat))) != cudaSuccess)
        return fail(set_error(BCG_ERR_CUDA, "server buffers: %s", cudaGetErrorString(e)));
    s->resident += o + W * S * sizeof(RootStat);
    *out = s;
    return BCG_OK;
}

int bcg_server_destroy(bcg_server *s) {
    clear_error();
    if (!s) return set_error(BCG_ERR_ARG, "null handle");
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &kv : s->reqs)
        if (kv.second.d_out) cudaFree(kv.second.d_out);
    cudaFree(s->d_blob);
    cudaFree(s->d_rstat);
    if (s->h_blob) cudaFreeHost(s->h_blob);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->g) bcg_graph_destroy(s->g);
    delete s;
    return BCG_OK;
}

int bcg_server_submit(bcg_server *s, uint32_t graph, const uint32_t *sources, uint64_t nsrc, uint64_t *id) {
    clear_error();
    if (!s || !id) return set_error(BCG_ERR_ARG, "null argument");
    if (graph >= s->ngraphs) return set_error(BCG_ERR_ARG, "graph %u >= %u graphs", graph, s->ngraphs);
    if (nsrc && !sources) return set_error(BCG_ERR_ARG, "null sources");
    Req r;
    r.graph = graph;
    r.bytes = (size_t)s->gn[graph] * sizeof(double);
    if (s->resident + r.bytes > s->budget)
        return set_error(BCG_ERR_OOM, "a result buffer of %zu bytes can never fit the budget", r.bytes);
    const uint32_t b = s->base[graph];
    if (nsrc == 0) {  // every vertex of the graph
        for (uint32_t v = 0; v < s->gn[graph]; ++v)
            if (s->hdeg[b + v]) r.src.push_back(b + v);
    } else {
        for (uint64_t i = 0; i < nsrc; ++i) {
            if (sources[i] >= s->gn[graph])
                return set_error(BCG_ERR_ARG, "source %u >= n=%u of graph %u", sources[i], s->gn[graph], graph);
            if (s->hdeg[b + sources[i]]) r.src.push_back(b + sources[i]);  // degree 0: skipped, as bcg_run
        }
    }
    *id = s->next_id++;
    s->reqs.emplace(*id, std::move(r));
    s->pending.push_back(*id);
    return BCG_OK;
}

int bcg_server_step(bcg_server *s, uint64_t *done_ids, uint32_t cap, uint32_t *ndone) {
    clear_error();
    if (!s || !ndone || (cap && !done_ids)) return set_error(BCG_ERR_ARG, "null argument");
    *ndone = 0;
    int rc = admit(s);
    if (rc) return rc;
    const uint32_t G = s->ngraphs, W = s->wave_batches;
    // the graphs active in this wave; the wave's width follows bcg_run's rule:
    // 6 sources per batch while the active graphs' 64-byte state rows fit
    // 64 MB (they then stay in L2), else 3
    std::vector<uint32_t> act;  // caller graph ids
    uint64_t act_n = 0;
    for (uint32_t gi = 0; gi < G; ++gi) {
        auto &q = s->queue[gi];
        while (!q.empty() && s->reqs[q.front()].next >= s->reqs[q.front()].src.size()) {
            s->reqs[q.front()].done = true;
            s->done.push_back(q.front());
            q.pop_front();
        }
        if (q.empty()) continue;
        act.push_back(gi);
        act_n += s->gn[gi];
    }
    const uint32_t S = (act_n * (uint64_t)row_bytes(6) <= (64ull << 20)) ? 6u : 3u;
    std::vector<size_t> c0, c1;  // the chunk each active graph runs in this wave
    for (uint32_t gi : act) {
        const Req &r = s->reqs[s->queue[gi].front()];
        c0.push_back(r.next);
        c1.push_back(std::min(r.src.size(), r.next + (size_t)W * S));
    }
    if (!act.empty()) {
        uint32_t nb = 0;
        for (size_t a = 0; a < act.size(); ++a) nb = std::max<uint32_t>(nb, (uint32_t)((c1[a] - c0[a] + S - 1) / S));
        unsigned char *h = s->h_blob;
        auto *xbeg = reinterpret_cast<uint32_t *>(h + s->off_xbeg);
        auto *xroots = reinterpret_cast<uint32_t *>(h + s->off_xroots);
        auto *xslot = h + s->off_xslot;
        auto *xpf = reinterpret_cast<unsigned long long *>(h + s->off_xpf);
        auto *xpu = reinterpret_cast<unsigned long long *>(h + s->off_xpu);
        auto *xtiles = reinterpret_cast<uint32_t *>(h + s->off_xtiles);
        auto *xrbeg = reinterpret_cast<uint32_t *>(h + s->off_xrbeg);
        auto *xrange = reinterpret_cast<uint2 *>(h + s->off_xrange);
        auto *drain = reinterpret_cast<DrainItem *>(h + s->off_drain);
        uint32_t nr = 0, nrange = 0;
        xbeg[0] = 0;
        xrbeg[0] = 0;
        for (uint32_t i = 0; i < nb; ++i) {
            xpf[i] = xpu[i] = 0;
            uint32_t cum = 0;
            for (size_t a = 0; a < act.size(); ++a) {
                const size_t j0 = c0[a] + (size_t)i * S;
                if (j0 >= c1[a]) continue;
                const uint32_t gi = act[a];
                const Req &r = s->reqs[s->queue[gi].front()];
                for (uint32_t k = 0; k < S && j0 + k < c1[a]; ++k) {
                    const uint32_t v = r.src[j0 + k];
                    xroots[nr] = v;
                    xslot[nr] = (unsigned char)k;
                    ++nr;
                    xpf[i] += s->hdeg[v];
                    xpu[i] += s->gnnz[gi] - s->hdeg[v];
                }
                xrange[nrange++] = make_uint2(s->grange[gi].x, cum);
                cum += s->grange[gi].y - s->grange[gi].x;
            }
            xbeg[i + 1] = nr;
            xrbeg[i + 1] = nrange;
            xtiles[i] = cum;
        }
        for (size_t a = 0; a < act.size(); ++a) {
            const uint32_t gi = act[a];
            drain[a] = DrainItem{s->reqs[s->queue[gi].front()].d_out, s->base[gi], s->gn[gi]};
        }
        CKS(cudaMemcpyAsync(s->d_blob, s->h_blob, s->blob_bytes, cudaMemcpyHostToDevice, s->stream));
        unsigned char *d = s->d_blob;
        PackedRun p{};
        p.xbeg = reinterpret_cast<const uint32_t *>(d + s->off_xbeg);
        p.xroots = reinterpret_cast<const uint32_t *>(d + s->off_xroots);
        p.xslot = d + s->off_xslot;
        p.xpf = reinterpret_cast<const unsigned long long *>(d + s->off_xpf);
        p.xpu = reinterpret_cast<const unsigned long long *>(d + s->off_xpu);
        p.xtiles = reinterpret_cast<const uint32_t *>(d + s->off_xtiles);
        p.xrbeg = reinterpret_cast<const uint32_t *>(d + s->off_xrbeg);
        p.xrange = reinterpret_cast<const uint2 *>(d + s->off_xrange);
        p.nbatch = nb;
        p.rstat = s->d_rstat;
        rc = enqueue_packed(s->g, p, S, s->stream);
        if (rc) return rc;
        double *d_bc = nullptr;
        rc = bcg_bc_device_ptr(s->g, &d_bc);
        if (rc) return rc;
        uint32_t maxn = 0;
        for (uint32_t gi : act) maxn = std::max(maxn, s->gn[gi]);
        const dim3 grid(std::min<uint32_t>((maxn + 255) / 256, 64u), (unsigned)act.size());
        k_drain<<<grid, 256, 0, s->stream>>>(reinterpret_cast<const DrainItem *>(d + s->off_drain),
                                             (uint32_t)act.size(), d_bc);
        CKS(cudaGetLastError());
        rc = check_ctrl(s->g, s->stream);
        if (rc) return rc;
        ++s->waves;
        for (size_t a = 0; a < act.size(); ++a) {
            const uint32_t gi = act[a];
            const uint64_t rid = s->queue[gi].front();
            Req &r = s->reqs[rid];
            r.next = c1[a];
            if (r.next >= r.src.size()) {
                r.done = true;
                s->done.push_back(rid);
                s->queue[gi].pop_front();
            }
        }
    }
    while (!s->done.empty() && *ndone < cap) {
        done_ids[(*ndone)++] = s->done.front();
        s->done.pop_front();
    }
    return BCG_OK;
}

int bcg_server_result(bcg_server *s, uint64_t id, double *bc_host) {
    clear_error();
    if (!s || !bc_host) return set_error(BCG_ERR_ARG, "null argument");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(BCG_ERR_ARG, "unknown request %llu", (unsigned long long)id);
    Req &r = it->second;
    if (!r.done) return set_error(BCG_ERR_ARG, "request %llu is not finished", (unsigned long long)id);
    CKS(cudaMemcpyAsync(bc_host, r.d_out, r.bytes, cudaMemcpyDeviceToHost, s->stream));
    CKS(cudaFreeAsync(r.d_out, s->stream));
    CKS(cudaStreamSynchronize(s->stream));
    s->admitted -= r.bytes;
    s->reqs.erase(it);
    return BCG_OK;
}

int bcg_server_info(bcg_server *s, uint64_t *resident_bytes, uint64_t *admitted_bytes, uint32_t *pending,
                    uint32_t *running, uint64_t *waves) {
    clear_error();
    if (!s) return set_error(BCG_ERR_ARG, "null handle");
    uint32_t run = 0;
    for (auto &q : s->queue) run += (uint32_t)q.size();
    if (resident_bytes) *resident_bytes = s->resident;
    if (admitted_bytes) *admitted_bytes = s->admitted;
    if (pending) *pending = (uint32_t)s->pending.size();
    if (running) *running = run;
    if (waves) *waves = s->waves;
    return BCG_OK;
}

}  // extern "C"
