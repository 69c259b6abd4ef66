// Serving form: BC requests against a pool of resident graphs, admitted under
// an HBM budget and run with continuous batching (no counterpart in the
// reference, whose program computes one graph per process).
//
// The pool is uploaded once as one disjoint union whose tiles never cross a
// graph boundary, so each graph owns a contiguous range of tiles.  A request
// asks for the BC of one graph over a list of sources (or all of its
// vertices); its result buffer (one double per vertex of the graph) is
// allocated when it is admitted, FIFO, while the pool plus the admitted
// buffers fit the budget.
//
// Waves.  A wave is one persistent launch of packed batches (component-packed:
// the graphs active in the wave share every batch, each graph filling the S
// slots with its own sources).  Each graph takes up to wave_batches * S of
// the not yet scheduled sources of ALL its admitted requests, oldest request
// first, so requests on the same graph share the adjacency passes of a
// batch.  The sweep kernel keeps each slot's dependencies apart and, at the
// end of every batch, adds them into the buffer of the request that owns the
// slot's source (SlotOut routing), one slot after the other: a request's
// sources reach its buffer in its own source order however they are packed,
// and a source's dependencies do not depend on its batch-mates, so its
// result is bitwise the same alone or in any mix.  S is 6 while the active graphs' 64-byte state rows
// fit 64 MB (they then stay in L2), else 3.
//
// Continuity.  bcg_server_step never waits for the GPU: it retires the waves
// that have finished (their requests become done), admits what fits, and
// keeps up to two waves queued on the server's stream, so the next wave is
// planned and enqueued while the current one runs and the device does not
// idle between waves.  Every entry point takes the server's lock, so other
// threads may submit while a wave is on the GPU: such a request is admitted
// at once if its buffer fits and joins the next wave that is planned.
#include <algorithm>
#include <deque>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "bcg_common.hpp"
#include "engine_internal.hpp"

using namespace bcg;

namespace {

struct Req {
    uint32_t graph = 0;
    std::vector<uint32_t> src;  // union ids of the request's non-isolated sources, in order
    size_t sched = 0;           // sources already placed in a wave
    double *d_out = nullptr;    // one accumulator per vertex of the graph (from admission on)
    size_t bytes = 0;
    bool done = false;
};

size_t up16(size_t x) { return (x + 15) & ~size_t(15); }

constexpr int kInFlight = 2;  // waves queued on the stream at once

}  // namespace

// One enqueued wave: its schedule buffers, completion event, error flags and
// the requests whose last source it holds.
struct ServeWave {
    unsigned char *h_blob = nullptr, *d_blob = nullptr;
    RootStat *d_rstat = nullptr;
    int *h_flags = nullptr;  // Ctrl::error, Ctrl::overflow after the wave (pinned)
    cudaEvent_t ev = nullptr;
    bool busy = false;
    std::vector<uint64_t> finishing;
};

struct bcg_server {
    std::mutex mu;
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
    std::vector<std::deque<uint64_t>> queue;  // per graph: admitted requests with unscheduled sources, in order
    std::deque<uint64_t> done;                // finished, not yet reported
    // wave schedule layout (one region per wave slot)
    size_t off_xbeg = 0, off_xroots = 0, off_xslot = 0, off_xpf = 0, off_xpu = 0, off_xtiles = 0, off_xrbeg = 0,
           off_xrange = 0, off_xout = 0, blob_bytes = 0;
    ServeWave slot[kInFlight];
    std::deque<int> inflight;  // wave slots in launch order
    cudaStream_t stream = nullptr, result_stream = nullptr;
    double *d_slot_delta = nullptr;  // width * n per-slot dependencies of a batch
    uint64_t waves = 0;
    int sticky_error = BCG_OK;  // a failed wave leaves the server unusable
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
    return 4 * (n + 5) + 4 * (g->nnz + 4) + 8 * (n + 4) /*vinfo*/ + 8 * n /*bc*/ + (uint64_t)row_bytes((int)S) * n +
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

// Retires the finished waves at the front of the queue (wait: block for the
// oldest one first).
int retire(bcg_server *s, bool wait) {
    while (!s->inflight.empty()) {
        ServeWave &w = s->slot[s->inflight.front()];
        if (wait) {
            CKS(cudaEventSynchronize(w.ev));
            wait = false;
        } else {
            const cudaError_t q = cudaEventQuery(w.ev);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) return set_error(BCG_ERR_CUDA, "wave event: %s", cudaGetErrorString(q));
        }
        if (w.h_flags[1] || w.h_flags[0] == BCG_ERR_OVERFLOW) {
            s->sticky_error = BCG_ERR_OVERFLOW;
            return set_error(BCG_ERR_OVERFLOW, "a shortest-path count exceeded 2^64 in a served wave");
        }
        if (w.h_flags[0]) {
            s->sticky_error = w.h_flags[0];
            return set_error(w.h_flags[0], "device reported error %d in a served wave", w.h_flags[0]);
        }
        for (uint64_t rid : w.finishing) {
            s->reqs[rid].done = true;
            s->done.push_back(rid);
        }
        w.finishing.clear();
        w.busy = false;
        s->inflight.pop_front();
    }
    return BCG_OK;
}

// Plans the next wave from the admitted requests' unscheduled sources and
// enqueues it on the server's stream.  *launched = false when there is no
// work (or no free wave slot).
int enqueue_wave(bcg_server *s, bool *launched) {
    *launched = false;
    int wi = -1;
    for (int i = 0; i < kInFlight; ++i)
        if (!s->slot[i].busy) { wi = i; break; }
    if (wi < 0) return BCG_OK;
    const uint32_t G = s->ngraphs, W = s->wave_batches;
    // the graphs with work, and their active vertices (for the width rule)
    std::vector<uint32_t> act;
    uint64_t act_n = 0;
    for (uint32_t gi = 0; gi < G; ++gi) {
        if (s->queue[gi].empty()) continue;
        act.push_back(gi);
        act_n += s->gn[gi];
    }
    if (act.empty()) return BCG_OK;
    const uint32_t S = (act_n * (uint64_t)row_bytes(6) <= (64ull << 20)) ? 6u : 3u;
    // each active graph's list for this wave: (source, request) pairs, its
    // admitted requests' unscheduled sources oldest request first
    struct Pick { uint32_t v; uint64_t rid; };
    std::vector<std::vector<Pick>> picks(act.size());
    ServeWave &w = s->slot[wi];
    w.finishing.clear();
    uint32_t nb = 0;
    for (size_t a = 0; a < act.size(); ++a) {
        auto &q = s->queue[act[a]];
        const size_t cap = (size_t)W * S;
        while (!q.empty() && picks[a].size() < cap) {
            Req &r = s->reqs[q.front()];
            const size_t take = std::min(cap - picks[a].size(), r.src.size() - r.sched);
            for (size_t j = 0; j < take; ++j) picks[a].push_back(Pick{r.src[r.sched + j], q.front()});
            r.sched += take;
            if (r.sched == r.src.size()) {
                w.finishing.push_back(q.front());
                q.pop_front();
            }
        }
        nb = std::max<uint32_t>(nb, (uint32_t)((picks[a].size() + S - 1) / S));
    }
    // requests with no source left to run (all of degree 0) finish with this wave
    unsigned char *h = w.h_blob;
    auto *xbeg = reinterpret_cast<uint32_t *>(h + s->off_xbeg);
    auto *xroots = reinterpret_cast<uint32_t *>(h + s->off_xroots);
    auto *xslot = h + s->off_xslot;
    auto *xpf = reinterpret_cast<unsigned long long *>(h + s->off_xpf);
    auto *xpu = reinterpret_cast<unsigned long long *>(h + s->off_xpu);
    auto *xtiles = reinterpret_cast<uint32_t *>(h + s->off_xtiles);
    auto *xrbeg = reinterpret_cast<uint32_t *>(h + s->off_xrbeg);
    auto *xrange = reinterpret_cast<uint2 *>(h + s->off_xrange);
    auto *xout = reinterpret_cast<SlotOut *>(h + s->off_xout);
    uint32_t nr = 0, nrange = 0;
    xbeg[0] = 0;
    xrbeg[0] = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        xpf[i] = xpu[i] = 0;
        uint32_t cum = 0;
        // act is in caller-graph order and the union keeps that order, so the
        // batch's ranges ascend by first tile (the kernel searches them)
        for (size_t a = 0; a < act.size(); ++a) {
            const size_t j0 = (size_t)i * S;
            if (j0 >= picks[a].size()) continue;
            const uint32_t gi = act[a];
            SlotOut o{};
            o.base = s->base[gi];
            for (uint32_t k = 0; k < S && j0 + k < picks[a].size(); ++k) {
                const Pick &pk = picks[a][j0 + k];
                xroots[nr] = pk.v;
                xslot[nr] = (unsigned char)k;
                ++nr;
                xpf[i] += s->hdeg[pk.v];
                xpu[i] += s->gnnz[gi] - s->hdeg[pk.v];
                o.out[k] = s->reqs[pk.rid].d_out;
            }
            xout[nrange] = o;
            xrange[nrange++] = make_uint2(s->grange[gi].x, cum);
            cum += s->grange[gi].y - s->grange[gi].x;
        }
        xbeg[i + 1] = nr;
        xrbeg[i + 1] = nrange;
        xtiles[i] = cum;
    }
    if (nb) {
        CKS(cudaMemcpyAsync(w.d_blob, w.h_blob, s->blob_bytes, cudaMemcpyHostToDevice, s->stream));
        unsigned char *d = w.d_blob;
        PackedRun p{};
        p.xbeg = reinterpret_cast<const uint32_t *>(d + s->off_xbeg);
        p.xroots = reinterpret_cast<const uint32_t *>(d + s->off_xroots);
        p.xslot = d + s->off_xslot;
        p.xpf = reinterpret_cast<const unsigned long long *>(d + s->off_xpf);
        p.xpu = reinterpret_cast<const unsigned long long *>(d + s->off_xpu);
        p.xtiles = reinterpret_cast<const uint32_t *>(d + s->off_xtiles);
        p.xrbeg = reinterpret_cast<const uint32_t *>(d + s->off_xrbeg);
        p.xrange = reinterpret_cast<const uint2 *>(d + s->off_xrange);
        p.xout = reinterpret_cast<const SlotOut *>(d + s->off_xout);
        p.slot_delta = s->d_slot_delta;
        p.nbatch = nb;
        p.rstat = w.d_rstat;
        int rc = enqueue_packed(s->g, p, S, s->stream);
        if (rc) return rc;
        // the wave's error flags, read by the host once its event has passed
        CKS(cudaMemcpyAsync(w.h_flags, &s->g->d_ctrl->error, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    } else {
        w.h_flags[0] = w.h_flags[1] = 0;
    }
    CKS(cudaEventRecord(w.ev, s->stream));
    w.busy = true;
    s->inflight.push_back(wi);
    ++s->waves;
    *launched = true;
    return BCG_OK;
}

// The common body of step and wait (lock held).
int step_locked(bcg_server *s, bool wait, uint64_t *done_ids, uint32_t cap, uint32_t *ndone) {
    *ndone = 0;
    if (s->sticky_error) return set_error(s->sticky_error, "an earlier served wave failed (error %d)", s->sticky_error);
    int rc = retire(s, wait && !s->inflight.empty());
    if (rc) return rc;
    rc = admit(s);
    if (rc) return rc;
    while ((int)s->inflight.size() < kInFlight) {
        bool launched = false;
        rc = enqueue_wave(s, &launched);
        if (rc) {
            s->sticky_error = rc;
            return rc;
        }
        if (!launched) break;
    }
    while (!s->done.empty() && *ndone < cap) {
        done_ids[(*ndone)++] = s->done.front();
        s->done.pop_front();
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
    for (uint32_t gi = 1; gi < ngraphs; ++gi)
        if (s->grange[gi].x < s->grange[gi - 1].x)
            return fail(set_error(BCG_ERR_ARG, "the pool union does not keep the graphs in caller order"));
    rc = ensure_state(s->g, s->width);
    if (rc) return fail(rc);
    if (cudaMalloc(&s->d_slot_delta, (size_t)s->width * s->g->n * sizeof(double)) != cudaSuccess)
        return fail(set_error(BCG_ERR_OOM, "per-slot dependency buffer"));
    s->budget = hbm_budget_bytes;
    s->resident = pool_bytes(s->g, s->width) + (uint64_t)s->width * s->g->n * sizeof(double);
    if (s->resident > s->budget)
        return fail(set_error(BCG_ERR_OOM, "the resident pool needs %llu bytes, over the %llu-byte budget",
                              (unsigned long long)s->resident, (unsigned long long)s->budget));
    // wave schedule regions (a wave has at most wave_batches batches, each
    // with every graph active)
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
    s->off_xout = o; o += up16(W * G * sizeof(SlotOut));
    s->blob_bytes = o;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->result_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(set_error(BCG_ERR_CUDA, "server streams: %s", cudaGetErrorString(e)));
    for (int i = 0; i < kInFlight; ++i) {
        ServeWave &w = s->slot[i];
        if ((e = cudaMalloc(&w.d_blob, o)) != cudaSuccess || (e = cudaMallocHost(&w.h_blob, o)) != cudaSuccess ||
            (e = cudaMalloc(&w.d_rstat, W * S * sizeof(RootStat))) != cudaSuccess ||
            (e = cudaMallocHost(&w.h_flags, 2 * sizeof(int))) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&w.ev, cudaEventDisableTiming)) != cudaSuccess)
            return fail(set_error(BCG_ERR_CUDA, "server buffers: %s", cudaGetErrorString(e)));
        s->resident += o + W * S * sizeof(RootStat);
    }
    *out = s;
    return BCG_OK;
}

int bcg_server_destroy(bcg_server *s) {
    clear_error();
    if (!s) return set_error(BCG_ERR_ARG, "null handle");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stream) cudaStreamSynchronize(s->stream);
        if (s->result_stream) cudaStreamSynchronize(s->result_stream);
        for (auto &kv : s->reqs)
            if (kv.second.d_out) cudaFree(kv.second.d_out);
        for (ServeWave &w : s->slot) {
            cudaFree(w.d_blob);
            cudaFree(w.d_rstat);
            if (w.h_blob) cudaFreeHost(w.h_blob);
            if (w.h_flags) cudaFreeHost(w.h_flags);
            if (w.ev) cudaEventDestroy(w.ev);
        }
        if (s->stream) cudaStreamDestroy(s->stream);
        if (s->result_stream) cudaStreamDestroy(s->result_stream);
        cudaFree(s->d_slot_delta);
        if (s->g) bcg_graph_destroy(s->g);
    }
    delete s;
    return BCG_OK;
}

int bcg_server_submit(bcg_server *s, uint32_t graph, const uint32_t *sources, uint64_t nsrc, uint64_t *id) {
    clear_error();
    if (!s || !id) return set_error(BCG_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
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
    std::lock_guard<std::mutex> lock(s->mu);
    return step_locked(s, false, done_ids, cap, ndone);
}

int bcg_server_wait(bcg_server *s, uint64_t *done_ids, uint32_t cap, uint32_t *ndone) {
    clear_error();
    if (!s || !ndone || (cap && !done_ids)) return set_error(BCG_ERR_ARG, "null argument");
    cudaEvent_t ev = nullptr;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (!s->inflight.empty()) ev = s->slot[s->inflight.front()].ev;
    }
    // wait without the lock, so other threads can submit meanwhile (the
    // event stays valid: only this server's own waves re-record it)
    if (ev) {
        const cudaError_t e = cudaEventSynchronize(ev);
        if (e != cudaSuccess) return set_error(BCG_ERR_CUDA, "waiting for a wave: %s", cudaGetErrorString(e));
    }
    std::lock_guard<std::mutex> lock(s->mu);
    return step_locked(s, false, done_ids, cap, ndone);
}

int bcg_server_result(bcg_server *s, uint64_t id, double *bc_host) {
    clear_error();
    if (!s || !bc_host) return set_error(BCG_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(BCG_ERR_ARG, "unknown request %llu", (unsigned long long)id);
    Req &r = it->second;
    if (!r.done) return set_error(BCG_ERR_ARG, "request %llu is not finished", (unsigned long long)id);
    // the last wave that wrote the buffer has completed: copy on the result
    // stream, so later waves queued on the server's stream keep running
    CKS(cudaMemcpyAsync(bc_host, r.d_out, r.bytes, cudaMemcpyDeviceToHost, s->result_stream));
    CKS(cudaFreeAsync(r.d_out, s->result_stream));
    CKS(cudaStreamSynchronize(s->result_stream));
    s->admitted -= r.bytes;
    s->reqs.erase(it);
    return BCG_OK;
}

int bcg_server_info(bcg_server *s, uint64_t *resident_bytes, uint64_t *admitted_bytes, uint32_t *pending,
                    uint32_t *running, uint64_t *waves) {
    clear_error();
    if (!s) return set_error(BCG_ERR_ARG, "null handle");
    std::lock_guard<std::mutex> lock(s->mu);
    uint32_t run = 0;
    for (auto &kv : s->reqs)
        if (kv.second.d_out && !kv.second.done) ++run;
    if (resident_bytes) *resident_bytes = s->resident;
    if (admitted_bytes) *admitted_bytes = s->admitted;
    if (pending) *pending = (uint32_t)s->pending.size();
    if (running) *running = run;
    if (waves) *waves = s->waves;
    return BCG_OK;
}

}  // extern "C"
