/*
 * bcg.h — C ABI of the B200 Brandes betweenness-centrality engine (libbcg.so).
 *
 * The engine replaces the single-GPU BC path of ck-bc's program/bc-cuda:
 * the per-source driver loop of bc2d.c (bc2d.c:1016-1050, bc_func_mono
 * bc2d.c:504-580) and the device state + kernels behind the bc2d.h C ABI
 * (bc2d.h:132-184, implemented in cuda_kernels.cu).  The reference keeps its
 * device state in file-static globals and exits on every error
 * (cudamacro.h:1-16); this ABI is handle based, re-entrant per handle and
 * returns a status code from every call.  The reference's own mono-path
 * symbols (initcuda, setcuda, scan_col_csc_cuda_mono, ...) are exported by the
 * compatibility library described in include/bc2d_compat.h.
 *
 * Conventions
 *   - Graphs are undirected, unweighted, stored as uint32 CSR: offsets[n+1],
 *     adj[offsets[n]] (the reference's LOCINT = uint32_t CSC, bc2d.h:14,
 *     build_csc bc2d.c:472-501; for a symmetric graph CSR == CSC).
 *   - bc values are FP64 sums over ORDERED (source, target) pairs for the
 *     given source set, i.e. the reference's bc[] before the "/2" it applies
 *     when writing the result file (bc2d.c:1065).
 *   - Every function returns BCG_OK (0) or a negative BCG_ERR_* code;
 *     bcg_last_error() gives a message for the calling thread.
 */
#ifndef BCG_H_
#define BCG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BCG_OK               0
#define BCG_ERR_ARG         -1  /* invalid argument (null pointer, id >= n, ...) */
#define BCG_ERR_CUDA        -2  /* a CUDA runtime call failed */
#define BCG_ERR_OOM         -3  /* device or host allocation failed / over budget */
#define BCG_ERR_OVERFLOW    -4  /* a shortest-path count exceeded uint64 */
#define BCG_ERR_TIMEOUT     -5  /* a device-side bounded wait gave up */
#define BCG_ERR_IO          -6  /* file could not be opened / parsed */
#define BCG_ERR_DEPTH       -7  /* BFS deeper than the engine's level limit */
#define BCG_ERR_RANGE       -8  /* graph too large for 32-bit ids/offsets */
#define BCG_ERR_NOGPU       -9  /* no CUDA device or kernel image for it */

/* flags for bcg_graph_create */
#define BCG_PRUNE_DEGREE1   0x1u  /* fold degree-1 vertices into their neighbour (bc2d -H 1):
                                     one round of BCG_PRUNE_TREES' peeling.  Not available with
                                     bcg_single_source, bcg_graph_set_reach, bcg_run_weighted,
                                     bcg_run_root_levels, bcg_run_slots. */
#define BCG_DIRECTED        0x2u  /* adjacency is not symmetric (bc2d -U): traversal follows
                                     adj[] only; pruning is ignored */
#define BCG_PRUNE_TREES     0x4u  /* fold whole pendant trees (iterated degree-1 removal), not
                                     just one layer as degree_reduction does (bc2d.c:314-419);
                                     the trees' betweenness is computed in closed form.  Takes
                                     precedence over BCG_PRUNE_DEGREE1.  Not available with
                                     the calls BCG_PRUNE_DEGREE1 lists. */

/* ---------------------------------------------------------------------------
 * Host-side graph ingest and generation (host code, no GPU needed).
 * ------------------------------------------------------------------------ */

/* Host CSR owned by the library; release with bcg_csr_free. */
typedef struct bcg_host_csr {
    uint32_t  n;        /* vertices */
    uint64_t  nnz;      /* directed adjacency entries = 2 * undirected edges */
    uint32_t *offsets;  /* n + 1 */
    uint32_t *adj;      /* nnz, each list sorted ascending, no loops, no duplicates */
} bcg_host_csr;

/* Reads the reference's edge-list text format (read_graph bc2d.c:175-254):
 * one "u v" pair per line, 0-based ids < n; any line containing '#' is a
 * comment ("# Nodes: X Edges: Y" is echoed to stdout when echo_header != 0).
 * undirected != 0 mirrors every non-loop edge (mirror bc2d.c:152-170, the
 * default; bc2d -U clears it).  Duplicates and self-loops are dropped
 * (norm_graph bc2d.c:430-453).  An id >= n fails with BCG_ERR_IO and a message
 * naming the line, like bc2d.c:232-237. */
int bcg_csr_read_edgelist(const char *path, uint64_t n, int undirected,
                          int echo_header, bcg_host_csr *out);

/* Builds a CSR from an explicit edge array (pairs[2*i], pairs[2*i+1]);
 * same normalisation as bcg_csr_read_edgelist. */
int bcg_csr_from_pairs(const uint64_t *pairs, uint64_t npairs, uint64_t n,
                       int undirected, bcg_host_csr *out);

/* Seeded synthetic graphs.  spec is "kind:key=value,..." with kind one of
 *   rmat  scale, ef, a, b, c, seed [, pendant_frac, pendant_mean, pendant_seed]
 *   er    scale, ef, seed            (G(n, M) with M = ef * 2^scale draws)
 *   grid  w, h, drop, seed           (4-neighbour grid, each edge dropped with
 *                                     probability drop, largest component kept)
 * The generators and their PRNG (splitmix64) are documented in graph.cpp. */
int bcg_csr_generate(const char *spec, bcg_host_csr *out);

/* Writes a CSR back as the reference's edge-list text (each undirected edge
 * once, u < v, with a "# Nodes: N Edges: E" header). */
int bcg_csr_write_edgelist(const char *path, const bcg_host_csr *g);

/* Binary CSR cache (fast ingest; no counterpart in the reference, which
 * parses the text file on every run, bc2d.c:214-247): "BCGCSR01", n, nnz
 * and a checksum, then offsets[n+1] and adj[nnz] as uint32.  Reading checks
 * the checksum and the CSR invariants (BCG_ERR_IO when they fail). */
int bcg_csr_write_binary(const char *path, const bcg_host_csr *g);
int bcg_csr_read_binary(const char *path, bcg_host_csr *out);

void bcg_csr_free(bcg_host_csr *g);

/* k distinct vertices drawn uniformly from [0, n) with the given seed
 * (partial Fisher-Yates over splitmix64). */
int bcg_sample_sources(uint32_t n, uint64_t k, uint64_t seed, uint32_t *out);

/* ---------------------------------------------------------------------------
 * Device engine.
 * ------------------------------------------------------------------------ */

typedef struct bcg_graph bcg_graph;   /* opaque: one graph resident in HBM */

/* Per-run statistics (all sources of one bcg_run call). */
typedef struct bcg_stats {
    uint64_t sources;        /* sources requested */
    uint64_t skipped;        /* sources with degree 0 (bc2d.c:1026-1034) */
    uint64_t roots;          /* BFS roots actually run (after pendant folding) */
    uint64_t batches;        /* multi-source batches launched */
    uint64_t teps_edges;     /* sum over sources of undirected edges in the
                                source's connected component (input graph) */
    uint64_t visited;        /* sum over roots of vertices reached (pruned graph) */
    uint64_t comp_vertices;  /* sum over sources of the vertex count of the
                                source's connected component (input graph) */
    uint32_t max_depth;      /* deepest BFS level seen */
    uint32_t batch_width;    /* sources per batch (S) */
    double   kernel_ms;      /* device time of the BC kernels (CUDA events) */
    uint32_t extended_sigma; /* 1: path counts ran as extended-range numbers */
    uint32_t reserved;
    uint64_t search_edges;   /* sum over roots of the undirected edges the search
                                holds in the root's component (the pruned graph's
                                edges: the work the sweeps actually read) */
    uint64_t launches;       /* kernels of this library the call launched */
} bcg_stats;

/* Number of CUDA devices visible (0 when none); never fails. */
int bcg_device_count(void);

/* Uploads a host CSR to the current device and prepares it (pendant
 * pruning on the device when a pruning flag is set, work tiles).  offsets/adj are only
 * read during the call.  Replaces initcuda (cuda_kernels.cu:1123-1198) +
 * init_bc_1degree/init_bc_1degree_device (bc2d.c:455-465,
 * cuda_kernels.cu:1083-1087) + degree_reduction (bc2d.c:314-419). */
int bcg_graph_create(const uint32_t *offsets, const uint32_t *adj, uint32_t n,
                     uint64_t nnz, uint32_t flags, bcg_graph **out);

/* Same, with offsets/adj already in device memory (copied, not retained). */
int bcg_graph_create_device(const uint32_t *d_offsets, const uint32_t *d_adj,
                            uint32_t n, uint64_t nnz, uint32_t flags,
                            bcg_graph **out);

/* Frees every device buffer of the graph (fincuda cuda_kernels.cu:1201-1232)
 * after the device has finished all queued work.  Graph buffers come from a
 * stream-ordered memory pool of the library (one per device) that keeps up
 * to 1 GiB reserved once freed, so the next creation reuses the memory. */
int bcg_graph_destroy(bcg_graph *g);

/* Sets every bc value of the graph to 0. */
int bcg_reset_bc(bcg_graph *g);

/* Runs Brandes from every source in sources[0..nsrc) (host array) and ADDS
 * each source's dependencies into the graph's device bc[] accumulator.
 * Sources with degree 0 are skipped and counted (bc2d.c:1026-1034).
 * Replaces the per-source loop bc2d.c:1016-1050 with setcuda/set_mlp_cuda/
 * scan_col_csc_cuda_mono/scan_frt_csc_cuda_mono/pre_update_bc_cuda/
 * update_bc_cuda (cuda_kernels.cu:263-336, 689-703, 766-918, 1100-1119). */
int bcg_run(bcg_graph *g, const uint32_t *sources, uint64_t nsrc,
            bcg_stats *stats);

/* Same with a device-resident source array; stream is a cudaStream_t (NULL =
 * legacy default stream).  The source list is read back to the host on that
 * stream (a stream synchronisation) to fold pendant sources into their
 * anchors; the BC kernel is then launched on the stream and the call returns
 * without waiting for it unless stats != NULL. */
int bcg_run_device(bcg_graph *g, const uint32_t *d_sources, uint64_t nsrc,
                   void *stream, bcg_stats *stats);

/* Copies the FP64 bc accumulator (n values) to host memory
 * (get_bc cuda_kernels.cu:1039-1041, which copies float). */
int bcg_get_bc(bcg_graph *g, double *bc_host);

/* Device pointer of the bc accumulator (n doubles), valid until destroy. */
int bcg_bc_device_ptr(bcg_graph *g, double **d_bc);

/* One-shot drop-in call on host buffers: upload, run all sources, copy bc
 * back (bc_out[n], overwritten), free.  flags as bcg_graph_create. */
int bcg_bc_csr(const uint32_t *offsets, const uint32_t *adj, uint32_t n,
               uint64_t nnz, const uint32_t *sources, uint64_t nsrc,
               uint32_t flags, double *bc_out, bcg_stats *stats);

/* Single-source detail for parity checks: BFS depth (-1 = unreachable),
 * shortest-path count sigma and dependency delta (delta_s(v) =
 * sum over w with d(w)=d(v)+1 of sigma_v/sigma_w * (1 + delta_w)) of every
 * vertex, for source src on the graph as created (BCG_ERR_ARG on a graph
 * created with a pruning flag: bcg_debug_batch reads pruned graphs).  Any
 * output pointer may be NULL.  Does not touch the bc accumulator. */
int bcg_single_source(bcg_graph *g, uint32_t src, int32_t *level,
                      uint64_t *sigma, double *delta);

/* Debug read-out of one real batch: runs the roots[0..nroots) (caller's ids,
 * nroots <= width) as one batch of the given width (1, 3 or 6: the S of the
 * sweep kernel's state rows) with root k in slot k, and copies out for every
 * slot k and vertex v, at [k * n + v] in the caller's numbering, the BFS
 * depth (-1 = unreachable), sigma, and delta.  The per-source state the
 * reference keeps in lvl/sig/delta (setcuda + set_mlp_cuda + scan_col_mono2
 * + scan_frt_mono, cuda_kernels.cu:471-599, 689-703, 1100-1119) for `width`
 * sources at once.  Works in every pruning mode: on a pruned graph the
 * roots must be kept vertices with a kept edge (BCG_ERR_ARG otherwise) and
 * folded vertices read -1 / 0 / 0.  Exact uint64 counts (overflow is
 * BCG_ERR_OVERFLOW).  Does not touch the bc accumulator.  Any output may be
 * NULL. */
int bcg_debug_batch(bcg_graph *g, uint32_t width, const uint32_t *roots, uint32_t nroots,
                    int32_t *level, uint64_t *sigma, double *delta);

/* Pruning result of a graph created with a pruning flag: anchor[v] = the
 * kept vertex v was folded into, or v itself when v was kept; reach[v] =
 * number of vertices folded into v (0 for folded vertices).  An unpruned
 * graph reads anchor[v] = v, reach[v] = 0.  Either pointer may be NULL. */
int bcg_graph_pruning(bcg_graph *g, uint32_t *anchor, uint32_t *reach);

/* Graph sizes after preparation. */
int bcg_graph_info(bcg_graph *g, uint32_t *n, uint64_t *nnz,
                   uint64_t *nnz_pruned, uint32_t *pruned_vertices);

/* Sets per-vertex pendant weights computed by the caller (the reference's
 * reach[] from its host-side degree_reduction, bc2d.c:314-419 + 455-465,
 * handed over by init_bc_1degree_device, cuda_kernels.cu:1083-1087).  Only
 * for graphs created without a pruning flag. */
int bcg_graph_set_reach(bcg_graph *g, const uint32_t *reach);

/* Runs explicit BFS roots with explicit weights: root k's dependencies are
 * added mult[k] times and bc[root] += pend[k] * (W - 2), W = sum over the
 * root's component of (1 + reach) (update_bc cuda_kernels.cu:263-277 with
 * reach_v0: mult = reach_v0 + 1, pend = reach_v0).  No degree-0 skip and no
 * pendant folding.  pend may be NULL (all 0). */
int bcg_run_weighted(bcg_graph *g, const uint32_t *roots, const double *mult,
                     const uint32_t *pend, uint64_t nroots, bcg_stats *stats);

/* bcg_run_weighted for one root (mult, pend as there) that also writes the
 * root's BFS depths level[n] (-1 = unreachable) in the same search: the
 * per-source state the reference's driver reads back between its kernel
 * calls (get_msk and pre_update_bc_cuda after scan_col_csc_cuda_mono,
 * bc2d.c:504-580).  stats may be NULL.  Only for graphs created without a
 * pruning flag. */
int bcg_run_root_levels(bcg_graph *g, uint32_t root, double mult, uint32_t pend, int32_t *level,
                        bcg_stats *stats);

/* Searches the nroots roots in batches of `width` (1, 3 or 6) in one launch
 * of the sweep kernel without adding anything to bc: root k's dependencies
 * (delta of every vertex, root included; 0 where not reached) go to the
 * device array d_delta[k * n .. k * n + n), its depths (-1 = not reached) to
 * the host array level[k * n ..] (may be NULL), the vertices it reached to
 * visited[k] and the sum of (1 + reach) over them to wsum[k] (both may be
 * NULL).  d_delta holds ceil(nroots / width) * width * n doubles.  Lets a
 * caller that learns its sources one at a time (the reference driver's
 * per-source loop, bc2d.c:1016-1050) search several ahead and commit each
 * with bcg_add_scaled once it is asked for.  Only for graphs created
 * without a pruning flag. */
int bcg_run_slots(bcg_graph *g, uint32_t width, const uint32_t *roots, uint32_t nroots, double *d_delta,
                  int32_t *level, uint64_t *visited, uint64_t *wsum);

/* Commits count (<= 64) searched roots into bc, in the order given: for root
 * j, bc[v] += mult[j] * d_delta[slot[j] * n + v] for every v != root[j], and
 * bc[root[j]] += root_add[j] (the root's weighted dependencies and its
 * pendant source term, update_bc, cuda_kernels.cu:263-277).  slot, mult,
 * root and root_add are host arrays; one kernel, queued on the default
 * stream. */
int bcg_add_scaled(bcg_graph *g, const double *d_delta, uint32_t count, const uint32_t *slot, const double *mult,
                   const uint32_t *root, const double *root_add);

/* Forces the sources-per-batch width (1, 3 or 6; 0 = automatic). */
int bcg_set_batch_width(bcg_graph *g, uint32_t width);

/* How shortest-path counts (sigma) are held.  BCG_SIGMA_AUTO (default):
 * exact uint64; a run in which a count exceeds 2^64 is redone with
 * extended-range numbers (16-bit exponent, 49-bit significand, rounded to
 * nearest: about 2^-49 relative error per add) after restoring the
 * accumulators, and bcg_stats.extended_sigma reports it.  BCG_SIGMA_EXACT:
 * overflow fails with BCG_ERR_OVERFLOW (the reference's uint32 counts wrap
 * silently, bc2d.h:14).  BCG_SIGMA_EXTENDED: always extended.  Graphs such
 * as large grids need it: their path counts reach 2^4000. */
#define BCG_SIGMA_AUTO      0
#define BCG_SIGMA_EXACT     1
#define BCG_SIGMA_EXTENDED  2
int bcg_set_sigma_mode(bcg_graph *g, int mode);

/* bcg_single_source in extended mode: sigma_ext[v] is v's path count in the
 * extended encoding (0 = unreachable or 0; otherwise bits 63..48 hold E,
 * bits 47..0 f, value (2^48 + f) * 2^(E - 32816)). */
int bcg_single_source_ext(bcg_graph *g, uint32_t src, int32_t *level, uint64_t *sigma_ext, double *delta);

/* ---------------------------------------------------------------------------
 * Batched form: exact all-sources BC of many independent graphs in one
 * persistent launch.  The reference runs one graph per process (bc2d.c main);
 * per graph the result is what bcg_run over all of its vertices gives.
 * ------------------------------------------------------------------------ */

typedef struct bcg_batch bcg_batch;   /* opaque: a set of graphs resident in HBM */

/* Uploads ngraphs host CSR graphs (offsets[i][n[i] + 1], adj[i], undirected,
 * lists as bcg_graph_create expects) as one disjoint union and builds the
 * packed source schedule (every non-isolated vertex of every graph). */
int bcg_batch_create(uint32_t ngraphs, const uint32_t *const *offsets,
                     const uint32_t *const *adj, const uint32_t *n, bcg_batch **out);
int bcg_batch_destroy(bcg_batch *b);

/* Adds every graph's all-sources BC (ordered-pair sums) into its
 * accumulator.  The first call captures the launch into a CUDA graph that
 * later calls replay (bcg_batch_info reports whether the capture was made).
 * stats: totals over all graphs; kernel_ms is the launch's device time. */
int bcg_batch_run(bcg_batch *b, bcg_stats *stats);
int bcg_batch_reset_bc(bcg_batch *b);
/* Graph `graph`'s bc (n[graph] doubles, the creation order's numbering). */
int bcg_batch_get_bc(bcg_batch *b, uint32_t graph, double *bc_host);

/* Times the first sample_batches batches (0: 4) of the schedule for each
 * batch width in {1, 3, 6} and each tile shape in {32x512, 32x256, 32x128,
 * 16x128, 16x64} (vertices x adjacency entries per tile), keeps the fastest per
 * root and resets the accumulators.  Any output pointer may be NULL. */
int bcg_batch_autotune(bcg_batch *b, uint32_t sample_batches, uint32_t *width,
                       uint32_t *tile_vertices, uint32_t *tile_entries);
/* Schedule length (packed batches), width, tile shape, and whether runs
 * replay a captured CUDA graph (1) or launch directly (0). */
int bcg_batch_info(bcg_batch *b, uint32_t *nbatch, uint32_t *width, uint32_t *tile_vertices,
                   uint32_t *tile_entries, int *captured);

/* ---------------------------------------------------------------------------
 * Serving form: BC requests against a pool of resident graphs, admitted
 * under an HBM budget and run with continuous batching.  The reference
 * answers one query per process run (bc2d.c main); per request the result is
 * what bcg_run over the request's sources gives on that graph.
 * ------------------------------------------------------------------------ */

typedef struct bcg_server bcg_server;  /* opaque: a resident pool and its requests */

/* Uploads the pool (as bcg_batch_create) and sizes the wave schedule:
 * wave_batches = batches of S sources each graph may advance per wave
 * (1..65535).  Fails with BCG_ERR_OOM when the pool alone exceeds
 * hbm_budget_bytes. */
int bcg_server_create(uint32_t ngraphs, const uint32_t *const *offsets,
                      const uint32_t *const *adj, const uint32_t *n,
                      uint64_t hbm_budget_bytes, uint32_t wave_batches, bcg_server **out);
int bcg_server_destroy(bcg_server *s);
/* Queues a request: BC of graph `graph` over sources[nsrc] (nsrc == 0: every
 * vertex of the graph, i.e. exact BC).  Sources of degree 0 are skipped, as
 * in bcg_run.  Its result buffer (8 bytes per vertex of the graph) is
 * allocated when the request is admitted, first come first served, while the
 * pool plus admitted buffers fit the budget.  Every bcg_server_* call takes
 * the server's lock: submit may be called from any thread, also while a wave
 * is on the GPU (the request joins the next wave planned). */
int bcg_server_submit(bcg_server *s, uint32_t graph, const uint32_t *sources, uint64_t nsrc,
                      uint64_t *id);
/* Never waits for the GPU: retires the waves that have finished (their
 * completed requests become done), admits what fits, and keeps up to two
 * waves queued (a wave: every graph with admitted requests runs up to
 * wave_batches * S of their unscheduled sources, oldest request first, all
 * graphs in one packed launch), then reports up to cap finished request ids.
 * A request's result is bitwise the same alone or in any mix. */
int bcg_server_step(bcg_server *s, uint64_t *done_ids, uint32_t cap, uint32_t *ndone);
/* bcg_server_step after waiting (without holding the lock) for the oldest
 * wave in flight, if any. */
int bcg_server_wait(bcg_server *s, uint64_t *done_ids, uint32_t cap, uint32_t *ndone);
/* Copies a finished request's bc (ordered-pair sums, n doubles of its
 * graph) and releases its buffer and the request. */
int bcg_server_result(bcg_server *s, uint64_t id, double *bc_host);
/* Pool bytes, admitted buffer bytes, requests waiting for admission,
 * admitted unfinished requests, waves run so far.  Outputs may be NULL. */
int bcg_server_info(bcg_server *s, uint64_t *resident_bytes, uint64_t *admitted_bytes,
                    uint32_t *pending, uint32_t *running, uint64_t *waves);

/* ---------------------------------------------------------------------------
 * No-allocation entry point.  No counterpart in the reference: its
 * cuda_kernels.cu allocates all device state in initcuda (cuda_kernels.cu:
 * 1123-1198).  For callers that must not allocate device memory themselves
 * or through a library: a framework whose own allocator owns the GPU's
 * memory, or a latency-bound loop where cudaMalloc/cudaFree would
 * synchronise the device.
 * ------------------------------------------------------------------------ */

#define BCG_NOALLOC_MAX_VERTICES 65536u    /* n */
#define BCG_NOALLOC_MAX_ADJ      1048576u  /* nnz: adjacency entries (2 x undirected edges) */
#define BCG_NOALLOC_MAX_SOURCES  65536u    /* sources per call */

/* Exact BC of an undirected device-resident CSR (d_offsets[n+1], d_adj[nnz],
 * lists as bcg_graph_create expects; no pruning) for the device-resident
 * source list d_sources[nsrc] (degree-0 sources skipped, as bcg_run does),
 * written into the caller's device buffer d_bc[n] (ordered-pair sums like
 * bcg_get_bc): overwritten, or added to when accumulate != 0.  Work is
 * enqueued on `stream` (a cudaStream_t, NULL = default stream).
 *   - Synchronous: the call reads a status block back to the host and waits
 *     for the stream before it returns, so it cannot be made while the
 *     stream (or the device) is being captured into a CUDA graph.
 *   - Allocates no device memory and calls no allocating CUDA or library
 *     function: all scratch lives in one fixed static device array of about
 *     19 MiB per device, so n, nnz and nsrc are limited to the
 *     BCG_NOALLOC_MAX_* values above; larger inputs return BCG_ERR_RANGE.
 *   - Path counts are exact uint64; when one overflows (graphs such as
 *     large grids) the sweep is redone with extended-range counts from a
 *     copy of d_bc saved before it, as bcg_run does with BCG_SIGMA_AUTO, so
 *     d_bc is never left with a partial run in it.
 *   - The first call on each device (made with that device current) does the
 *     setup: it takes the array's address with cudaGetSymbolAddress, which
 *     loads the module.
 *   - One scratch per device: calls that overlap on the same device (other
 *     threads or streams) race and must be serialised by the caller.
 *   - Invalid CSR or source ids are found on the device before the sweep
 *     runs and return BCG_ERR_ARG. */
int bcg_bc_noalloc(const uint32_t *d_offsets, const uint32_t *d_adj, uint32_t n, uint64_t nnz,
                   const uint32_t *d_sources, uint64_t nsrc, double *d_bc, int accumulate,
                   void *stream);

/* Message for the last error of the calling thread ("" if none). */
const char *bcg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* BCG_H_ */
