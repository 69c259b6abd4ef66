/*
 * ORACLE — test infrastructure only.  Serial FP64 Brandes betweenness
 * centrality on an undirected CSR graph, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline / reference arm as
 * the checker and the CPU baseline.  It is never linked into, loaded by or
 * called from the product library (ck-bc_b200/libbcg.so).
 *
 * It restates the algorithm of ck-bc program/bc-cuda on the CPU, one source
 * at a time, in the reference's own order of operations:
 *   source loop        bc2d.c:1016-1036   sources given by the caller; a
 *                                          source of degree 0 is skipped and
 *                                          counted (bc2d.c:1026-1034)
 *   forward level      scan_col_mono2      cuda_kernels.cu:471-541
 *                        level[r] = level(c) + 1 for undiscovered r,
 *                        sigma[r] += sigma[c] for every edge c -> r with
 *                        level[r] == level(c) + 1 (cuda_kernels.cu:533-537)
 *   backward level     scan_frt_mono       cuda_kernels.cu:546-599
 *                        for depth = maxlevel-1 .. 1 and every edge c -> r
 *                        with level[r] == depth + 1:
 *                        delta[c] += (delta[r] + 1) / sigma[r] * sigma[c]
 *                        (cuda_kernels.cu:590-595)
 *   bc update          update_bc           cuda_kernels.cu:263-277
 *                        bc[v] += delta[v] for every v != source
 *   output             bc2d.c:1057-1068    the caller prints bc/2
 * Differences from the reference, each deliberate (the oracle computes the
 * definition of Brandes BC):
 *   - sigma is uint64 with overflow detection (reference: uint32 that wraps,
 *     bc2d.h:14, cuda_kernels.cu:536);
 *   - delta and bc are FP64 (reference: float32 with atomic adds,
 *     cuda_kernels.cu:65,69,595);
 *   - no MAX_LVL=1000 depth cap (bc2d.h:25);
 *   - the level-0 source also gets its delta computed (it is not added to bc).
 * The degree-1 pruning of the reference (-H 1) is an optimisation of the same
 * quantity; the oracle always runs on the unpruned graph, so it is the
 * definition against which the pruned GPU path is checked.
 */
#include <math.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

/* BFS + dependency accumulation for one source.  Work arrays are caller
 * provided (n each).  Returns the number of visited vertices; sets *overflow
 * when a sigma sum wrapped. */
static uint64_t brandes_one(uint32_t n, const uint32_t *offs, const uint32_t *adj, uint32_t s,
                            int32_t *lvl, uint64_t *sigma, double *delta, uint32_t *queue,
                            uint32_t *lvl_start, int *overflow, uint32_t *depth_out) {
    for (uint32_t v = 0; v < n; ++v) { lvl[v] = -1; sigma[v] = 0; delta[v] = 0.0; }
    uint32_t head = 0, tail = 0, nlev = 0;
    lvl[s] = 0;
    sigma[s] = 1;
    queue[tail++] = s;
    lvl_start[0] = 0;
    /* forward: one BFS level at a time (the reference's host-driven loop,
     * bc2d.c:535-542) */
    while (head < tail) {
        uint32_t level_end = tail;
        int32_t d = lvl[queue[head]];
        lvl_start[++nlev] = level_end;
        for (; head < level_end; ++head) {
            uint32_t c = queue[head];
            for (uint32_t e = offs[c]; e < offs[c + 1]; ++e) {
                uint32_t r = adj[e];
                if (lvl[r] == -1) { lvl[r] = d + 1; queue[tail++] = r; }
                if (lvl[r] == d + 1) {
                    uint64_t t = sigma[r] + sigma[c];
                    if (t < sigma[r]) *overflow = 1;
                    sigma[r] = t;
                }
            }
        }
    }
    /* nlev levels: level k occupies queue[lvl_start[k] .. lvl_start[k+1]) */
    /* backward: depth = nlev-2 .. 0 (the reference stops at 1; level 0 is
     * computed here too but never added to bc) */
    for (int64_t depth = (int64_t)nlev - 2; depth >= 0; --depth) {
        for (uint32_t i = lvl_start[depth]; i < lvl_start[depth + 1]; ++i) {
            uint32_t c = queue[i];
            double sc = (double)sigma[c];
            double acc = delta[c];
            for (uint32_t e = offs[c]; e < offs[c + 1]; ++e) {
                uint32_t r = adj[e];
                if (lvl[r] == (int32_t)depth + 1)
                    acc += (delta[r] + 1.0) / (double)sigma[r] * sc;
            }
            delta[c] = acc;
        }
    }
    if (depth_out) *depth_out = nlev ? nlev - 1 : 0;
    return tail;
}

int oracle_single_source(uint32_t n, const uint32_t *offs, const uint32_t *adj, uint32_t src,
                         int32_t *level, uint64_t *sigma, double *delta, int *overflow) {
    if (src >= n) return -1;
    uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    uint32_t *ls = (uint32_t *)malloc(((size_t)n + 2) * sizeof(uint32_t));
    int32_t *l = level ? level : (int32_t *)malloc((size_t)n * sizeof(int32_t));
    uint64_t *sg = sigma ? sigma : (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    double *dl = delta ? delta : (double *)malloc((size_t)n * sizeof(double));
    int ov = 0;
    int rc = (queue && ls && l && sg && dl) ? 0 : -2;
    if (!rc) brandes_one(n, offs, adj, src, l, sg, dl, queue, ls, &ov, NULL);
    if (overflow) *overflow = ov;
    free(queue); free(ls);
    if (!level) free(l);
    if (!sigma) free(sg);
    if (!delta) free(dl);
    return rc;
}

int oracle_bc(uint32_t n, const uint32_t *offs, const uint32_t *adj, const uint32_t *sources,
              uint64_t nsrc, int nthreads, double *bc, oracle_stats *st) {
    int nt = nthreads > 0 ? nthreads : 1;
#ifndef _OPENMP
    nt = 1;
#endif
    double *part = (double *)calloc((size_t)nt * n, sizeof(double));
    if (!part) return -2;
    uint64_t skipped = 0, visited = 0, teps_edges = 0, ran = 0;
    uint32_t maxdepth = 0;
    int overflow = 0, err = 0;
#pragma omp parallel num_threads(nt) reduction(+ : skipped, visited, teps_edges, ran) \
    reduction(max : maxdepth) reduction(| : overflow, err)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int32_t *lvl = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        uint64_t *sigma = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
        double *delta = (double *)malloc((size_t)n * sizeof(double));
        uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        uint32_t *ls = (uint32_t *)malloc(((size_t)n + 2) * sizeof(uint32_t));
        double *mine = part + (size_t)tid * n;
        if (!lvl || !sigma || !delta || !queue || !ls) err = 1;
#pragma omp for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)nsrc; ++i) {
            if (err) continue;
            uint32_t s = sources[i];
            if (s >= n) { err = 1; continue; }
            if (offs[s + 1] == offs[s]) { skipped++; continue; }
            int ov = 0;
            uint32_t depth = 0;
            uint64_t nv = brandes_one(n, offs, adj, s, lvl, sigma, delta, queue, ls, &ov, &depth);
            overflow |= ov;
            uint64_t degsum = 0;
            for (uint64_t q = 0; q < nv; ++q) {
                uint32_t v = queue[q];
                degsum += offs[v + 1] - offs[v];
                if (v != s) mine[v] += delta[v];
            }
            visited += nv;
            teps_edges += degsum / 2;
            ran++;
            if (depth > maxdepth) maxdepth = depth;
        }
        free(lvl); free(sigma); free(delta); free(queue); free(ls);
    }
    /* thread partials summed in thread order */
    for (uint32_t v = 0; v < n; ++v) {
        double acc = 0.0;
        for (int t = 0; t < nt; ++t) acc += part[(size_t)t * n + v];
        bc[v] += acc;
    }
    free(part);
    if (st) {
        st->skipped = skipped;
        st->ran = ran;
        st->visited = visited;
        st->teps_edges = teps_edges;
        st->max_depth = maxdepth;
        st->overflow = overflow;
    }
    return err ? -1 : 0;
}

/* Sum over the given sources (degree 0 skipped) and every vertex t != s
 * reachable from s of (d(s,t) - 1).  Brandes' dependencies satisfy
 * sum_v delta_s(v) = sum_t (d(s,t) - 1) (each shortest s-t path has d - 1
 * interior vertices and the pair's weights sum to one per interior position),
 * so this is the exact total of bc[] over a source set: a size-independent
 * check that needs only a BFS per source. */
int oracle_path_length_sum(uint32_t n, const uint32_t *offs, const uint32_t *adj, const uint32_t *sources,
                           uint64_t nsrc, int nthreads, uint64_t *total) {
    int nt = nthreads > 0 ? nthreads : 1;
#ifndef _OPENMP
    nt = 1;
#endif
    uint64_t sum = 0;
    int err = 0;
#pragma omp parallel num_threads(nt) reduction(+ : sum) reduction(| : err)
    {
        int32_t *lvl = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        if (!lvl || !queue) err = 1;
#pragma omp for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)nsrc; ++i) {
            if (err) continue;
            uint32_t s = sources[i];
            if (s >= n) { err = 1; continue; }
            if (offs[s + 1] == offs[s]) continue;
            for (uint32_t v = 0; v < n; ++v) lvl[v] = -1;
            uint32_t head = 0, tail = 0;
            lvl[s] = 0;
            queue[tail++] = s;
            while (head < tail) {
                uint32_t c = queue[head++];
                for (uint32_t e = offs[c]; e < offs[c + 1]; ++e) {
                    uint32_t r = adj[e];
                    if (lvl[r] == -1) {
                        lvl[r] = lvl[c] + 1;
                        queue[tail++] = r;
                        sum += (uint64_t)lvl[r] - 1;
                    }
                }
            }
        }
        free(lvl); free(queue);
    }
    if (total) *total = sum;
    return err ? -1 : 0;
}

/* The same algorithm with sigma and delta held as __float128 (113-bit
 * significand, exponents to 2^16383): the definition for graphs whose path
 * counts overflow uint64 and double, such as large grids (counts near
 * 2^4088 on a 2048 x 2048 grid).  Order of operations as brandes_one. */
static uint64_t brandes_one_q(uint32_t n, const uint32_t *offs, const uint32_t *adj, uint32_t s, int32_t *lvl,
                              __float128 *sigma, __float128 *delta, uint32_t *queue, uint32_t *lvl_start,
                              uint32_t *depth_out) {
    for (uint32_t v = 0; v < n; ++v) { lvl[v] = -1; sigma[v] = 0; delta[v] = 0; }
    uint32_t head = 0, tail = 0, nlev = 0;
    lvl[s] = 0;
    sigma[s] = 1;
    queue[tail++] = s;
    lvl_start[0] = 0;
    while (head < tail) {
        uint32_t level_end = tail;
        int32_t d = lvl[queue[head]];
        lvl_start[++nlev] = level_end;
        for (; head < level_end; ++head) {
            uint32_t c = queue[head];
            for (uint32_t e = offs[c]; e < offs[c + 1]; ++e) {
                uint32_t r = adj[e];
                if (lvl[r] == -1) { lvl[r] = d + 1; queue[tail++] = r; }
                if (lvl[r] == d + 1) sigma[r] += sigma[c];
            }
        }
    }
    for (int64_t depth = (int64_t)nlev - 2; depth >= 0; --depth) {
        for (uint32_t i = lvl_start[depth]; i < lvl_start[depth + 1]; ++i) {
            uint32_t c = queue[i];
            __float128 acc = delta[c];
            for (uint32_t e = offs[c]; e < offs[c + 1]; ++e) {
                uint32_t r = adj[e];
                if (lvl[r] == (int32_t)depth + 1) acc += (delta[r] + 1) / sigma[r] * sigma[c];
            }
            delta[c] = acc;
        }
    }
    if (depth_out) *depth_out = nlev ? nlev - 1 : 0;
    return tail;
}

int oracle_single_source_q(uint32_t n, const uint32_t *offs, const uint32_t *adj, uint32_t src, int32_t *level,
                           double *sigma_log2, double *delta) {
    if (src >= n) return -1;
    uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    uint32_t *ls = (uint32_t *)malloc(((size_t)n + 2) * sizeof(uint32_t));
    int32_t *l = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    __float128 *sg = (__float128 *)malloc((size_t)n * sizeof(__float128));
    __float128 *dl = (__float128 *)malloc((size_t)n * sizeof(__float128));
    int rc = (queue && ls && l && sg && dl) ? 0 : -2;
    if (!rc) {
        brandes_one_q(n, offs, adj, src, l, sg, dl, queue, ls, NULL);
        for (uint32_t v = 0; v < n; ++v) {
            if (level) level[v] = l[v];
            if (sigma_log2) sigma_log2[v] = sg[v] > 0 ? (double)log2q(sg[v]) : -INFINITY;
            if (delta) delta[v] = (double)dl[v];
        }
    }
    free(queue); free(ls); free(l); free(sg); free(dl);
    return rc;
}

int oracle_bc_q(uint32_t n, const uint32_t *offs, const uint32_t *adj, const uint32_t *sources, uint64_t nsrc,
                int nthreads, double *bc, oracle_stats *st) {
    int nt = nthreads > 0 ? nthreads : 1;
#ifndef _OPENMP
    nt = 1;
#endif
    __float128 *part = (__float128 *)calloc((size_t)nt * n, sizeof(__float128));
    if (!part) return -2;
    uint64_t skipped = 0, visited = 0, teps_edges = 0, ran = 0;
    uint32_t maxdepth = 0;
    int err = 0;
#pragma omp parallel num_threads(nt) reduction(+ : skipped, visited, teps_edges, ran) reduction(max : maxdepth) \
    reduction(| : err)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int32_t *lvl = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        __float128 *sigma = (__float128 *)malloc((size_t)n * sizeof(__float128));
        __float128 *delta = (__float128 *)malloc((size_t)n * sizeof(__float128));
        uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        uint32_t *ls = (uint32_t *)malloc(((size_t)n + 2) * sizeof(uint32_t));
        __float128 *mine = part + (size_t)tid * n;
        if (!lvl || !sigma || !delta || !queue || !ls) err = 1;
#pragma omp for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)nsrc; ++i) {
            if (err) continue;
            uint32_t s = sources[i];
            if (s >= n) { err = 1; continue; }
            if (offs[s + 1] == offs[s]) { skipped++; continue; }
            uint32_t depth = 0;
            uint64_t nv = brandes_one_q(n, offs, adj, s, lvl, sigma, delta, queue, ls, &depth);
            uint64_t degsum = 0;
            for (uint64_t q = 0; q < nv; ++q) {
                uint32_t v = queue[q];
                degsum += offs[v + 1] - offs[v];
                if (v != s) mine[v] += delta[v];
            }
            visited += nv;
            teps_edges += degsum / 2;
            ran++;
            if (depth > maxdepth) maxdepth = depth;
        }
        free(lvl); free(sigma); free(delta); free(queue); free(ls);
    }
    for (uint32_t v = 0; v < n; ++v) {
        __float128 acc = 0;
        for (int t = 0; t < nt; ++t) acc += part[(size_t)t * n + v];
        bc[v] += (double)acc;
    }
    free(part);
    if (st) {
        st->skipped = skipped;
        st->ran = ran;
        st->visited = visited;
        st->teps_edges = teps_edges;
        st->max_depth = maxdepth;
        st->overflow = 0;
    }
    return err ? -1 : 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
