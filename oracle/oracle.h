/* ORACLE — test infrastructure only (see brandes.c).  Not part of the product. */
#ifndef BCG_ORACLE_H_
#define BCG_ORACLE_H_
#include <stdint.h>

typedef struct oracle_stats {
    uint64_t skipped;     /* sources of degree 0 */
    uint64_t ran;         /* sources run */
    uint64_t visited;     /* sum of visited vertices */
    uint64_t teps_edges;  /* sum over sources of (sum of degrees of visited) / 2 */
    uint32_t max_depth;
    int overflow;         /* a uint64 sigma sum wrapped */
} oracle_stats;

int oracle_single_source(uint32_t n, const uint32_t *offs, const uint32_t *adj, uint32_t src,
                         int32_t *level, uint64_t *sigma, double *delta, int *overflow);
/* Adds every source's dependencies into bc[n] (ordered-pair sums). */
int oracle_bc(uint32_t n, const uint32_t *offs, const uint32_t *adj, const uint32_t *sources,
              uint64_t nsrc, int nthreads, double *bc, oracle_stats *st);
/* Sum over sources (degree 0 skipped) and reachable t != s of (d(s,t) - 1):
 * the exact total of bc[] over that source set. */
int oracle_path_length_sum(uint32_t n, const uint32_t *offs, const uint32_t *adj, const uint32_t *sources,
                           uint64_t nsrc, int nthreads, uint64_t *total);
/* Sigma and delta as __float128 (graphs whose path counts overflow uint64):
 * sigma_log2[v] = log2(sigma_v) (-inf for 0). */
int oracle_single_source_q(uint32_t n, const uint32_t *offs, const uint32_t *adj, uint32_t src, int32_t *level,
                           double *sigma_log2, double *delta);
int oracle_bc_q(uint32_t n, const uint32_t *offs, const uint32_t *adj, const uint32_t *sources, uint64_t nsrc,
                int nthreads, double *bc, oracle_stats *st);
int oracle_max_threads(void);
#endif
