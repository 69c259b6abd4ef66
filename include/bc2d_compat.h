/*
 * bc2d_compat.h — the reference's own C ABI for the single-GPU ("mono") BC
 * path, exported by libbc2d_compat.so on top of the B200 engine (libbcg.so).
 *
 * Each declaration has the signature of the reference's bc2d.h and replaces
 * the cuda_kernels.cu implementation named beside it, so that the
 * reference's host driver bc2d.c compiles unmodified and links against this
 * library instead of cuda_kernels.cu (recipe: oracle/Makefile target
 * ref-compat).  LOCINT is the reference's
 * 32-bit vertex id (bc2d.h:14).
 *
 * Semantics kept: the same call order and per-level return values as the
 * reference's bc_func_mono (bc2d.c:504-580): set_mlp_cuda seeds a source,
 * scan_col_csc_cuda_mono(ncol, level) returns the number of vertices found at
 * `level`, scan_frt_csc_cuda_mono walks back one level, update_bc_cuda adds
 * the source's dependencies (weighted by reach as in update_bc,
 * cuda_kernels.cu:263-277).  The work itself runs on the engine: one BFS +
 * dependency pass per source on the GPU, FP64 internally, float at get_bc.
 *
 * The library reads the driver's globals N (bc2d.h:187) as the vertex count,
 * like cuda_kernels.cu does.
 */
#ifndef BC2D_COMPAT_H_
#define BC2D_COMPAT_H_
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef LOCINT
#define LOCINT uint32_t
#endif

/* initcuda   cuda_kernels.cu:1123-1198  (bc2d.h:134): uploads the CSC
 * (col[N+1] offsets, row[ned] ids); returns device bytes allocated. */
size_t initcuda(uint64_t ned, LOCINT *col, LOCINT *row);
/* setcuda    cuda_kernels.cu:1100-1119  (bc2d.h:132): per-source reset. */
void setcuda(uint64_t ned, LOCINT *col, LOCINT *row, LOCINT reach_v0);
/* set_mlp_cuda cuda_kernels.cu:689-703 (bc2d.h:136): seeds source `row`. */
void set_mlp_cuda(LOCINT row, int level, int sigma);
/* scan_col_csc_cuda_mono cuda_kernels.cu:835-918 (bc2d.h:142): one forward
 * level; returns the number of vertices discovered at `level`. */
LOCINT scan_col_csc_cuda_mono(int ncol, int level);
/* scan_frt_csc_cuda_mono cuda_kernels.cu:766-827 (bc2d.h:146): one backward
 * level; returns ncol. */
LOCINT scan_frt_csc_cuda_mono(int offset, int ncol, int depth);
/* pre_update_bc_cuda cuda_kernels.cu:330-336 (bc2d.h:158): *all = sum of
 * reach over the vertices reached at level > 0. */
void pre_update_bc_cuda(LOCINT *reach, uint64_t v0, LOCINT *all);
/* update_bc_cuda cuda_kernels.cu:280-286 (bc2d.h:155): adds the source's
 * dependencies times (reach_v0 + 1) and the source term
 * reach_v0 * (nvisited - 2). */
void update_bc_cuda(uint64_t v0, int ncol, const uint64_t nvisited);
/* init_bc_1degree_device cuda_kernels.cu:1083-1087 (bc2d.h:159). */
void init_bc_1degree_device(LOCINT *reach);
/* get_deg cuda_kernels.cu:1031-1033, get_msk :1027-1029, get_bc :1039-1041. */
void get_deg(LOCINT *deg);
void get_msk(LOCINT *msk);
void get_bc(float *bc);
/* fincuda cuda_kernels.cu:1201-1232 (bc2d.h:173). */
void fincuda(void);
/* CudaMallocHostSet / CudaFreeHost cuda_kernels.cu:664-677 (bc2d.h:177-178). */
void *CudaMallocHostSet(size_t size, int val);
void CudaFreeHost(void *ptr);

#ifdef __cplusplus
}
#endif
#endif /* BC2D_COMPAT_H_ */
