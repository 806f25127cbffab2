/*
 * Stub implementations of the H2Pack entry points the reference calls that need no
 * matrix (test infrastructure only, linked into oracle/_ref/libtsne_ref.so): timers,
 * printing, the allocation pool, proxy-point files (the oracle's bases use their own
 * analytic proxies) and dense-matrix release. The entry points that make the matrix
 * (H2P_init, H2P_partition_points, H2P_build, H2P_destroy) and the kernel evaluation are
 * in h2_assemble.c: they build the oracle's H2 matrix and hand it to the reference.
 */
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "H2Pack.h"
#include "utils.h"

double get_wtime_sec(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

void H2P_generate_proxy_point_ID_file(H2Pack_p h2pack, const void *krnl_param,
                                      shim_krnl_eval_fptr krnl_eval, const char *fname,
                                      H2P_dense_mat_p **pp_)
{
    (void)krnl_param; (void)krnl_eval; (void)fname;
    const int n = (h2pack->max_level > 0 ? h2pack->max_level : 0) + 1;
    H2P_dense_mat_p *pp = (H2P_dense_mat_p *)calloc((size_t)n, sizeof(H2P_dense_mat_p));
    for (int i = 0; pp != NULL && i < n; i++) pp[i] = (H2P_dense_mat_p)calloc(1, sizeof(shim_dense_mat_t));
    *pp_ = pp;
}

void H2P_matvec(H2Pack_p h2pack, const DTYPE *x, DTYPE *y)
{
    (void)h2pack; (void)x; (void)y;
}

void H2P_print_statistic(H2Pack_p h2pack) { (void)h2pack; }

void H2P_dense_mat_destroy(H2P_dense_mat_p *mat_)
{
    if (*mat_ != NULL) free((*mat_)->data);
    free(*mat_);
    *mat_ = NULL;
}

void malloc_aligned_pool_enable(int enable) { (void)enable; }
void malloc_aligned_pool_stats(long *hits, long *misses) { *hits = 0; *misses = 0; }

/* The reference's fused product never calls the bi-directional kernel routine; it is only
 * passed to H2P_build. */
void tsne_repulsive_kernel_bimv(const DTYPE *coord0, const int ld0, const int n0,
                                const DTYPE *coord1, const int ld1, const int n1,
                                const void *krnl_param, const DTYPE *x_in_0,
                                const DTYPE *x_in_1, DTYPE *x_out_0, DTYPE *x_out_1)
{
    (void)coord0; (void)ld0; (void)n0; (void)coord1; (void)ld1; (void)n1; (void)krnl_param;
    (void)x_in_0; (void)x_in_1; (void)x_out_0; (void)x_out_1;
}

int tsne_repulsive_kernel_bimv_flop(int pt_dim, int n0, int n1)
{
    (void)pt_dim; (void)n0; (void)n1;
    return 0;
}
