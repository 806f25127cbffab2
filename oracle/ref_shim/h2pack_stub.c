/*
 * Stub implementations of the H2Pack entry points the reference calls
 * (test infrastructure only, linked into oracle/_ref/libtsne_ref.so).
 *
 * H2P_partition_points reports a single-level tree (max_level = 0), which the
 * reference's update_h2_matrix() treats as "too shallow for an H2 matrix"
 * (tsne_h2pack.c:874-892): it destroys the matrix and leaves h2pack_W NULL, so
 * compute_repulsive_forces_h2pack() takes its exact O(N^2) branch
 * (tsne_h2pack.c:404-491) on every iteration. The H2 build, matvec and kernel
 * routines are never reached on that path; they only have to link.
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

void H2P_init(H2Pack_p *h2pack_, const int pt_dim, const int krnl_dim, const int QR_stop_type,
              void *QR_stop_param)
{
    (void)QR_stop_type; (void)QR_stop_param;
    H2Pack_p h = (H2Pack_p)calloc(1, sizeof(shim_h2pack_t));
    if (h != NULL) {
        h->pt_dim = pt_dim;
        h->krnl_dim = krnl_dim;
        h->n_thread = 1;
    }
    *h2pack_ = h;
}

void H2P_destroy(H2Pack_p *h2pack_)
{
    H2Pack_p h = *h2pack_;
    if (h == NULL) return;
    free(h->root_enbox);
    free(h);
    *h2pack_ = NULL;
}

void H2P_partition_points(H2Pack_p h2pack, const int n_point, const DTYPE *coord,
                          int max_leaf_points, DTYPE max_leaf_size)
{
    (void)coord; (void)max_leaf_points; (void)max_leaf_size;
    h2pack->n_point = n_point;
    h2pack->krnl_mat_size = n_point;
    h2pack->max_level = 0;      /* root only: the caller switches to its direct path */
    h2pack->n_node = 1;
    h2pack->n_leaf_node = 1;
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

void H2P_build(H2Pack_p h2pack, H2P_dense_mat_p *pp, const int BD_JIT, void *krnl_param,
               shim_krnl_eval_fptr krnl_eval, shim_krnl_bimv_fptr krnl_bimv,
               const int krnl_bimv_flop)
{
    (void)h2pack; (void)pp; (void)BD_JIT; (void)krnl_param; (void)krnl_eval;
    (void)krnl_bimv; (void)krnl_bimv_flop;
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

/* Kernel routines of the reference's tsne_kernels.c, which includes H2Pack headers by
 * relative path and cannot be compiled here. They are only passed to H2P_build /
 * H2P_generate_proxy_point_ID_file above, which never call them. */
void tsne_repulsive_kernel_eval(const DTYPE *coord0, const int ld0, const int n0,
                                const DTYPE *coord1, const int ld1, const int n1,
                                const void *krnl_param, DTYPE *mat, const int ldm)
{
    (void)coord0; (void)ld0; (void)n0; (void)coord1; (void)ld1; (void)n1;
    (void)krnl_param; (void)mat; (void)ldm;
}

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
