/*
 * Interface stand-in for the absent H2Pack library (test infrastructure only).
 *
 * The reference's optimisation loop (src/tsne_h2pack.c, src/tsne_h2_matmul.c,
 * src/tsne_reorder.c, src/tsne_utils.c) is compiled unmodified against this
 * header. The H2Pack git submodule is empty in the reference checkout, so nothing
 * here is H2Pack code: the struct below only declares the member names the reference
 * sources read (tsne_h2pack.c:107-136, 772-953; tsne_h2_matmul.c:196-249) so that
 * they compile, and h2_assemble.c fills them with the H2 matrix the oracle builds
 * (oracle/tsne_oracle.c). The reference's own loop, rebuild schedule, renumbering,
 * fused product, Z identity and force then run on the oracle's matrices; for
 * N < 2000 or a tree of at most two levels they take their direct O(N^2) branch.
 */
#ifndef ORACLE_REF_SHIM_H2PACK_H
#define ORACLE_REF_SHIM_H2PACK_H

#include <stddef.h>
#include <stdio.h>

#ifndef DTYPE
#define DTYPE double
#endif
#define DTYPE_SIZE 8

#define QR_REL_NRM 1

typedef struct {
    int nrow, ncol, ld, size;
    DTYPE *data;
} shim_dense_mat_t;
typedef shim_dense_mat_t *H2P_dense_mat_p;

typedef void (*shim_krnl_eval_fptr)(const DTYPE *coord0, const int ld0, const int n0,
                                    const DTYPE *coord1, const int ld1, const int n1,
                                    const void *krnl_param, DTYPE *mat, const int ldm);
typedef void (*shim_krnl_bimv_fptr)(const DTYPE *coord0, const int ld0, const int n0,
                                    const DTYPE *coord1, const int ld1, const int n1,
                                    const void *krnl_param, const DTYPE *x_in_0,
                                    const DTYPE *x_in_1, DTYPE *x_out_0, DTYPE *x_out_1);

typedef struct {
    int pt_dim, krnl_dim, n_point, krnl_mat_size, n_thread;
    int max_level, min_adm_level, max_child, n_node, n_leaf_node, n_UJ;
    int is_HSS, BD_JIT, print_timers, print_dbginfo;
    int n_r_adm_pair, n_r_inadm_pair;
    int *children, *n_child, *level_nodes, *level_n_node, *node_level, *height_nodes;
    int *mat_cluster, *pt_cluster, *r_adm_pairs, *r_inadm_pairs;
    int *fwd_pmt_idx, *bwd_pmt_idx;
    int *B_nrow, *B_ncol, *D_nrow, *D_ncol;
    size_t *B_ptr, *D_ptr;
    DTYPE *B_data, *D_data;
    DTYPE *coord, *root_enbox;
    H2P_dense_mat_p *U, *J_coord;
    shim_krnl_eval_fptr krnl_eval;
    const void *krnl_param;
    double timers[9];
    /* shim only: the oracle's matrix behind H2P_partition_points / H2P_build, and the
     * relative tolerance H2P_init received */
    void *ora;
    double qr_tol;
    const DTYPE *coord_src;   /* the points the partition saw (the caller's order) */
} shim_h2pack_t;
typedef shim_h2pack_t *H2Pack_p;

void H2P_init(H2Pack_p *h2pack_, const int pt_dim, const int krnl_dim, const int QR_stop_type,
              void *QR_stop_param);
void H2P_destroy(H2Pack_p *h2pack_);
void H2P_partition_points(H2Pack_p h2pack, const int n_point, const DTYPE *coord,
                          int max_leaf_points, DTYPE max_leaf_size);
void H2P_generate_proxy_point_ID_file(H2Pack_p h2pack, const void *krnl_param,
                                      shim_krnl_eval_fptr krnl_eval, const char *fname,
                                      H2P_dense_mat_p **pp_);
void H2P_build(H2Pack_p h2pack, H2P_dense_mat_p *pp, const int BD_JIT, void *krnl_param,
               shim_krnl_eval_fptr krnl_eval, shim_krnl_bimv_fptr krnl_bimv,
               const int krnl_bimv_flop);
void H2P_matvec(H2Pack_p h2pack, const DTYPE *x, DTYPE *y);
void H2P_print_statistic(H2Pack_p h2pack);
void H2P_dense_mat_destroy(H2P_dense_mat_p *mat_);
void malloc_aligned_pool_enable(int enable);
void malloc_aligned_pool_stats(long *hits, long *misses);

#endif
