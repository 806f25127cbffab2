/*
 * Hands an H2 matrix built by the oracle (oracle/tsne_oracle.c) to the reference's own
 * product and force code (test infrastructure only, linked into oracle/_ref/libtsne_ref.so).
 *
 * shim_h2_assemble fills the H2Pack fields that the reference's fused product
 * (src/tsne_h2_matmul.c:225-452, just-in-time B and D blocks) reads: tree arrays, reduced
 * admissible / inadmissible pair lists, U bases and skeleton coordinates. shim_ref_repulsion
 * then runs the reference's compute_repulsive_forces_h2pack (src/tsne_h2pack.c:389-630) on it:
 * the fused product, the removal of the diagonal, the Z identity and the force. Comparing
 * that with the oracle's own product and force on the same matrix pins the oracle's
 * restatement of those steps to the reference's code.
 */
#include <stdlib.h>
#include <string.h>

#include "H2Pack.h"
#include "tsne_h2pack.h"

/* (1 + r^2)^-2 for every pair of two point sets; coordinate k of point i at c[k * ld + i];
 * krnl_param points to the dimension, as for the reference's tsne_repulsive_kernel_eval */
static void shim_rkernel_eval(const DTYPE *c0, const int ld0, const int n0, const DTYPE *c1, const int ld1,
                              const int n1, const void *param, DTYPE *mat, const int ldm)
{
    const int d = *(const int *)param;
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++) {
            DTYPE r2 = 0.0;
            for (int k = 0; k < d; k++) {
                const DTYPE df = c0[(size_t)k * ld0 + i] - c1[(size_t)k * ld1 + j];
                r2 += df * df;
            }
            const DTYPE q = 1.0 + r2;
            mat[(size_t)i * ldm + j] = 1.0 / (q * q);
        }
}

typedef struct {
    shim_h2pack_t h;
    int dim;
} shim_assembled_t;

static H2P_dense_mat_p shim_mat(int nrow, int ncol)
{
    H2P_dense_mat_p m = (H2P_dense_mat_p)calloc(1, sizeof(shim_dense_mat_t));
    m->nrow = nrow;
    m->ncol = ncol;
    m->ld = ncol;
    m->size = nrow * ncol;
    m->data = (DTYPE *)calloc((size_t)nrow * ncol + 1, sizeof(DTYPE));
    return m;
}

/*
 * n points in d dimensions; perm: tree position -> point; coord: d x n in tree order.
 * Node t: points [start, end) in tree order, level, first child and child count (children
 * are consecutive ids), is_leaf. adm_pairs / inadm_pairs: n_adm / n_inadm unordered node
 * pairs (the inadmissible ones between distinct leaves). rank, ncand, U (U_off: block of
 * node t, ncand x rank row-major), skeleton points skel (d coordinates each, skel_off).
 */
H2Pack_p shim_h2_assemble(int n, int d, int max_level, int n_node, const int *perm, const double *coord,
                          const int *start, const int *end, const int *level, const int *fchild,
                          const int *nchild, const int *is_leaf, int n_adm, const int *adm_pairs, int n_inadm,
                          const int *inadm_pairs, const int *rank, const int *ncand, const double *U,
                          const int *U_off, const double *skel, const int *skel_off)
{
    shim_assembled_t *a = (shim_assembled_t *)calloc(1, sizeof(shim_assembled_t));
    shim_h2pack_t *h = &a->h;
    a->dim = d;
    const int max_child = 1 << d;
    int n_leaf = 0;
    for (int t = 0; t < n_node; t++) n_leaf += is_leaf[t] != 0;
    h->pt_dim = d;
    h->krnl_dim = 1;
    h->n_point = n;
    h->krnl_mat_size = n;
    h->n_thread = 1;
    h->max_level = max_level;
    h->min_adm_level = 2;
    h->max_child = max_child;
    h->n_node = n_node;
    h->n_leaf_node = n_leaf;
    h->BD_JIT = 1;
    h->children = (int *)calloc((size_t)n_node * max_child, sizeof(int));
    h->n_child = (int *)calloc((size_t)n_node, sizeof(int));
    h->node_level = (int *)calloc((size_t)n_node, sizeof(int));
    h->level_nodes = (int *)calloc((size_t)(max_level + 1) * n_leaf, sizeof(int));
    h->level_n_node = (int *)calloc((size_t)(max_level + 1), sizeof(int));
    h->height_nodes = (int *)calloc((size_t)n_leaf, sizeof(int));
    h->mat_cluster = (int *)calloc((size_t)2 * n_node, sizeof(int));
    h->pt_cluster = (int *)calloc((size_t)2 * n_node, sizeof(int));
    int nl = 0;
    for (int t = 0; t < n_node; t++) {
        h->n_child[t] = nchild[t];
        for (int k = 0; k < nchild[t]; k++) h->children[(size_t)t * max_child + k] = fchild[t] + k;
        h->node_level[t] = level[t];
        h->level_nodes[(size_t)level[t] * n_leaf + h->level_n_node[level[t]]++] = t;
        if (is_leaf[t]) h->height_nodes[nl++] = t;
        h->mat_cluster[2 * t] = h->pt_cluster[2 * t] = start[t];
        h->mat_cluster[2 * t + 1] = h->pt_cluster[2 * t + 1] = end[t] - 1;
    }
    h->fwd_pmt_idx = (int *)malloc(sizeof(int) * n);
    h->bwd_pmt_idx = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++) {
        h->fwd_pmt_idx[i] = perm[i];
        h->bwd_pmt_idx[perm[i]] = i;
    }
    h->coord = (DTYPE *)malloc(sizeof(DTYPE) * (size_t)d * n);
    memcpy(h->coord, coord, sizeof(DTYPE) * (size_t)d * n);

    h->U = (H2P_dense_mat_p *)calloc((size_t)n_node, sizeof(H2P_dense_mat_p));
    h->J_coord = (H2P_dense_mat_p *)calloc((size_t)n_node, sizeof(H2P_dense_mat_p));
    for (int t = 0; t < n_node; t++) {
        const int r = rank[t], m = r > 0 ? ncand[t] : 0;
        h->U[t] = shim_mat(m, r);
        memcpy(h->U[t]->data, U + U_off[t], sizeof(DTYPE) * (size_t)m * r);
        h->J_coord[t] = shim_mat(d, r);
        for (int b = 0; b < r; b++)
            for (int k = 0; k < d; k++)
                h->J_coord[t]->data[(size_t)k * r + b] = skel[((size_t)skel_off[t] + b) * d + k];
    }

    h->n_r_adm_pair = n_adm;
    h->r_adm_pairs = (int *)malloc(sizeof(int) * (2 * (size_t)n_adm + 1));
    memcpy(h->r_adm_pairs, adm_pairs, sizeof(int) * 2 * (size_t)n_adm);
    h->B_nrow = (int *)malloc(sizeof(int) * ((size_t)n_adm + 1));
    h->B_ncol = (int *)malloc(sizeof(int) * ((size_t)n_adm + 1));
    for (int i = 0; i < n_adm; i++) {
        const int t0 = adm_pairs[2 * i], t1 = adm_pairs[2 * i + 1];
        h->B_nrow[i] = level[t0] >= level[t1] ? rank[t0] : end[t0] - start[t0];
        h->B_ncol[i] = level[t1] >= level[t0] ? rank[t1] : end[t1] - start[t1];
    }
    h->n_r_inadm_pair = n_inadm;
    h->r_inadm_pairs = (int *)malloc(sizeof(int) * (2 * (size_t)n_inadm + 1));
    memcpy(h->r_inadm_pairs, inadm_pairs, sizeof(int) * 2 * (size_t)n_inadm);
    h->D_nrow = (int *)malloc(sizeof(int) * ((size_t)n_leaf + n_inadm + 1));
    h->D_ncol = (int *)malloc(sizeof(int) * ((size_t)n_leaf + n_inadm + 1));
    for (int i = 0; i < n_leaf; i++) {
        const int t = h->height_nodes[i];
        h->D_nrow[i] = h->D_ncol[i] = end[t] - start[t];
    }
    for (int i = 0; i < n_inadm; i++) {
        const int t0 = inadm_pairs[2 * i], t1 = inadm_pairs[2 * i + 1];
        h->D_nrow[n_leaf + i] = end[t0] - start[t0];
        h->D_ncol[n_leaf + i] = end[t1] - start[t1];
    }
    h->krnl_eval = shim_rkernel_eval;
    h->krnl_param = &a->dim;
    return (H2Pack_p)a;
}

void shim_h2_free(H2Pack_p hp)
{
    if (hp == NULL) return;
    shim_h2pack_t *h = hp;
    for (int t = 0; t < h->n_node; t++) {
        H2P_dense_mat_destroy(&h->U[t]);
        H2P_dense_mat_destroy(&h->J_coord[t]);
    }
    free(h->U); free(h->J_coord);
    free(h->children); free(h->n_child); free(h->node_level); free(h->level_nodes); free(h->level_n_node);
    free(h->height_nodes); free(h->mat_cluster); free(h->pt_cluster); free(h->fwd_pmt_idx); free(h->bwd_pmt_idx);
    free(h->coord); free(h->r_adm_pairs); free(h->B_nrow); free(h->B_ncol); free(h->r_inadm_pairs);
    free(h->D_nrow); free(h->D_ncol);
    free(hp);   /* the shim_assembled_t that holds h at offset 0 */
}

/* The reference's repulsive force on the assembled matrix: grad -= F (grad d x n, caller's
 * order, zero on entry gives -F); returns Z. */
double shim_ref_repulsion(H2Pack_p h, const double *Y, int d, int n, double *grad)
{
    tsne_params_t prm = tsne_create_default_params();
    prm.num_threads = 1;
    prm.h2_rebuild_freq = 3;
    tsne_workspace_t ws;
    memset(&ws, 0, sizeof(ws));
    ws.n_point = n;
    ws.low_dim = d;
    ws.params = &prm;
    ws.s = (DTYPE *)calloc((size_t)n, sizeof(DTYPE));
    ws.v = (DTYPE *)calloc((size_t)d * n, sizeof(DTYPE));
    ws.ones = (DTYPE *)malloc(sizeof(DTYPE) * (size_t)n);
    for (int i = 0; i < n; i++) ws.ones[i] = 1.0;
    const double Z = compute_repulsive_forces_h2pack(h, Y, d, n, &ws, grad, 0);
    tsne_h2_matmul_free(&ws.mm_ws);
    free(ws.s); free(ws.v); free(ws.ones);
    return Z;
}
