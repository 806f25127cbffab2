/*
 * The H2 matrix the oracle builds (oracle/tsne_oracle.c), handed to the reference's own code
 * (test infrastructure only, linked into oracle/_ref/libtsne_ref.so together with the
 * oracle library).
 *
 * H2P_init / H2P_partition_points / H2P_build / H2P_destroy stand in for H2Pack's: the
 * partition builds the oracle's matrix (tree, lists, bases) for the reference's Y, and the
 * build fills the H2Pack fields that the reference's fused product
 * (src/tsne_h2_matmul.c:225-452, just-in-time B and D blocks) reads: tree arrays, reduced
 * admissible / inadmissible pair lists, U bases and skeleton coordinates. The reference's
 * update_h2_matrix, tsne_run schedule, renumbering, product, Z identity and force
 * (src/tsne_h2pack.c) then run unmodified on it.
 *
 * shim_h2_assemble does the same from arrays (any matrix, e.g. the device's), and
 * shim_ref_repulsion runs the reference's compute_repulsive_forces_h2pack
 * (src/tsne_h2pack.c:389-630) on such a matrix.
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "H2Pack.h"
#include "tsne_h2pack.h"
#include "../tsne_oracle.h"

/* (1 + r^2)^-2 for every pair of two point sets; coordinate k of point i at c[k * ld + i];
 * krnl_param points to the dimension (the reference passes &low_dim). The reference's own
 * routine (tsne_kernels.c) includes H2Pack headers and cannot be compiled here. */
void tsne_repulsive_kernel_eval(const DTYPE *coord0, const int ld0, const int n0, const DTYPE *coord1,
                                const int ld1, const int n1, const void *krnl_param, DTYPE *mat, const int ldm)
{
    const int d = krnl_param ? *(const int *)krnl_param : 2;
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++) {
            DTYPE r2 = 0.0;
            for (int k = 0; k < d; k++) {
                const DTYPE df = coord0[(size_t)k * ld0 + i] - coord1[(size_t)k * ld1 + j];
                r2 += df * df;
            }
            const DTYPE q = 1.0 + r2;
            mat[(size_t)i * ldm + j] = 1.0 / (q * q);
        }
}

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

/* Fills h from a matrix given as arrays. n points in d dimensions; perm: tree position ->
 * point; coord: d x n in tree order. Node t: points [start, end) in tree order, level,
 * first child and child count (children are consecutive ids), is_leaf. adm_pairs /
 * inadm_pairs: n_adm / n_inadm unordered node pairs (the inadmissible ones between
 * distinct leaves). rank, ncand, U (U_off: block of node t, ncand x rank row-major),
 * skeleton points skel (d coordinates each, skel_off). */
static void shim_fill(shim_h2pack_t *h, int n, int d, int max_level, int n_node, const int *perm,
                      const double *coord, const int *start, const int *end, const int *level, const int *fchild,
                      const int *nchild, const int *is_leaf, int n_adm, const int *adm_pairs, int n_inadm,
                      const int *inadm_pairs, const int *rank, const int *ncand, const double *U,
                      const int *U_off, const double *skel, const int *skel_off)
{
    const int max_child = 1 << d;
    int n_leaf = 0;
    for (int t = 0; t < n_node; t++) n_leaf += is_leaf[t] != 0;
    h->pt_dim = d;
    h->krnl_dim = 1;
    h->n_point = n;
    h->krnl_mat_size = n;
    h->max_level = max_level;
    h->min_adm_level = 2;
    h->max_child = max_child;
    h->n_node = n_node;
    h->n_leaf_node = n_leaf;
    h->n_UJ = n_node;
    h->BD_JIT = 1;   /* B and D blocks are never stored here: the product evaluates them */
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
}

static void shim_release(shim_h2pack_t *h)
{
    if (h->U != NULL)
        for (int t = 0; t < h->n_node; t++) {
            H2P_dense_mat_destroy(&h->U[t]);
            H2P_dense_mat_destroy(&h->J_coord[t]);
        }
    free(h->U); free(h->J_coord);
    free(h->children); free(h->n_child); free(h->node_level); free(h->level_nodes); free(h->level_n_node);
    free(h->height_nodes); free(h->mat_cluster); free(h->pt_cluster); free(h->fwd_pmt_idx); free(h->bwd_pmt_idx);
    free(h->coord); free(h->r_adm_pairs); free(h->B_nrow); free(h->B_ncol); free(h->r_inadm_pairs);
    free(h->D_nrow); free(h->D_ncol);
    free(h->root_enbox);
    ora_h2_free((ora_h2 *)h->ora);
}

/* ---- H2Pack entry points the reference calls to make its matrix ---- */

void H2P_init(H2Pack_p *h2pack_, const int pt_dim, const int krnl_dim, const int QR_stop_type,
              void *QR_stop_param)
{
    (void)QR_stop_type;
    H2Pack_p h = (H2Pack_p)calloc(1, sizeof(shim_h2pack_t));
    if (h != NULL) {
        h->pt_dim = pt_dim;
        h->krnl_dim = krnl_dim;
        h->n_thread = omp_get_max_threads();   /* the reference sets num_threads just before */
        h->qr_tol = QR_stop_param ? *(const DTYPE *)QR_stop_param : 1e-6;
    }
    *h2pack_ = h;
}

void H2P_destroy(H2Pack_p *h2pack_)
{
    H2Pack_p h = *h2pack_;
    if (h == NULL) return;
    shim_release(h);
    free(h);
    *h2pack_ = NULL;
}

/* The oracle's tree, lists and bases for the points (coord: pt_dim x n_point, the caller's
 * order). max_leaf_points 0 means the default leaf size of 200. A tree of at most two
 * levels reports its depth, which makes the reference take its direct path. */
void H2P_partition_points(H2Pack_p h, const int n_point, const DTYPE *coord, int max_leaf_points,
                          DTYPE max_leaf_size)
{
    (void)max_leaf_size;
    const int leaf = max_leaf_points > 0 ? max_leaf_points : 200;
    int status = 0;
    ora_h2 *o = ora_h2_build(coord, n_point, h->pt_dim, leaf, h->qr_tol, h->n_thread, &status);
    h->n_point = n_point;
    h->krnl_mat_size = n_point;
    h->coord_src = coord;
    h->ora = o;
    if (o == NULL) {
        h->n_leaf_node = 0;   /* the reference reports the failure */
        return;
    }
    h->max_level = ora_h2_max_level(o);
    h->n_node = ora_h2_n_node(o);
    h->n_leaf_node = 1;
    if (status != 0) return;   /* too shallow: the caller switches to its direct path */
}

void H2P_build(H2Pack_p h, H2P_dense_mat_p *pp, const int BD_JIT, void *krnl_param, shim_krnl_eval_fptr krnl_eval,
               shim_krnl_bimv_fptr krnl_bimv, const int krnl_bimv_flop)
{
    (void)pp; (void)BD_JIT; (void)krnl_bimv; (void)krnl_bimv_flop;
    ora_h2 *o = (ora_h2 *)h->ora;
    if (o == NULL) return;
    const int n = h->n_point, d = h->pt_dim, nn = ora_h2_n_node(o);
    int *start = (int *)malloc(sizeof(int) * nn * 7);
    int *end = start + nn, *level = end + nn, *parent = level + nn, *fchild = parent + nn, *nchild = fchild + nn,
        *is_leaf = nchild + nn;
    ora_h2_nodes(o, start, end, level, parent, fchild, nchild, is_leaf);
    const int nf = ora_h2_n_far(o), nr = ora_h2_n_near(o);
    int *fp = (int *)malloc(sizeof(int) * (nn + 1)), *np_ = (int *)malloc(sizeof(int) * (nn + 1));
    int *fi = (int *)malloc(sizeof(int) * (nf + 1)), *ni = (int *)malloc(sizeof(int) * (nr + 1));
    ora_h2_lists(o, fp, fi, np_, ni);
    int *adm = (int *)malloc(sizeof(int) * (nf + 1)), *inadm = (int *)malloc(sizeof(int) * (nr + 1));
    int n_adm = 0, n_inadm = 0;
    for (int t = 0; t < nn; t++) {
        for (int e = fp[t]; e < fp[t + 1]; e++)
            if (fi[e] > t) { adm[2 * n_adm] = t; adm[2 * n_adm + 1] = fi[e]; n_adm++; }
        for (int e = np_[t]; e < np_[t + 1]; e++)
            if (ni[e] > t) { inadm[2 * n_inadm] = t; inadm[2 * n_inadm + 1] = ni[e]; n_inadm++; }
    }
    int *rank = (int *)malloc(sizeof(int) * nn), *ncand = (int *)malloc(sizeof(int) * nn);
    int *skel_off = (int *)malloc(sizeof(int) * (nn + 1)), *U_off = (int *)malloc(sizeof(int) * (nn + 1));
    ora_h2_ranks(o, rank);
    ora_h2_bases(o, ncand, skel_off, U_off);
    const int *perm = ora_h2_perm(o);
    double *xt = (double *)malloc(sizeof(double) * (size_t)d * n);
    /* the tree order's coordinates, from the points the partition saw */
    const double *Y = h->coord_src;
    for (int k = 0; k < d; k++)
        for (int i = 0; i < n; i++) xt[(size_t)k * n + i] = Y[(size_t)k * n + perm[i]];
    shim_fill(h, n, d, ora_h2_max_level(o), nn, perm, xt, start, end, level, fchild, nchild, is_leaf, n_adm, adm,
              n_inadm, inadm, rank, ncand, ora_h2_U(o), U_off, ora_h2_skel(o), skel_off);
    h->krnl_eval = krnl_eval;
    h->krnl_param = krnl_param;
    free(xt); free(start); free(fp); free(np_); free(fi); free(ni); free(adm); free(inadm);
    free(rank); free(ncand); free(skel_off); free(U_off);
}

/* ---- the same from arrays, and the reference's force on such a matrix ---- */

typedef struct {
    shim_h2pack_t h;
    int dim;
} shim_assembled_t;

H2Pack_p shim_h2_assemble(int n, int d, int max_level, int n_node, const int *perm, const double *coord,
                          const int *start, const int *end, const int *level, const int *fchild,
                          const int *nchild, const int *is_leaf, int n_adm, const int *adm_pairs, int n_inadm,
                          const int *inadm_pairs, const int *rank, const int *ncand, const double *U,
                          const int *U_off, const double *skel, const int *skel_off)
{
    shim_assembled_t *a = (shim_assembled_t *)calloc(1, sizeof(shim_assembled_t));
    a->dim = d;
    a->h.n_thread = 1;
    shim_fill(&a->h, n, d, max_level, n_node, perm, coord, start, end, level, fchild, nchild, is_leaf, n_adm,
              adm_pairs, n_inadm, inadm_pairs, rank, ncand, U, U_off, skel, skel_off);
    a->h.krnl_eval = tsne_repulsive_kernel_eval;
    a->h.krnl_param = &a->dim;
    return &a->h;
}

void shim_h2_free(H2Pack_p h)
{
    if (h == NULL) return;
    shim_release(h);
    free(h);   /* the shim_assembled_t that holds h at offset 0 */
}

/* The reference's repulsive force on the matrix: grad -= F (grad d x n, the caller's order;
 * zero on entry gives -F); returns Z. */
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
