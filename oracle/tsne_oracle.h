/*
 * CPU oracle for the t-SNE optimisation phase (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C, FP64 restatement of the reference's optimisation path, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker. Nothing on
 * the product path links or calls it.
 *
 * What it restates (reference files, paths within the reference project):
 *   - conditional P by beta bisection ........ src/tsne_utils.c:952-1105
 *   - random initial embedding (srand/Box-Muller) src/tsne_utils.c:1111-1150
 *   - attractive force ........................ src/tsne_h2pack.c:290-356
 *   - exact repulsion, Z identity, force ...... src/tsne_h2pack.c:404-491, 538-627
 *   - KL divergence ........................... src/tsne_h2pack.c:1870-1895
 *   - gains / momentum update, centring ....... src/tsne_h2pack.c:1942-1984
 *   - rebuild / reuse / renumbering schedule .. src/tsne_h2pack.c:1652-1860
 *   - point renumbering (P permuted, rows sorted by new column) src/tsne_reorder.c:112-167
 *   - H2 construction and fused product: the reference delegates these to the absent
 *     H2Pack library (tsne_h2pack.c:772-953, tsne_h2_matmul.c:225-452). This file holds
 *     this project's own H2 design (tree from sorted Morton keys, per-target near/far
 *     lists, proxy-point interpolative decomposition), which the device code follows
 *     bit for bit on the tree and the lists.
 *
 * Parity status: the exact path, P calibration and initialisation are pinned against
 * the reference's own sources compiled here (oracle/_ref) and its known-answer tests;
 * the H2 part is pinned against the exact FP64 O(N^2) sums only (H2Pack absent).
 */
#ifndef TSNE_ORACLE_H
#define TSNE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- setup ---- */
int  ora_conditional_P(const double *dist, const int *indptr, int n, double perplexity,
                       double *P_out, int nthreads);
void ora_init_embedding(double *Y, int n, int d, unsigned int seed);

/* ---- per-iteration pieces (Y is d x n, dimension-major) ---- */
void   ora_exact_sv(const double *Y, int n, int d, double *s, double *v, int nthreads);
/* the same sums for the m points rows[]: s (m), v (d x m) */
void   ora_exact_rows(const double *Y, int n, int d, const int *rows, int m, double *s, double *v, int nthreads);
double ora_z_force(const double *Y, int n, int d, const double *s, const double *v, double *F);
void   ora_attractive(int n, int d, const int *rp, const int *ci, const double *pv,
                      const double *Y, double exag, double *attr, int nthreads);
double ora_kl(int n, int d, const int *rp, const int *ci, const double *pv, const double *Y,
              double exag, double Z, int nthreads);

/* ---- H2 matrix of (1 + r^2)^-2 ---- */
typedef struct ora_h2 ora_h2;

/* Geometry + lists + bases. Returns NULL on bad input; *status: 0 ok, -1 non-finite Y,
 * 1 tree too shallow for an H2 matrix (max_level <= 2: the caller uses the exact path). */
ora_h2 *ora_h2_build(const double *Y, int n, int d, int leaf_size, double tol, int nthreads,
                     int *status);
void    ora_h2_free(ora_h2 *h);
/* s = K 1 - 1 and v = K Y - Y (diagonal excluded), in the caller's point order */
void    ora_h2_product(const ora_h2 *h, const double *Y, double *s, double *v, int nthreads);

/* Inspection (for bit-exact comparison with the device build) */
int  ora_h2_n_node(const ora_h2 *h);
int  ora_h2_max_level(const ora_h2 *h);
int  ora_h2_tree_depth(const ora_h2 *h);
void ora_h2_root(const ora_h2 *h, double *corner, double *radius);
const int *ora_h2_perm(const ora_h2 *h);             /* tree position -> point */
const uint64_t *ora_h2_keys(const ora_h2 *h);        /* sorted keys (tree order) */
/* node table: start, end, level, parent, first_child, n_child, is_leaf */
void ora_h2_nodes(const ora_h2 *h, int *start, int *end, int *level, int *parent,
                  int *first_child, int *n_child, int *is_leaf);
int  ora_h2_n_far(const ora_h2 *h);
int  ora_h2_n_near(const ora_h2 *h);
/* CSR by target node, partners ascending */
void ora_h2_lists(const ora_h2 *h, int *far_ptr, int *far_idx, int *near_ptr, int *near_idx);
void ora_h2_ranks(const ora_h2 *h, int *rank);
/* Bases, for handing the matrix to another product code: per node the candidate rows of U
 * (a leaf's points, or its children's skeletons in child order), and the offsets of its
 * skeleton points (skel_off, n_node + 1 entries) and of its U block (U_off, n_node + 1);
 * U blocks are ncand x rank row-major, skeleton points d coordinates each. */
void ora_h2_bases(const ora_h2 *h, int *ncand, int *skel_off, int *U_off);
const double *ora_h2_U(const ora_h2 *h);
const double *ora_h2_skel(const ora_h2 *h);
int  ora_h2_n_proxy(int d);
void ora_h2_proxies(int d, double h, double *out);   /* d x n_proxy, relative to a box centre */

/* ---- whole optimisation phase (the reference's tsne_run schedule) ---- */
typedef struct {
    int    n_iter;
    double learning_rate;        /* > 0 */
    double momentum, initial_momentum;
    int    momentum_switch_iter;
    double early_exag;
    int    early_exag_iter;
    double h2_tol;
    int    h2_rebuild_freq, h2_rebuild_freq_early, h2_leaf_size;
    int    use_h2;               /* 0: exact repulsion every iteration */
    int    rep_reuse, reorder;   /* A/B switches, default 1 */
    int    nthreads;
    int    iter_begin, iter_end; /* run iterations [begin, end) only (bounded samples) */
} ora_run_params;

typedef struct {
    int n, d;
    int *rp, *ci;  double *pv;   /* P (CSR, owned) */
    double *Y, *uY, *gains, *rep;
    double rep_Z, kl;
    int rep_valid;
    int *point_order;            /* current -> caller's number */
    ora_h2 *h2;
    int next_reorder;
    int n_rebuild;
} ora_state;

ora_state *ora_state_create(int n, int d, const int *rp, const int *ci, const double *pv,
                            const double *Y0);
void ora_state_free(ora_state *st);
int  ora_run(ora_state *st, const ora_run_params *p);
void ora_get_embedding(const ora_state *st, double *Y_out);
int  ora_renumber(ora_state *st, const int *ord);

#ifdef __cplusplus
}
#endif
#endif
