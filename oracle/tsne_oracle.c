/*
 * CPU oracle for the t-SNE optimisation phase -- TEST INFRASTRUCTURE ONLY.
 * See tsne_oracle.h for what is restated from which reference file. FP64 throughout,
 * IEEE semantics (built with -ffp-contract=off), OpenMP only over independent rows,
 * nodes or targets, so every result is independent of the thread count.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "tsne_oracle.h"

#define ORA_MIN(a, b) ((a) < (b) ? (a) : (b))
#define ORA_MAX(a, b) ((a) > (b) ? (a) : (b))

/* ===================================================================================
 * Design constants of the H2 matrix. The device build defines the same values; a
 * unit test compares the two.
 * =================================================================================== */
#define ORA_KEY_DEPTH_2D 24          /* tree depth limit = Morton bits per dimension */
#define ORA_KEY_DEPTH_3D 20
#define ORA_MIN_HALF_WIDTH 5e-5      /* root half-width = this * 2^k (k >= 0) */
#define ORA_MIN_ADM_LEVEL 2          /* first level that can hold admissible pairs */
/* The ID stops at this fraction of h2_tol, which keeps the per-iteration repulsive force
 * within h2_tol (relative 2-norm) of the exact force. */
#define ORA_ID_TOL_FACTOR 0.1
#define ORA_MAX_RANK_2D 64
#define ORA_MAX_RANK_3D 160
/* Proxy points: shells |y - c|_inf = rho * h around a box of half-width h */
#ifndef ORA_SHELL_RHO_LIST
#define ORA_SHELL_RHO_LIST 3.0, 4.5, 7.0, 12.0
#endif
static const double ORA_SHELL_RHO[] = {ORA_SHELL_RHO_LIST};
#ifndef ORA_N_SHELL_2D
#define ORA_N_SHELL_2D 4
#endif
#ifndef ORA_SHELL_PTS_2D
#define ORA_SHELL_PTS_2D 16          /* points per square shell */
#endif
#ifndef ORA_N_SHELL_3D
#define ORA_N_SHELL_3D 4
#endif
#ifndef ORA_SHELL_GRID_3D
#define ORA_SHELL_GRID_3D 3          /* g x g points per cube face */
#endif
#ifndef ORA_ADM_EXTRA
#define ORA_ADM_EXTRA 2              /* admissible: dist >= w_t + w_s + EXTRA * min(w) */
#endif

static int ora_key_depth(int d) { return d == 2 ? ORA_KEY_DEPTH_2D : ORA_KEY_DEPTH_3D; }
static int ora_max_rank(int d) { return d == 2 ? ORA_MAX_RANK_2D : ORA_MAX_RANK_3D; }

static inline double ora_kernel(double r2) { const double t = 1.0 + r2; return 1.0 / (t * t); }

/* ===================================================================================
 * Conditional P: beta bisection on min-shifted squared distances
 * (reference src/tsne_utils.c:952-1005, driver :1022-1105)
 * =================================================================================== */
static void ora_row_P(const double *dist, int k, double perplexity, double *p)
{
    const double tol = 1e-5, target = log(perplexity);
    double dmin = dist[0] * dist[0];
    for (int j = 1; j < k; j++) { const double d2 = dist[j] * dist[j]; if (d2 < dmin) dmin = d2; }
    double beta = 1.0, lo = 0.0, hi = 0.0;
    int have_lo = 0, have_hi = 0;
    for (int it = 0; it < 200; it++) {
        double sp = 0.0, sdp = 0.0;
        for (int j = 0; j < k; j++) {
            const double dd = dist[j] * dist[j] - dmin;
            p[j] = exp(-beta * dd);
            sp += p[j];
            sdp += dd * p[j];
        }
        const double H = log(sp) + beta * sdp / sp;
        const double inv = 1.0 / sp;
        for (int j = 0; j < k; j++) p[j] *= inv;
        const double diff = H - target;
        if (fabs(diff) < tol) break;
        if (diff > 0.0) { lo = beta; have_lo = 1; beta = have_hi ? 0.5 * (beta + hi) : 2.0 * beta; }
        else            { hi = beta; have_hi = 1; beta = have_lo ? 0.5 * (beta + lo) : 0.5 * beta; }
    }
}

int ora_conditional_P(const double *dist, const int *indptr, int n, double perplexity,
                      double *P_out, int nthreads)
{
    if (n < 0 || perplexity <= 0.0) return -1;
    #pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1)
    for (int i = 0; i < n; i++) {
        const int s = indptr[i], k = indptr[i + 1] - indptr[i];
        if (k > 0) ora_row_P(dist + s, k, perplexity, P_out + s);
    }
    return 0;
}

/* Random initial embedding N(0, 1e-4^2) by Box-Muller on the C library's rand()
 * (reference src/tsne_utils.c:1130-1149): the same generator, so the same numbers. */
void ora_init_embedding(double *Y, int n, int d, unsigned int seed)
{
    srand(seed);
    const long total = (long)n * d;
    for (long i = 0; i < total; i += 2) {
        double u1 = (double)rand() / RAND_MAX;
        double u2 = (double)rand() / RAND_MAX;
        if (u1 < 1e-10) u1 = 1e-10;
        const double rad = sqrt(-2.0 * log(u1));
        Y[i] = 1e-4 * (rad * cos(2.0 * M_PI * u2));
        if (i + 1 < total) Y[i + 1] = 1e-4 * (rad * sin(2.0 * M_PI * u2));
    }
}

/* ===================================================================================
 * Exact pieces (reference src/tsne_h2pack.c:290-356, 404-491, 538-627, 1870-1895)
 * =================================================================================== */
void ora_exact_sv(const double *Y, int n, int d, double *s, double *v, int nthreads)
{
    #pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
    for (int i = 0; i < n; i++) {
        double si = 0.0, vi[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            double r2 = 0.0;
            for (int k = 0; k < d; k++) { const double df = Y[(size_t)k * n + i] - Y[(size_t)k * n + j]; r2 += df * df; }
            const double w = ora_kernel(r2);
            si += w;
            for (int k = 0; k < d; k++) vi[k] += w * Y[(size_t)k * n + j];
        }
        s[i] = si;
        for (int k = 0; k < d; k++) v[(size_t)k * n + i] = vi[k];
    }
}

void ora_exact_rows(const double *Y, int n, int d, const int *rows, int m, double *s, double *v, int nthreads)
{
    #pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads > 0 ? nthreads : 1)
    for (int r = 0; r < m; r++) {
        const int i = rows[r];
        double si = 0.0, vi[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            double r2 = 0.0;
            for (int k = 0; k < d; k++) { const double df = Y[(size_t)k * n + i] - Y[(size_t)k * n + j]; r2 += df * df; }
            const double w = ora_kernel(r2);
            si += w;
            for (int k = 0; k < d; k++) vi[k] += w * Y[(size_t)k * n + j];
        }
        s[r] = si;
        for (int k = 0; k < d; k++) v[(size_t)k * m + r] = vi[k];
    }
}

double ora_z_force(const double *Y, int n, int d, const double *s, const double *v, double *F)
{
    double t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (int i = 0; i < n; i++) {
        double yy = 0.0, yv = 0.0;
        for (int k = 0; k < d; k++) {
            const double y = Y[(size_t)k * n + i];
            yy += y * y;
            yv += y * v[(size_t)k * n + i];
        }
        t1 += s[i];
        t2 += yy * s[i];
        t3 += yv;
    }
    const double Z = t1 + 2.0 * t2 - 2.0 * t3;
    if (F != NULL) {
        const double c = 4.0 / Z;
        for (int k = 0; k < d; k++)
            for (int i = 0; i < n; i++)
                F[(size_t)k * n + i] = c * (Y[(size_t)k * n + i] * s[i] - v[(size_t)k * n + i]);
    }
    return Z;
}

void ora_attractive(int n, int d, const int *rp, const int *ci, const double *pv,
                    const double *Y, double exag, double *attr, int nthreads)
{
    const double scale = 4.0 * exag;
    #pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 0 ? nthreads : 1)
    for (int i = 0; i < n; i++) {
        double g[3] = {0.0, 0.0, 0.0};
        for (int e = rp[i]; e < rp[i + 1]; e++) {
            const int j = ci[e];
            double df[3], r2 = 0.0;
            for (int k = 0; k < d; k++) { df[k] = Y[(size_t)k * n + i] - Y[(size_t)k * n + j]; r2 += df[k] * df[k]; }
            const double q = pv[e] / (1.0 + r2);
            for (int k = 0; k < d; k++) g[k] += q * df[k];
        }
        for (int k = 0; k < d; k++) attr[(size_t)k * n + i] = scale * g[k];
    }
}

double ora_kl(int n, int d, const int *rp, const int *ci, const double *pv, const double *Y,
              double exag, double Z, int nthreads)
{
    double *row = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    #pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 0 ? nthreads : 1)
    for (int i = 0; i < n; i++) {
        double acc = 0.0;
        for (int e = rp[i]; e < rp[i + 1]; e++) {
            const int j = ci[e];
            const double p = pv[e] * exag;
            double r2 = 0.0;
            for (int k = 0; k < d; k++) { const double df = Y[(size_t)k * n + i] - Y[(size_t)k * n + j]; r2 += df * df; }
            const double q = 1.0 / ((1.0 + r2) * Z);
            if (p > 1e-12 && q > 1e-12) acc += p * log(p / q);
        }
        row[i] = acc;
    }
    double kl = 0.0;
    for (int i = 0; i < n; i++) kl += row[i];
    free(row);
    return kl;
}

/* ===================================================================================
 * H2 matrix: geometry
 *
 * Root box: centre = midpoint of the bounding box, half-width R = MIN_HALF_WIDTH * 2^k,
 * the smallest such value >= half the largest extent (an order-independent definition,
 * so host and device agree bit for bit). Every point gets integer cell coordinates
 * q = floor((y - corner) / cell) at depth L (cell = 2R / 2^L), clamped to [0, 2^L - 1],
 * and a Morton key whose top d bits are the level-1 child digit. Points are stably
 * sorted by key; a node at level l is a maximal run of points sharing the top d*l key
 * bits; it is split into its non-empty children when it holds more than leaf_size
 * points and l < L. Nodes are numbered level by level, and in key order within a level.
 * =================================================================================== */
struct ora_h2 {
    int n, d, leaf_size, L, max_level, n_node, nv;
    double corner[3], R, tol;
    uint64_t *keys;           /* tree order */
    int *perm;                /* tree position -> point */
    uint32_t *q;              /* tree order, d per point */
    int *start, *end, *level, *parent, *fchild, *nchild, *leaf;
    int64_t *ix;              /* d per node: integer box coordinates at the node's level */
    int *lvl_begin;           /* L + 2 entries */
    int *far_ptr, *far_idx, *near_ptr, *near_idx;
    int *rank, *skel_off, *U_off, *ncand;
    double *skel;             /* d per skeleton point */
    double *U;                /* per node: ncand x rank, row-major */
};

static uint64_t ora_interleave(const uint32_t *q, int d, int L)
{
    uint64_t key = 0;
    for (int b = L - 1; b >= 0; b--)
        for (int k = d - 1; k >= 0; k--)
            key = (key << 1) | ((q[k] >> b) & 1u);
    return key;
}

/* Node admissibility on integer coordinates: with w = box width in finest cells and
 * 2*centre = 2*ix*w + w, boxes t, s are well separated iff
 *   max_k |2c_t - 2c_s| >= w_t + w_s + 2 min(w_t, w_s)
 * i.e. the larger box lies outside 3x the smaller box's half-width from its centre. */
static int ora_admissible(const ora_h2 *h, int t, int s)
{
    const int64_t wt = (int64_t)1 << (h->L - h->level[t]);
    const int64_t ws = (int64_t)1 << (h->L - h->level[s]);
    int64_t dist = 0;
    for (int k = 0; k < h->d; k++) {
        const int64_t ct = 2 * h->ix[(size_t)t * h->d + k] * wt + wt;
        const int64_t cs = 2 * h->ix[(size_t)s * h->d + k] * ws + ws;
        const int64_t df = ct > cs ? ct - cs : cs - ct;
        if (df > dist) dist = df;
    }
    return dist >= wt + ws + ORA_ADM_EXTRA * (wt < ws ? wt : ws);
}

static void ora_node_center(const ora_h2 *h, int t, double *c)
{
    const double hl = h->R / (double)((int64_t)1 << h->level[t]);
    for (int k = 0; k < h->d; k++)
        c[k] = h->corner[k] + (double)(2 * h->ix[(size_t)t * h->d + k] + 1) * hl;
}

/* growable int list */
typedef struct { int *a; int n, cap; } ora_ivec;
static void iv_push(ora_ivec *v, int x)
{
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 16; v->a = (int *)realloc(v->a, sizeof(int) * v->cap); }
    v->a[v->n++] = x;
}
static int ora_int_cmp(const void *a, const void *b) { const int x = *(const int *)a, y = *(const int *)b; return (x > y) - (x < y); }

/* Stable LSD radix sort of perm (initially 0..n-1) by keys[perm[i]] over the low `bits`
 * bits: equal keys keep index order, as a comparison sort with the index as tie-break. */
static void ora_radix_sort(int *perm, const uint64_t *keys, int n, int bits)
{
    int *tmp = (int *)malloc(sizeof(int) * (size_t)n);
    uint64_t *kv = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t *kt = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    for (int i = 0; i < n; i++) kv[i] = keys[perm[i]];
    for (int shift = 0; shift < bits; shift += 8) {
        size_t cnt[257] = {0};
        for (int i = 0; i < n; i++) cnt[((kv[i] >> shift) & 255u) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (int i = 0; i < n; i++) {
            const size_t o = cnt[(kv[i] >> shift) & 255u]++;
            tmp[o] = perm[i];
            kt[o] = kv[i];
        }
        memcpy(perm, tmp, sizeof(int) * (size_t)n);
        memcpy(kv, kt, sizeof(uint64_t) * (size_t)n);
    }
    free(tmp); free(kv); free(kt);
}

static int ora_build_tree(ora_h2 *h, const double *Y, int nthreads)
{
    const int n = h->n, d = h->d, L = h->L;
    const int nth = nthreads > 0 ? nthreads : 1;
    double lo[3], hi[3];
    int bad = 0;
    for (int k = 0; k < d; k++) {
        double l0 = INFINITY, h0 = -INFINITY;
        int b0 = 0;
        #pragma omp parallel for num_threads(nth) reduction(min:l0) reduction(max:h0) reduction(|:b0)
        for (int i = 0; i < n; i++) {
            const double y = Y[(size_t)k * n + i];
            if (!isfinite(y)) { b0 = 1; continue; }
            if (y < l0) l0 = y;
            if (y > h0) h0 = y;
        }
        lo[k] = l0; hi[k] = h0; bad |= b0;
    }
    if (bad) return -1;
    double ext = 0.0, ctr[3];
    for (int k = 0; k < d; k++) {
        ctr[k] = 0.5 * (lo[k] + hi[k]);
        const double e = 0.5 * (hi[k] - lo[k]);
        if (e > ext) ext = e;
    }
    double R = ORA_MIN_HALF_WIDTH;
    while (R < ext) R *= 2.0;
    h->R = R;
    for (int k = 0; k < d; k++) h->corner[k] = ctr[k] - R;
    const double cell = 2.0 * R / (double)((int64_t)1 << L);
    const int64_t qmax = ((int64_t)1 << L) - 1;

    uint32_t *q0 = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n * d);
    uint64_t *k0 = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    #pragma omp parallel for num_threads(nth) schedule(static)
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < d; k++) {
            const double t = (Y[(size_t)k * n + i] - h->corner[k]) / cell;
            int64_t qi = (int64_t)floor(t);
            if (qi < 0) qi = 0;
            if (qi > qmax) qi = qmax;
            q0[(size_t)i * d + k] = (uint32_t)qi;
        }
        k0[i] = ora_interleave(q0 + (size_t)i * d, d, L);
    }
    for (int i = 0; i < n; i++) h->perm[i] = i;
    ora_radix_sort(h->perm, k0, n, d * L);
    #pragma omp parallel for num_threads(nth) schedule(static)
    for (int t = 0; t < n; t++) {
        const int i = h->perm[t];
        h->keys[t] = k0[i];
        for (int k = 0; k < d; k++) h->q[(size_t)t * d + k] = q0[(size_t)i * d + k];
    }
    free(q0); free(k0);

    /* level-by-level split */
    int cap = 1024, nn = 1;
    h->start = (int *)malloc(sizeof(int) * cap); h->end = (int *)malloc(sizeof(int) * cap);
    h->level = (int *)malloc(sizeof(int) * cap); h->parent = (int *)malloc(sizeof(int) * cap);
    h->start[0] = 0; h->end[0] = n; h->level[0] = 0; h->parent[0] = -1;
    h->lvl_begin = (int *)calloc((size_t)L + 2, sizeof(int));
    h->lvl_begin[0] = 0;
    int lb = 0, le = 1, l = 0;
    const int nch = 1 << d;
    while (lb < le) {
        h->lvl_begin[l + 1] = le;   /* provisional; fixed below */
        for (int t = lb; t < le; t++) {
            const int cnt = h->end[t] - h->start[t];
            if (cnt <= h->leaf_size || l >= L) continue;
            const int shift = d * (L - l - 1);
            int s = h->start[t];
            for (int c = 0; c < nch; c++) {
                int e = s;
                while (e < h->end[t] && (int)((h->keys[e] >> shift) & (uint64_t)(nch - 1)) == c) e++;
                if (e > s) {
                    if (nn == cap) {
                        cap *= 2;
                        h->start = (int *)realloc(h->start, sizeof(int) * cap);
                        h->end = (int *)realloc(h->end, sizeof(int) * cap);
                        h->level = (int *)realloc(h->level, sizeof(int) * cap);
                        h->parent = (int *)realloc(h->parent, sizeof(int) * cap);
                    }
                    h->start[nn] = s; h->end[nn] = e; h->level[nn] = l + 1; h->parent[nn] = t;
                    nn++;
                }
                s = e;
            }
        }
        lb = le; le = nn; l++;
        h->lvl_begin[l] = lb;
    }
    /* lvl_begin[l] = first node of level l, for l = 0..max_level+1 */
    h->max_level = l - 1;
    for (int ll = l; ll <= L + 1; ll++) h->lvl_begin[ll] = nn;
    h->n_node = nn;
    h->fchild = (int *)malloc(sizeof(int) * nn);
    h->nchild = (int *)calloc((size_t)nn, sizeof(int));
    h->leaf = (int *)malloc(sizeof(int) * nn);
    h->ix = (int64_t *)malloc(sizeof(int64_t) * (size_t)nn * d);
    for (int t = 0; t < nn; t++) h->fchild[t] = -1;
    for (int t = 1; t < nn; t++) {
        const int p = h->parent[t];
        if (h->fchild[p] < 0) h->fchild[p] = t;
        h->nchild[p]++;
    }
    for (int t = 0; t < nn; t++) {
        h->leaf[t] = (h->nchild[t] == 0);
        for (int k = 0; k < d; k++)
            h->ix[(size_t)t * d + k] = (int64_t)(h->q[(size_t)h->start[t] * d + k] >> (L - h->level[t]));
    }
    return 0;
}

/* ===================================================================================
 * H2 matrix: per-target interaction lists.
 *
 * Derived from the symmetric dual-tree traversal DT(a, b): a == b -> leaf: near,
 * else all child pairs; admissible -> far; both leaves -> near; one leaf -> split the
 * other; else split both. Per target t with parent p, the sources s of the calls
 * DT(t, s) are expand(N(p)), where N(p) holds the sources that did not terminate for p
 * and expand(s) = children(s) for a non-leaf s, {s} for a leaf. A leaf target keeps
 * descending into non-leaf sources until they are admissible or leaves.
 * =================================================================================== */
static void ora_classify_leaf(const ora_h2 *h, int t, int c, ora_ivec *far, ora_ivec *near)
{
    /* explicit DFS: leaf target t against the subtree of c */
    int stack[4096];
    int sp = 0;
    stack[sp++] = c;
    while (sp > 0) {
        const int s = stack[--sp];
        if (s == t) { iv_push(near, s); continue; }
        if (ora_admissible(h, t, s)) { iv_push(far, s); continue; }
        if (h->leaf[s]) { iv_push(near, s); continue; }
        for (int k = h->nchild[s] - 1; k >= 0; k--) {
            if (sp >= 4096) { fprintf(stderr, "oracle: list stack overflow\n"); abort(); }
            stack[sp++] = h->fchild[s] + k;
        }
    }
}

static void ora_build_lists(ora_h2 *h, int nthreads)
{
    const int nth = nthreads > 0 ? nthreads : 1;
    const int nn = h->n_node;
    ora_ivec *Nset = (ora_ivec *)calloc((size_t)nn, sizeof(ora_ivec));
    ora_ivec *far = (ora_ivec *)calloc((size_t)nn, sizeof(ora_ivec));
    ora_ivec *near = (ora_ivec *)calloc((size_t)nn, sizeof(ora_ivec));
    if (h->leaf[0]) iv_push(&near[0], 0);
    else iv_push(&Nset[0], 0);
    /* the targets of a level depend only on their parents' sets: one level at a time, the
     * targets of a level in parallel (each writes only its own sets) */
    for (int l = 1; l <= h->max_level; l++) {
        #pragma omp parallel for num_threads(nth) schedule(dynamic, 16)
        for (int t = h->lvl_begin[l]; t < h->lvl_begin[l + 1]; t++) {
            const int p = h->parent[t];
            for (int a = 0; a < Nset[p].n; a++) {
                const int s = Nset[p].a[a];
                const int c0 = h->leaf[s] ? s : h->fchild[s];
                const int c1 = h->leaf[s] ? s + 1 : h->fchild[s] + h->nchild[s];
                for (int c = c0; c < c1; c++) {
                    if (c == t) {
                        if (h->leaf[t]) iv_push(&near[t], t); else iv_push(&Nset[t], t);
                    } else if (ora_admissible(h, t, c)) {
                        iv_push(&far[t], c);
                    } else if (h->leaf[t]) {
                        if (h->leaf[c]) iv_push(&near[t], c);
                        else ora_classify_leaf(h, t, c, &far[t], &near[t]);
                    } else {
                        iv_push(&Nset[t], c);
                    }
                }
            }
        }
    }
    h->far_ptr = (int *)malloc(sizeof(int) * (nn + 1));
    h->near_ptr = (int *)malloc(sizeof(int) * (nn + 1));
    h->far_ptr[0] = h->near_ptr[0] = 0;
    for (int t = 0; t < nn; t++) {
        h->far_ptr[t + 1] = h->far_ptr[t] + far[t].n;
        h->near_ptr[t + 1] = h->near_ptr[t] + near[t].n;
    }
    h->far_idx = (int *)malloc(sizeof(int) * (h->far_ptr[nn] + 1));
    h->near_idx = (int *)malloc(sizeof(int) * (h->near_ptr[nn] + 1));
    #pragma omp parallel for num_threads(nth) schedule(dynamic, 64)
    for (int t = 0; t < nn; t++) {
        if (far[t].n) {
            qsort(far[t].a, far[t].n, sizeof(int), ora_int_cmp);
            memcpy(h->far_idx + h->far_ptr[t], far[t].a, sizeof(int) * far[t].n);
        }
        if (near[t].n) {
            qsort(near[t].a, near[t].n, sizeof(int), ora_int_cmp);
            memcpy(h->near_idx + h->near_ptr[t], near[t].a, sizeof(int) * near[t].n);
        }
        free(Nset[t].a); free(far[t].a); free(near[t].a);
    }
    free(Nset); free(far); free(near);
}

/* ===================================================================================
 * H2 matrix: proxy points and interpolative decomposition
 *
 * The far field of a box of half-width h is sampled by data-independent proxy points on
 * shells |y - c|_inf = rho * h (rho in ORA_SHELL_RHO). For every node at level >= 2 the
 * candidate points (a leaf's own points, or the concatenated skeletons of a node's
 * children) are compressed by an ID of A = K(candidates, proxies): column-pivoted
 * Gram-Schmidt on A^T picks r skeleton rows J with A ~= U A[J, :], stopping when the
 * largest residual row norm drops to tol times the largest initial row norm.
 * =================================================================================== */
int ora_h2_n_proxy(int d)
{
    if (d == 2) return ORA_N_SHELL_2D * ORA_SHELL_PTS_2D;
    return ORA_N_SHELL_3D * 6 * ORA_SHELL_GRID_3D * ORA_SHELL_GRID_3D;
}

void ora_h2_proxies(int d, double h, double *out)
{
    const int np = ora_h2_n_proxy(d);
    int p = 0;
    if (d == 2) {
        for (int sh = 0; sh < ORA_N_SHELL_2D; sh++) {
            const double rad = ORA_SHELL_RHO[sh] * h;
            const double off = (sh & 1) ? 0.0 : 0.5;   /* alternate shells are staggered */
            for (int k = 0; k < ORA_SHELL_PTS_2D; k++, p++) {
                const double u = ((double)k + off) * (8.0 / ORA_SHELL_PTS_2D);
                const int side = (int)(u * 0.5);
                const double a = u - 2.0 * side - 1.0;
                double x, y;
                switch (side) {
                    case 0: x = a;    y = -1.0; break;
                    case 1: x = 1.0;  y = a;    break;
                    case 2: x = -a;   y = 1.0;  break;
                    default: x = -1.0; y = -a;  break;
                }
                out[p] = x * rad;
                out[np + p] = y * rad;
            }
        }
        return;
    }
    const int g = ORA_SHELL_GRID_3D;
    for (int sh = 0; sh < ORA_N_SHELL_3D; sh++) {
        const double rad = ORA_SHELL_RHO[sh] * h;
        for (int f = 0; f < 6; f++) {
            const int ax = f >> 1;                 /* normal axis */
            const double sgn = (f & 1) ? 1.0 : -1.0;
            for (int i = 0; i < g; i++)
                for (int j = 0; j < g; j++, p++) {
                    const double a = ((double)i + 0.5) * (2.0 / g) - 1.0;
                    const double b = ((double)j + 0.5) * (2.0 / g) - 1.0;
                    double c[3];
                    c[ax] = sgn;
                    c[(ax + 1) % 3] = a;
                    c[(ax + 2) % 3] = b;
                    for (int k = 0; k < 3; k++) out[(size_t)k * np + p] = c[k] * rad;
                }
        }
    }
}

/* Dot product in four interleaved partial sums (p mod 4), joined in a fixed order: the
 * same result on every run, and a loop the compiler vectorises. */
static inline double ora_dot(const double *x, const double *y, int np)
{
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    int p = 0;
    for (; p + 4 <= np; p += 4)
        for (int k = 0; k < 4; k++) acc[k] += x[p + k] * y[p + k];
    for (; p < np; p++) acc[0] += x[p] * y[p];
    return (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

/* ID of the m x np matrix A (row-major). Returns the rank r; sel[0..r) = selected rows
 * (in pivot order); U (m x r, row-major) with A ~= U A[sel, :]. */
static int ora_id(double *A, int m, int np, double tol, int max_rank, int *sel, double *U)
{
    /* work on rows of A as vectors of length np (== columns of A^T) */
    int *piv = (int *)malloc(sizeof(int) * m);
    double *nrm = (double *)malloc(sizeof(double) * m);
    double *R = (double *)calloc((size_t)max_rank * m, sizeof(double));   /* R[k][j], j in pivoted order */
    for (int i = 0; i < m; i++) {
        piv[i] = i;
        nrm[i] = ora_dot(A + (size_t)i * np, A + (size_t)i * np, np);
    }
    double n0 = 0.0;
    for (int i = 0; i < m; i++) if (nrm[i] > n0) n0 = nrm[i];
    const double stop2 = tol * tol * n0;
    int r = 0;
    const int rmax = ORA_MIN(ORA_MIN(m, np), max_rank);
    while (r < rmax) {
        int best = r;
        for (int i = r + 1; i < m; i++) if (nrm[i] > nrm[best]) best = i;
        if (!(nrm[best] > stop2) || nrm[best] <= 0.0) break;
        if (best != r) {
            for (int p = 0; p < np; p++) {
                const double t = A[(size_t)r * np + p];
                A[(size_t)r * np + p] = A[(size_t)best * np + p];
                A[(size_t)best * np + p] = t;
            }
            { const int t = piv[r]; piv[r] = piv[best]; piv[best] = t; }
            { const double t = nrm[r]; nrm[r] = nrm[best]; nrm[best] = t; }
            for (int k = 0; k < r; k++) { const double t = R[(size_t)k * m + r]; R[(size_t)k * m + r] = R[(size_t)k * m + best]; R[(size_t)k * m + best] = t; }
        }
        const double *q = A + (size_t)r * np;
        const double rr = sqrt(ora_dot(q, q, np));
        R[(size_t)r * m + r] = rr;
        const double inv = 1.0 / rr;
        for (int p = 0; p < np; p++) A[(size_t)r * np + p] *= inv;   /* q_r */
        for (int i = r + 1; i < m; i++) {
            double *a = A + (size_t)i * np;
            const double dot = ora_dot(q, a, np);
            R[(size_t)r * m + i] = dot;
            for (int p = 0; p < np; p++) a[p] -= dot * q[p];
            nrm[i] = ora_dot(a, a, np);
        }
        r++;
    }
    if (r == 0) r = 1;   /* unreachable for this positive kernel; keep one skeleton row */
    /* T = R11^{-1} R12 (r x (m - r)); U rows: skeleton -> identity, others -> T^T */
    memset(U, 0, sizeof(double) * (size_t)m * r);
    for (int k = 0; k < r; k++) { sel[k] = piv[k]; U[(size_t)piv[k] * r + k] = 1.0; }
    double *col = (double *)malloc(sizeof(double) * r);
    for (int j = r; j < m; j++) {
        for (int k = r - 1; k >= 0; k--) {
            double acc = R[(size_t)k * m + j];
            for (int kk = k + 1; kk < r; kk++) acc -= R[(size_t)k * m + kk] * col[kk];
            col[k] = acc / R[(size_t)k * m + k];
        }
        for (int k = 0; k < r; k++) U[(size_t)piv[j] * r + k] = col[k];
    }
    free(col); free(piv); free(nrm); free(R);
    return r;
}

static void ora_build_bases(ora_h2 *h, const double *Y, int nthreads)
{
    const int nn = h->n_node, d = h->d, n = h->n;
    const int np = ora_h2_n_proxy(d), maxr = ora_max_rank(d);
    h->rank = (int *)calloc((size_t)nn, sizeof(int));
    h->ncand = (int *)calloc((size_t)nn, sizeof(int));
    h->skel_off = (int *)calloc((size_t)nn + 1, sizeof(int));
    h->U_off = (int *)calloc((size_t)nn + 1, sizeof(int));
    double **skel_n = (double **)calloc((size_t)nn, sizeof(double *));
    double **U_n = (double **)calloc((size_t)nn, sizeof(double *));
    double *prox = (double *)malloc(sizeof(double) * (size_t)np * d);
    for (int l = h->max_level; l >= ORA_MIN_ADM_LEVEL; l--) {
        const double hl = h->R / (double)((int64_t)1 << l);
        ora_h2_proxies(d, hl, prox);
        #pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads > 0 ? nthreads : 1)
        for (int t = h->lvl_begin[l]; t < h->lvl_begin[l + 1]; t++) {
            int m = 0;
            double *cand;
            if (h->leaf[t]) {
                m = h->end[t] - h->start[t];
                cand = (double *)malloc(sizeof(double) * (size_t)m * d);
                for (int a = 0; a < m; a++) {
                    const int i = h->perm[h->start[t] + a];
                    for (int k = 0; k < d; k++) cand[(size_t)a * d + k] = Y[(size_t)k * n + i];
                }
            } else {
                for (int c = h->fchild[t]; c < h->fchild[t] + h->nchild[t]; c++) m += h->rank[c];
                cand = (double *)malloc(sizeof(double) * (size_t)m * d);
                int a = 0;
                for (int c = h->fchild[t]; c < h->fchild[t] + h->nchild[t]; c++)
                    for (int k = 0; k < h->rank[c]; k++, a++)
                        memcpy(cand + (size_t)a * d, skel_n[c] + (size_t)k * d, sizeof(double) * d);
            }
            double ctr[3];
            ora_node_center(h, t, ctr);
            double *A = (double *)malloc(sizeof(double) * (size_t)m * np);
            for (int a = 0; a < m; a++)
                for (int p = 0; p < np; p++) {
                    double r2 = 0.0;
                    for (int k = 0; k < d; k++) {
                        const double df = (cand[(size_t)a * d + k] - ctr[k]) - prox[(size_t)k * np + p];
                        r2 += df * df;
                    }
                    A[(size_t)a * np + p] = ora_kernel(r2);
                }
            int *sel = (int *)malloc(sizeof(int) * (size_t)ORA_MIN(m, maxr) + sizeof(int));
            double *U = (double *)malloc(sizeof(double) * (size_t)m * ORA_MIN(ORA_MAX(m, 1), maxr));
            const int r = ora_id(A, m, np, h->tol, maxr, sel, U);
            skel_n[t] = (double *)malloc(sizeof(double) * (size_t)r * d);
            for (int k = 0; k < r; k++) memcpy(skel_n[t] + (size_t)k * d, cand + (size_t)sel[k] * d, sizeof(double) * d);
            U_n[t] = U;
            h->rank[t] = r;
            h->ncand[t] = m;
            free(A); free(sel); free(cand);
        }
    }
    for (int t = 0; t < nn; t++) {
        h->skel_off[t + 1] = h->skel_off[t] + h->rank[t];
        h->U_off[t + 1] = h->U_off[t] + h->ncand[t] * h->rank[t];
    }
    h->skel = (double *)malloc(sizeof(double) * ((size_t)h->skel_off[nn] * d + 1));
    h->U = (double *)malloc(sizeof(double) * ((size_t)h->U_off[nn] + 1));
    for (int t = 0; t < nn; t++) {
        if (h->rank[t] == 0) continue;
        memcpy(h->skel + (size_t)h->skel_off[t] * d, skel_n[t], sizeof(double) * (size_t)h->rank[t] * d);
        memcpy(h->U + h->U_off[t], U_n[t], sizeof(double) * (size_t)h->ncand[t] * h->rank[t]);
        free(skel_n[t]); free(U_n[t]);
    }
    free(skel_n); free(U_n); free(prox);
}

ora_h2 *ora_h2_build(const double *Y, int n, int d, int leaf_size, double tol, int nthreads,
                     int *status)
{
    if (status) *status = 0;
    if (n < 1 || (d != 2 && d != 3) || leaf_size < 1) return NULL;
    ora_h2 *h = (ora_h2 *)calloc(1, sizeof(ora_h2));
    h->n = n; h->d = d; h->leaf_size = leaf_size; h->L = ora_key_depth(d); h->tol = tol * ORA_ID_TOL_FACTOR;
    h->nv = d + 1;
    h->keys = (uint64_t *)malloc(sizeof(uint64_t) * n);
    h->perm = (int *)malloc(sizeof(int) * n);
    h->q = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n * d);
    if (ora_build_tree(h, Y, nthreads) != 0) { if (status) *status = -1; ora_h2_free(h); return NULL; }
    ora_build_lists(h, nthreads);
    if (h->max_level <= 2) { if (status) *status = 1; return h; }
    ora_build_bases(h, Y, nthreads);
    return h;
}

void ora_h2_free(ora_h2 *h)
{
    if (h == NULL) return;
    free(h->keys); free(h->perm); free(h->q);
    free(h->start); free(h->end); free(h->level); free(h->parent); free(h->fchild);
    free(h->nchild); free(h->leaf); free(h->ix); free(h->lvl_begin);
    free(h->far_ptr); free(h->far_idx); free(h->near_ptr); free(h->near_idx);
    free(h->rank); free(h->skel_off); free(h->U_off); free(h->ncand); free(h->skel); free(h->U);
    free(h);
}

/* ===================================================================================
 * H2 product [s | v] = K [1 | Y] with the diagonal excluded.
 *   upward   : y0[t] = U_t^T (x of a leaf's points | children's y0), levels max..2
 *   far      : same level          y1[t] += K(J_t, J_s) y0[s]
 *              s a coarser leaf     y1[t] += K(J_t, X_s) x_s
 *              t a coarser leaf     yp[X_t] += K(X_t, J_s) y0[s]
 *   near     : yp[X_t] += K(X_t, X_s) x_s, i != j
 *   downward : y1[child] += U_t[rows of child] y1[t]; leaves: yp[X_t] += U_t y1[t]
 * =================================================================================== */
void ora_h2_product(const ora_h2 *h, const double *Y, double *s, double *v, int nthreads)
{
    const int n = h->n, d = h->d, nv = h->nv, nn = h->n_node;
    const int nth = nthreads > 0 ? nthreads : 1;
    double *xt = (double *)malloc(sizeof(double) * (size_t)n * d);    /* tree-order coords */
    for (int t = 0; t < n; t++)
        for (int k = 0; k < d; k++) xt[(size_t)t * d + k] = Y[(size_t)k * n + h->perm[t]];
    const size_t nsk = (size_t)h->skel_off[nn];
    double *y0 = (double *)calloc(nsk * nv + 1, sizeof(double));
    double *y1 = (double *)calloc(nsk * nv + 1, sizeof(double));
    double *yp = (double *)calloc((size_t)n * nv, sizeof(double));

    /* upward */
    for (int l = h->max_level; l >= ORA_MIN_ADM_LEVEL; l--) {
        #pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
        for (int t = h->lvl_begin[l]; t < h->lvl_begin[l + 1]; t++) {
            const int r = h->rank[t], m = h->ncand[t];
            const double *U = h->U + h->U_off[t];
            double *o = y0 + (size_t)h->skel_off[t] * nv;
            for (int a = 0; a < m; a++) {
                double in[4];
                if (h->leaf[t]) {
                    in[0] = 1.0;
                    for (int k = 0; k < d; k++) in[1 + k] = xt[(size_t)(h->start[t] + a) * d + k];
                } else {
                    int c = h->fchild[t], aa = a;
                    while (aa >= h->rank[c]) { aa -= h->rank[c]; c++; }
                    for (int w = 0; w < nv; w++) in[w] = y0[((size_t)h->skel_off[c] + aa) * nv + w];
                }
                for (int k = 0; k < r; k++)
                    for (int w = 0; w < nv; w++) o[(size_t)k * nv + w] += U[(size_t)a * r + k] * in[w];
            }
        }
    }
    /* interactions, per target node (compressed y1, or a leaf's points) */
    #pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
    for (int t = 0; t < nn; t++) {
        for (int e = h->far_ptr[t]; e < h->far_ptr[t + 1]; e++) {
            const int src = h->far_idx[e];
            if (h->level[src] == h->level[t]) {
                for (int a = 0; a < h->rank[t]; a++) {
                    const double *ja = h->skel + ((size_t)h->skel_off[t] + a) * d;
                    for (int b = 0; b < h->rank[src]; b++) {
                        const double *jb = h->skel + ((size_t)h->skel_off[src] + b) * d;
                        double r2 = 0.0;
                        for (int k = 0; k < d; k++) { const double df = ja[k] - jb[k]; r2 += df * df; }
                        const double w = ora_kernel(r2);
                        for (int c = 0; c < nv; c++) y1[((size_t)h->skel_off[t] + a) * nv + c] += w * y0[((size_t)h->skel_off[src] + b) * nv + c];
                    }
                }
            } else if (h->level[src] < h->level[t]) {   /* coarser raw leaf source */
                for (int a = 0; a < h->rank[t]; a++) {
                    const double *ja = h->skel + ((size_t)h->skel_off[t] + a) * d;
                    for (int j = h->start[src]; j < h->end[src]; j++) {
                        double r2 = 0.0;
                        for (int k = 0; k < d; k++) { const double df = ja[k] - xt[(size_t)j * d + k]; r2 += df * df; }
                        const double w = ora_kernel(r2);
                        y1[((size_t)h->skel_off[t] + a) * nv] += w;
                        for (int k = 0; k < d; k++) y1[((size_t)h->skel_off[t] + a) * nv + 1 + k] += w * xt[(size_t)j * d + k];
                    }
                }
            } else {                                   /* t is a coarser raw leaf */
                for (int i = h->start[t]; i < h->end[t]; i++)
                    for (int b = 0; b < h->rank[src]; b++) {
                        const double *jb = h->skel + ((size_t)h->skel_off[src] + b) * d;
                        double r2 = 0.0;
                        for (int k = 0; k < d; k++) { const double df = xt[(size_t)i * d + k] - jb[k]; r2 += df * df; }
                        const double w = ora_kernel(r2);
                        for (int c = 0; c < nv; c++) yp[(size_t)i * nv + c] += w * y0[((size_t)h->skel_off[src] + b) * nv + c];
                    }
            }
        }
        for (int e = h->near_ptr[t]; e < h->near_ptr[t + 1]; e++) {
            const int src = h->near_idx[e];
            for (int i = h->start[t]; i < h->end[t]; i++)
                for (int j = h->start[src]; j < h->end[src]; j++) {
                    if (i == j) continue;
                    double r2 = 0.0;
                    for (int k = 0; k < d; k++) { const double df = xt[(size_t)i * d + k] - xt[(size_t)j * d + k]; r2 += df * df; }
                    const double w = ora_kernel(r2);
                    yp[(size_t)i * nv] += w;
                    for (int k = 0; k < d; k++) yp[(size_t)i * nv + 1 + k] += w * xt[(size_t)j * d + k];
                }
        }
    }
    /* downward */
    for (int l = ORA_MIN_ADM_LEVEL; l <= h->max_level; l++) {
        #pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
        for (int t = h->lvl_begin[l]; t < h->lvl_begin[l + 1]; t++) {
            const int r = h->rank[t], m = h->ncand[t];
            const double *U = h->U + h->U_off[t];
            const double *in = y1 + (size_t)h->skel_off[t] * nv;
            for (int a = 0; a < m; a++) {
                double acc[4] = {0, 0, 0, 0};
                for (int k = 0; k < r; k++)
                    for (int w = 0; w < nv; w++) acc[w] += U[(size_t)a * r + k] * in[(size_t)k * nv + w];
                double *o;
                if (h->leaf[t]) {
                    o = yp + (size_t)(h->start[t] + a) * nv;
                } else {
                    int c = h->fchild[t], aa = a;
                    while (aa >= h->rank[c]) { aa -= h->rank[c]; c++; }
                    o = y1 + ((size_t)h->skel_off[c] + aa) * nv;
                }
                for (int w = 0; w < nv; w++) o[w] += acc[w];
            }
        }
    }
    for (int t = 0; t < n; t++) {
        const int i = h->perm[t];
        s[i] = yp[(size_t)t * nv];
        for (int k = 0; k < d; k++) v[(size_t)k * n + i] = yp[(size_t)t * nv + 1 + k];
    }
    free(xt); free(y0); free(y1); free(yp);
}

int ora_h2_n_node(const ora_h2 *h) { return h->n_node; }
int ora_h2_max_level(const ora_h2 *h) { return h->max_level; }
int ora_h2_tree_depth(const ora_h2 *h) { return h->L; }
void ora_h2_root(const ora_h2 *h, double *corner, double *radius)
{
    for (int k = 0; k < h->d; k++) corner[k] = h->corner[k];
    *radius = h->R;
}
const int *ora_h2_perm(const ora_h2 *h) { return h->perm; }
const uint64_t *ora_h2_keys(const ora_h2 *h) { return h->keys; }
void ora_h2_nodes(const ora_h2 *h, int *start, int *end, int *level, int *parent,
                  int *first_child, int *n_child, int *is_leaf)
{
    const size_t b = sizeof(int) * (size_t)h->n_node;
    memcpy(start, h->start, b); memcpy(end, h->end, b); memcpy(level, h->level, b);
    memcpy(parent, h->parent, b); memcpy(first_child, h->fchild, b);
    memcpy(n_child, h->nchild, b); memcpy(is_leaf, h->leaf, b);
}
int ora_h2_n_far(const ora_h2 *h) { return h->far_ptr[h->n_node]; }
int ora_h2_n_near(const ora_h2 *h) { return h->near_ptr[h->n_node]; }
void ora_h2_lists(const ora_h2 *h, int *far_ptr, int *far_idx, int *near_ptr, int *near_idx)
{
    memcpy(far_ptr, h->far_ptr, sizeof(int) * (h->n_node + 1));
    memcpy(near_ptr, h->near_ptr, sizeof(int) * (h->n_node + 1));
    memcpy(far_idx, h->far_idx, sizeof(int) * h->far_ptr[h->n_node]);
    memcpy(near_idx, h->near_idx, sizeof(int) * h->near_ptr[h->n_node]);
}
void ora_h2_ranks(const ora_h2 *h, int *rank)
{
    if (h->rank) memcpy(rank, h->rank, sizeof(int) * h->n_node);
    else memset(rank, 0, sizeof(int) * h->n_node);
}
void ora_h2_bases(const ora_h2 *h, int *ncand, int *skel_off, int *U_off)
{
    const int nn = h->n_node;
    if (h->rank == NULL) {
        memset(ncand, 0, sizeof(int) * nn);
        memset(skel_off, 0, sizeof(int) * (nn + 1));
        memset(U_off, 0, sizeof(int) * (nn + 1));
        return;
    }
    memcpy(ncand, h->ncand, sizeof(int) * nn);
    memcpy(skel_off, h->skel_off, sizeof(int) * (nn + 1));
    memcpy(U_off, h->U_off, sizeof(int) * (nn + 1));
}
const double *ora_h2_U(const ora_h2 *h) { return h->U; }
const double *ora_h2_skel(const ora_h2 *h) { return h->skel; }

/* ===================================================================================
 * Whole optimisation phase (reference src/tsne_h2pack.c:1652-2102, sklearn mode)
 * =================================================================================== */
ora_state *ora_state_create(int n, int d, const int *rp, const int *ci, const double *pv,
                            const double *Y0)
{
    ora_state *st = (ora_state *)calloc(1, sizeof(ora_state));
    st->n = n; st->d = d;
    const int nnz = rp[n];
    st->rp = (int *)malloc(sizeof(int) * (n + 1)); memcpy(st->rp, rp, sizeof(int) * (n + 1));
    st->ci = (int *)malloc(sizeof(int) * (nnz + 1)); memcpy(st->ci, ci, sizeof(int) * nnz);
    st->pv = (double *)malloc(sizeof(double) * (nnz + 1)); memcpy(st->pv, pv, sizeof(double) * nnz);
    const size_t dn = (size_t)n * d;
    st->Y = (double *)malloc(sizeof(double) * dn); memcpy(st->Y, Y0, sizeof(double) * dn);
    st->uY = (double *)calloc(dn, sizeof(double));
    st->gains = (double *)malloc(sizeof(double) * dn);
    for (size_t i = 0; i < dn; i++) st->gains[i] = 1.0;
    st->rep = (double *)calloc(dn, sizeof(double));
    return st;
}

void ora_state_free(ora_state *st)
{
    if (st == NULL) return;
    free(st->rp); free(st->ci); free(st->pv); free(st->Y); free(st->uY); free(st->gains);
    free(st->rep); free(st->point_order); ora_h2_free(st->h2);
    free(st);
}

/* new point k = old point ord[k] (reference src/tsne_reorder.c:112-167): P rows and
 * columns renumbered, every row sorted by its new column numbers */
int ora_renumber(ora_state *st, const int *ord)
{
    const int n = st->n, d = st->d, nnz = st->rp[n];
    int *inv = (int *)malloc(sizeof(int) * n);
    for (int k = 0; k < n; k++) inv[ord[k]] = k;
    int *rp = (int *)malloc(sizeof(int) * (n + 1));
    int *ci = (int *)malloc(sizeof(int) * (nnz + 1));
    double *pv = (double *)malloc(sizeof(double) * (nnz + 1));
    rp[0] = 0;
    for (int k = 0; k < n; k++) rp[k + 1] = rp[k] + (st->rp[ord[k] + 1] - st->rp[ord[k]]);
    for (int k = 0; k < n; k++) {
        const int i = ord[k], b = rp[k], len = rp[k + 1] - rp[k];
        for (int e = 0; e < len; e++) { ci[b + e] = inv[st->ci[st->rp[i] + e]]; pv[b + e] = st->pv[st->rp[i] + e]; }
        for (int a = 1; a < len; a++) {   /* insertion sort by new column */
            const int c = ci[b + a]; const double p = pv[b + a];
            int z = a - 1;
            while (z >= 0 && ci[b + z] > c) { ci[b + z + 1] = ci[b + z]; pv[b + z + 1] = pv[b + z]; z--; }
            ci[b + z + 1] = c; pv[b + z + 1] = p;
        }
    }
    free(st->rp); free(st->ci); free(st->pv);
    st->rp = rp; st->ci = ci; st->pv = pv;
    double *tmp = (double *)malloc(sizeof(double) * n);
    double *arrs[4] = {st->Y, st->uY, st->gains, st->rep_valid ? st->rep : NULL};
    for (int a = 0; a < 4; a++) {
        if (arrs[a] == NULL) continue;
        for (int k = 0; k < d; k++) {
            double *col = arrs[a] + (size_t)k * n;
            for (int j = 0; j < n; j++) tmp[j] = col[ord[j]];
            memcpy(col, tmp, sizeof(double) * n);
        }
    }
    int *po = (int *)malloc(sizeof(int) * n);
    for (int k = 0; k < n; k++) po[k] = st->point_order ? st->point_order[ord[k]] : ord[k];
    free(st->point_order);
    st->point_order = po;
    free(tmp); free(inv);
    return 0;
}

static int ora_rebuild(ora_state *st, const ora_run_params *p)
{
    ora_h2_free(st->h2);
    st->h2 = NULL;
    int status = 0;
    ora_h2 *h = ora_h2_build(st->Y, st->n, st->d, p->h2_leaf_size, p->h2_tol > 0 ? p->h2_tol : 1e-6,
                             p->nthreads, &status);
    if (status < 0 || h == NULL) { ora_h2_free(h); return -1; }
    if (status == 1) { ora_h2_free(h); return 0; }   /* shallow: exact path */
    st->h2 = h;
    return 0;
}

int ora_run(ora_state *st, const ora_run_params *p)
{
    const int n = st->n, d = st->d;
    const size_t dn = (size_t)n * d;
    const int nth = p->nthreads > 0 ? p->nthreads : 1;
    const int rep_reuse = p->rep_reuse && n >= 2000;
    static const int reorder_iters[6] = {30, 100, 250, 400, 600, 800};
    const int n_reorder = p->reorder ? 6 : 0;
    double *grad = (double *)malloc(sizeof(double) * dn);
    double *s = (double *)malloc(sizeof(double) * n), *v = (double *)malloc(sizeof(double) * dn);
    double *F = (double *)malloc(sizeof(double) * dn);
    const int never_h2 = !p->use_h2 || p->h2_rebuild_freq > 100000;
    const int it0 = p->iter_begin, it1 = (p->iter_end > 0 ? p->iter_end : p->n_iter);
    if (it0 == 0 && n >= 2000 && !never_h2 && st->h2 == NULL) {
        if (ora_rebuild(st, p) != 0) return -1;     /* tsne_init_with_P builds the first H2 */
    }
    int ret = 0;
    for (int iter = it0; iter < it1; iter++) {
        const double mom = iter >= p->momentum_switch_iter ? p->momentum : p->initial_momentum;
        const double exag = iter < p->early_exag_iter ? p->early_exag : 1.0;
        const int freq = p->h2_rebuild_freq > 0 ? p->h2_rebuild_freq : 10;
        int eff = iter < 20 ? 1 : freq;
        if (iter >= 20 && iter < p->early_exag_iter && rep_reuse && p->h2_rebuild_freq_early > eff)
            eff = p->h2_rebuild_freq_early;
        int rebuilt = (iter == 0);
        if (n >= 2000 && iter > 0 && iter % eff == 0 && !never_h2) {
            if (st->next_reorder < n_reorder && iter >= reorder_iters[st->next_reorder] && st->h2 != NULL) {
                while (st->next_reorder < n_reorder && iter >= reorder_iters[st->next_reorder]) st->next_reorder++;
                int *ord = (int *)malloc(sizeof(int) * n);
                memcpy(ord, st->h2->perm, sizeof(int) * n);
                ora_renumber(st, ord);
                free(ord);
            }
            if (ora_rebuild(st, p) != 0) { ret = -1; break; }
            rebuilt = 1;
            st->n_rebuild++;
        }
        ora_attractive(n, d, st->rp, st->ci, st->pv, st->Y, exag, grad, nth);
        double Z;
        if (rep_reuse && !rebuilt && st->rep_valid) {
            for (size_t i = 0; i < dn; i++) grad[i] -= st->rep[i];
            Z = st->rep_Z;
        } else {
            const int use = !never_h2 && st->h2 != NULL;
            if (use) ora_h2_product(st->h2, st->Y, s, v, nth);
            else ora_exact_sv(st->Y, n, d, s, v, nth);
            Z = ora_z_force(st->Y, n, d, s, v, F);
            if (use && (!(Z > 0.0) || !isfinite(Z))) {
                Z = 1.0;   /* the H2 path reports and skips the force (tsne_h2pack.c:604-611) */
            } else {
                for (size_t i = 0; i < dn; i++) grad[i] -= F[i];
                if (use && rep_reuse) { memcpy(st->rep, F, sizeof(double) * dn); st->rep_Z = Z; st->rep_valid = 1; }
            }
        }
        if (iter == p->n_iter - 1)
            st->kl = ora_kl(n, d, st->rp, st->ci, st->pv, st->Y, exag, Z, nth);
        for (size_t i = 0; i < dn; i++) {
            const int flip = st->uY[i] * grad[i] < 0.0;
            double g = flip ? st->gains[i] + 0.2 : st->gains[i] * 0.8;
            if (g < 0.01) g = 0.01;
            st->gains[i] = g;
            const double gr = grad[i] * g;
            st->uY[i] = mom * st->uY[i] - p->learning_rate * gr;
            st->Y[i] += st->uY[i];
        }
        for (int k = 0; k < d; k++) {
            double m = 0.0;
            for (int i = 0; i < n; i++) m += st->Y[(size_t)k * n + i];
            m /= n;
            for (int i = 0; i < n; i++) st->Y[(size_t)k * n + i] -= m;
        }
    }
    free(grad); free(s); free(v); free(F);
    return ret;
}

void ora_get_embedding(const ora_state *st, double *Y_out)
{
    const int n = st->n;
    for (int k = 0; k < st->d; k++)
        for (int j = 0; j < n; j++) {
            const int dst = st->point_order ? st->point_order[j] : j;
            Y_out[(size_t)k * n + dst] = st->Y[(size_t)k * n + j];
        }
}
