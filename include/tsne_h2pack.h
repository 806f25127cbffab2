/*
 * tsne_h2pack.h -- C ABI of the B200 t-SNE optimisation engine.
 *
 * Drop-in for the reference's C ABI (include/tsne_h2pack.h of xinxing02/tsne-h2pack-python):
 * the same types, layouts and entry points, bound by the reference's own Python loader
 * (tsne_h2pack/_backend.py:345-448). Every entry point below names the reference
 * declaration it replaces. Plain C types only; all device state stays behind the opaque
 * workspace.
 *
 * Differences a caller can observe:
 *   - tsne_workspace_t is opaque (the reference's Python treats it as opaque too,
 *     _backend.py:123-127); H2Pack_p is an opaque handle to this engine's H2 matrix.
 *   - num_threads only sets the host threads of compute_P_from_knn_distances' host
 *     side; the optimisation runs on the current CUDA device.
 *   - Diagnostics go to stdout/stderr as in the reference; errors are reported through
 *     the same NULL / non-zero returns.
 */
#ifndef TSNE_H2PACK_B200_H
#define TSNE_H2PACK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* exported entry points (the library is built with hidden default visibility) */
#ifndef TSNE_API
#define TSNE_API __attribute__((visibility("default")))
#endif

#ifndef DTYPE
#define DTYPE double
#endif

/* CSR matrix, int32 indices, double values (reference include/tsne_h2pack.h:17-24) */
typedef struct {
    int n_rows;
    int n_cols;
    int nnz;
    int *row_ptr;
    int *col_idx;
    DTYPE *values;
} sparse_matrix_t;

/* Run parameters, 160 bytes, field for field the reference's layout
 * (reference include/tsne_h2pack.h:27-85; mirrored by _backend.py:51-96). */
typedef struct {
    int n_iter;
    DTYPE perplexity;
    DTYPE learning_rate;          /* < 0: max(N / 12, 200) */
    DTYPE momentum;
    DTYPE initial_momentum;
    int momentum_switch_iter;
    DTYPE early_exag;
    int early_exag_iter;
    int use_vptree;               /* legacy k-NN selector of tsne_init; ignored */
    DTYPE h2_tol;
    int h2_rebuild_freq;
    int h2pack_print_level;
    int init_method;              /* 0: random N(0, 1e-4^2); 1: copy init_Y */
    int random_seed;
    int verbose;
    int print_freq;
    int enable_early_stopping;
    DTYPE convergence_tol;
    int convergence_patience;
    int min_iter;
    int sklearn_compatible;
    int enable_profiling;
    char *profiling_output_file;
    int num_threads;
    int h2_leaf_size;
    int h2_rebuild_freq_early;
    const DTYPE *init_Y;          /* low_dim x n_point, read only inside tsne_init* */
} tsne_params_t;

/* Per-iteration stage times in seconds (reference include/tsne_h2pack.h:88-99) */
typedef struct {
    double *knn_time;
    double *p_construction_time;
    double *p_matvec_time;
    double *h2_rebuild_time;
    double *h2_matvec_s_time;
    double *h2_matvec_v_time;
    double *z_computation_time;
    double *gradient_time;
    double *other_time;
} profiling_data_t;

typedef struct tsne_workspace tsne_workspace_t;      /* opaque */
typedef struct tsne_h2_matrix *H2Pack_p;             /* opaque H2 matrix handle */

/* ---- public API (reference include/tsne_h2pack.h:163-263) ---- */

/* reference tsne_h2pack.h:167 / src/tsne_h2pack.c:56-104 */
TSNE_API tsne_params_t tsne_create_default_params(void);

/* reference tsne_h2pack.h:178; builds P from X with a brute-force k-NN (k = 3 * perplexity)
 * on the device, then behaves like tsne_init_with_P */
TSNE_API tsne_workspace_t *tsne_init(const DTYPE *X, int n_point, int pt_dim, int low_dim,
                            const tsne_params_t *params);

/* reference tsne_h2pack.h:196 / src/tsne_h2pack.c:1356-1547. Takes ownership of P (which
 * must come from sparse_matrix_create); uploads P and the initial embedding and builds
 * the first H2 matrix on the device. NULL on bad low_dim or P shape, or a failed build;
 * also NULL, with P left to the caller, for row pointers that do not start at 0 or that
 * decrease, and for a column index outside [0, n_point) (checked on the host). */
TSNE_API tsne_workspace_t *tsne_init_with_P(const DTYPE *X, int n_point, int pt_dim, int low_dim,
                                   const tsne_params_t *params, sparse_matrix_t *P);

/* reference tsne_h2pack.h:210 / src/tsne_h2pack.c:1652-2102. 0 on success, -1 on a failed
 * H2 rebuild (e.g. non-finite coordinates) or a device error. */
TSNE_API int tsne_run(tsne_workspace_t *workspace);

/* reference tsne_h2pack.h:217 / src/tsne_h2pack.c:2108-2122: low_dim x n_point, caller's order */
TSNE_API void tsne_get_embedding(tsne_workspace_t *workspace, DTYPE *Y_out);

/* reference tsne_h2pack.h:223 / src/tsne_h2pack.c:2128-2184 */
TSNE_API void tsne_destroy(tsne_workspace_t *workspace);

/* reference tsne_h2pack.h:236 / src/tsne_h2pack.c:2190-2212 */
TSNE_API int tsne_fit_transform(const DTYPE *X, int n_point, int pt_dim, int low_dim,
                       const tsne_params_t *params, DTYPE *Y_out);

/* reference tsne_h2pack.h:256 / src/tsne_h2pack.c:2214-2236 */
TSNE_API int tsne_fit_transform_with_P(const DTYPE *X, int n_point, int pt_dim, int low_dim,
                              const tsne_params_t *params, sparse_matrix_t *P, DTYPE *Y_out);

/* ---- P built on the device (no counterpart entry point in the reference: these do the
 * reference's calibration, src/tsne_utils.c:1022-1105, and the symmetrisation and
 * normalisation its Python layer does on the host, tsne_h2pack/_backend.py:709-718) ---- */

/* Symmetric normalised P = (P_c + P_c^T) / sum from a k-NN distance graph, P_c the
 * conditional probabilities at `perplexity`: every step on the device. The graph's rows must
 * be sorted by column, without self entries (as _backend.prepare_knn_graph leaves them);
 * entries whose symmetric sum is exactly zero are dropped, as scipy's addition drops them.
 * Entry values equal the reference's host computation bit for bit except for the total
 * (a fixed-order device sum instead of numpy's). Returns a C-allocated matrix (free with
 * sparse_matrix_destroy); NULL on bad input (reported on stderr) or a device error. */
TSNE_API sparse_matrix_t *tsne_joint_P_from_knn_distances(const DTYPE *knn_distances, const int *knn_indices,
                                                          const int *knn_indptr, int n_samples, int nnz,
                                                          DTYPE perplexity);

/* tsne_init_with_P with P built on the device from a k-NN distance graph, as
 * tsne_joint_P_from_knn_distances does at params->perplexity: P never visits the host. The
 * graph arrays are read during the call only. NULL on bad input or a device error. */
TSNE_API tsne_workspace_t *tsne_init_with_knn_distances(const DTYPE *X, int n_point, int pt_dim, int low_dim,
                                                        const tsne_params_t *params, const DTYPE *knn_distances,
                                                        const int *knn_indices, const int *knn_indptr, int nnz);

/* Exact k nearest neighbours (Euclidean) of every row of X (n_samples x n_features, row-major
 * float32, host) on the device: the graph the reference's Python front ends build on the host
 * (tsne_h2pack/_knn_methods.py:71-119, knn_method='exact'; no counterpart entry point in its C
 * ABI). indices and distances (host, n_samples x k each) receive each row's k neighbours
 * sorted by index, self excluded, distances not squared (single precision; ties of distance
 * keep the smaller index). With at most 64 features and k <= 128 the distances come from the
 * tensor cores (FP16 high and low parts of the centred coordinates, FP32 accumulation) and the
 * best k + 16 of each row are re-ranked by exact FP32 distances; otherwise from an FP32 scan on
 * the CUDA cores. 1 <= k <= min(n_samples - 1, 256), n_samples <= 2^24. Returns 0, -1 on bad
 * arguments, -2 on a device error (a bounded wait of the tensor-core scan that gave up
 * included). */
TSNE_API int tsne_knn_graph(const float *X, int n_samples, int n_features, int k, int *indices, float *distances);

/* init='pca' on the device (reference tsne_h2pack/manifold.py:399-416, there scikit-learn's
 * randomized PCA on the host; no counterpart entry point in its C ABI). X: n_samples x
 * n_features, row-major FP64 (host). Y_out (host, n_samples x n_components, row-major) receives
 * the exact principal-component projection of the centred data (each component's
 * largest-magnitude loading positive, scikit-learn's sign rule) scaled to a first-coordinate
 * standard deviation of 1e-4. 0 on success; -1 bad arguments (n_components above
 * min(n_samples, n_features), n_features > 4096); -2 device error; -3 non-finite data or no
 * variance along the first component. */
TSNE_API int tsne_pca_init(const DTYPE *X, int n_samples, int n_features, int n_components, DTYPE *Y_out);

/* Quality scores of an embedding (reference benchmarks/quality.py:56-90; no counterpart in its
 * C ABI), on the device. Y: low_dim x n_point (the layout of tsne_get_embedding); P: a fixed
 * joint P (host CSR). kl receives sum p log p + sum p log(1 + d^2) + log Z with Z the exact sum
 * of (1 + d^2)^-1 over all ordered pairs (the reference estimates Z from anchor rows).
 * knn_preservation receives the mean fraction of each query's k input-space neighbours
 * (hd_neighbors, n_eval x k, row per query) found among its k nearest points in the embedding.
 * 1 <= k <= 128. 0 on success, -1 bad arguments, -2 device error. */
TSNE_API int tsne_score_embedding(const DTYPE *Y, int n_point, int low_dim, const sparse_matrix_t *P,
                                  const int *queries, int n_eval, const int *hd_neighbors, int k,
                                  DTYPE *knn_preservation, DTYPE *kl);

/* ---- sparse matrix utilities (reference tsne_h2pack.h:269-295, src/tsne_utils.c:18-60) ---- */
TSNE_API sparse_matrix_t *sparse_matrix_create(int n_rows, int n_cols, int nnz);
TSNE_API void sparse_matrix_destroy(sparse_matrix_t *mat);
TSNE_API void sparse_matvec(const sparse_matrix_t *A, const DTYPE *x, DTYPE *y);

/* ---- internal functions exposed for testing (reference tsne_h2pack.h:301-446) ---- */

/* reference tsne_h2pack.h:312 / src/tsne_utils.c:828-933 (device brute-force k-NN here) */
TSNE_API sparse_matrix_t *compute_sparse_P(const DTYPE *X, int n_point, int pt_dim, DTYPE perplexity,
                                  int use_vptree, int verbose, int num_threads);

/* reference tsne_h2pack.h:338 / src/tsne_utils.c:1022-1105: conditional P_j|i by FP64 beta
 * bisection on the device; returns a C-allocated matrix (free with sparse_matrix_destroy) */
TSNE_API sparse_matrix_t *compute_P_from_knn_distances(const DTYPE *knn_distances, const int *knn_indices,
                                              const int *knn_indptr, int n_samples, int nnz,
                                              DTYPE perplexity, int num_threads);

/* reference tsne_h2pack.h:358 / src/tsne_utils.c:1111-1150 (host; the same generator) */
TSNE_API void initialize_embedding(DTYPE *Y, int n_point, int low_dim, int method, const DTYPE *Y0,
                          unsigned int seed);

/* reference tsne_h2pack.h:377 / src/tsne_h2pack.c:290-356: grad += attractive force,
 * host arrays in, host array out (computed on the device) */
TSNE_API void compute_attractive_forces(const sparse_matrix_t *P, const DTYPE *Y, int low_dim, int n_point,
                               DTYPE early_exag, DTYPE *grad, int num_threads);

/* reference tsne_h2pack.h:398 / src/tsne_h2pack.c:389-630: grad -= repulsive force of the
 * workspace's current H2 matrix (exact O(N^2) sums when h2pack_W is NULL); returns Z */
TSNE_API DTYPE compute_repulsive_forces_h2pack(H2Pack_p h2pack_W, const DTYPE *Y, int low_dim, int n_point,
                                      tsne_workspace_t *workspace, DTYPE *grad, int iter);

/* reference tsne_h2pack.h:413 / src/tsne_h2pack.c:772-953: rebuild the workspace's H2 matrix
 * for its current embedding; 0 on success, -1 on failure */
TSNE_API int update_h2_matrix(tsne_workspace_t *workspace, int force_rebuild);

/* reference tsne_h2pack.h:420 / src/tsne_h2pack.c:2243-2247: last KL divergence */
TSNE_API DTYPE compute_kl_divergence(tsne_workspace_t *workspace);

/* reference tsne_h2pack.h:427 / src/tsne_h2pack.c:1553-1628: same CSV schema */
TSNE_API void tsne_write_profiling_data(tsne_workspace_t *workspace, const char *filename);

/* reference tsne_h2pack.h:436 / src/tsne_h2pack.c:1634-1646 */
TSNE_API void tsne_set_init_profiling_times(tsne_workspace_t *workspace, double knn_time,
                                   double p_construction_time);

/* reference tsne_h2pack.h:441 / src/tsne_h2_matmul.c:225-452: Y[c] = W X[c] for nv columns
 * (host arrays of length n, the caller's order). Returns -1 if unsupported. */
TSNE_API int tsne_h2_matmul(H2Pack_p h2, const int nv, const DTYPE *const *X, DTYPE *const *Y, void **ws);
TSNE_API void tsne_h2_matmul_free(void **ws);

/* reference tsne_h2pack.h:446 / src/tsne_reorder.c:112-167: new point k = old point ord[k] */
TSNE_API int tsne_renumber_points(tsne_workspace_t *workspace, const int *ord, int num_threads);

/* ---- engine inspection (no reference counterpart: lets host tests compare the device
 * H2 matrix with the oracle; all arrays are host arrays) ---- */

/* The workspace's current H2 matrix, or NULL when the exact path is in use */
TSNE_API H2Pack_p tsne_get_h2_matrix(tsne_workspace_t *workspace);
/* n_node, max_level, total far entries, total near entries */
TSNE_API int tsne_h2_info(H2Pack_p h2, int *n_node, int *max_level, int *n_far, int *n_near);
/* tree position -> current point number (n), root corner (low_dim) and half-width */
TSNE_API int tsne_h2_get_tree(H2Pack_p h2, int *perm, double *corner, double *radius);
/* node table (n_node each): start, end, level, parent, first child, child count, leaf flag */
TSNE_API int tsne_h2_get_nodes(H2Pack_p h2, int *start, int *end, int *level, int *parent,
                      int *first_child, int *n_child, int *is_leaf);
/* per-target CSR of far and near partners (n_node + 1 pointers; partners ascending) */
TSNE_API int tsne_h2_get_lists(H2Pack_p h2, int *far_ptr, int *far_idx, int *near_ptr, int *near_idx);
/* per-node skeleton rank (n_node) */
TSNE_API int tsne_h2_get_ranks(H2Pack_p h2, int *rank);
/* the bases: node t's U rows are row_off[t] .. row_off[t] + m_t - 1 (m_t = its leaf's points,
 * or its children's ranks summed, in child order), max_rank floats each, row-major (columns
 * past the node's rank unused); skel: n_node x max_rank skeleton points of low_dim floats.
 * row_off has n_node + 1 entries, U n_rows x max_rank. With U == NULL only *n_rows and
 * *max_rank are set. 0 on success, -1 without a built matrix. */
TSNE_API int tsne_h2_get_bases(H2Pack_p h2, int *n_rows, int *max_rank, long long *row_off, float *U,
                               float *skel);
/* Failure-path test of the dependency-ordered H2 launches (no counterpart in the reference):
 * one device wait, bounded to max_polls polls (1 .. 2^22, about 0.1 us each), on a tree-node
 * flag that nothing publishes. The wait gives up and records the failure in the matrix, as a
 * real wait that ran out would; the next rebuild reports it, so the workspace's next
 * tsne_run / tsne_run_range returns -1. Other workspaces are unaffected. Returns 1 when the
 * failure was recorded, -1 without a built matrix, with max_polls out of range or on a CUDA
 * error. */
TSNE_API int tsne_h2_probe_dependency_timeout(H2Pack_p h2, int max_polls);
/* Current device state in the caller's order: Y (low_dim x n_point), and the repulsive
 * force of the last rebuild (low_dim x n_point, NULL to skip) */
TSNE_API int tsne_get_state(tsne_workspace_t *workspace, DTYPE *Y_out, DTYPE *rep_out, DTYPE *rep_Z);
/* Replace the embedding (low_dim x n_point, caller's order) and reset gains / velocity */
TSNE_API int tsne_set_embedding(tsne_workspace_t *workspace, const DTYPE *Y_in);
/* Run iterations [iter_begin, iter_end) of the schedule (tsne_run = [0, n_iter)) */
TSNE_API int tsne_run_range(tsne_workspace_t *workspace, int iter_begin, int iter_end);
/* Device time of the last tsne_run / tsne_run_range (CUDA events on the workspace's stream,
 * ms) and, when the environment sets TSNE_KERNEL_TIMING=1, the summed device time and count of
 * its attractive-pass launches */
TSNE_API int tsne_get_timing(tsne_workspace_t *workspace, double *run_ms, double *attr_ms, int *attr_launches);
/* Number of H2 rebuilds and kernel launches issued by the last tsne_run / tsne_run_range */
TSNE_API int tsne_get_run_stats(tsne_workspace_t *workspace, int *n_rebuild, long long *n_launch);

/* ---- no-allocation entry point (no counterpart in the reference) ----
 *
 * Exact repulsive force of an embedding, for callers that must not allocate device memory
 * (a process serving under a fixed, pre-carved memory budget, code where the implicit
 * device synchronisation of an allocation is not acceptable, or hosts with their own
 * allocator). Y (input) and F (output) are device arrays of n_point x low_dim floats,
 * point-major (x0, y0[, z0], x1, ...); Z is a device double receiving the normalisation.
 * F must not overlap Y (an overlapping call is rejected with -1).
 * F_i = (4 / Z) sum_{j != i} (1 + |y_i - y_j|^2)^-2 (y_i - y_j) and
 * Z = sum_{i != j} (1 + |y_i - y_j|^2)^-1: the reference's exact force and Z
 * (src/tsne_h2pack.c:404-491), summed pair by pair instead of through its identity
 * Z = sum s + 2 sum |y|^2 s - 2 sum y.v, which loses digits in single precision when the
 * embedding is wide. If Z is not positive and finite (Y holds a NaN or an infinity), *Z
 * receives it and F is set to zero: check *Z after the call when Y may be bad.
 *
 * The scratch lives in a file-scope __device__ array sized for at most 65536 points (about
 * 1 MB, held by every device that loads the library until the process exits); larger
 * n_point is rejected with -1. The first call on a device looks up that array's device
 * address (once per device, with the device current), so make the first call on each device
 * before any stream capture. All calls on a device share the array: calls that overlap on
 * the GPU race on it. stream: a cudaStream_t, or NULL for the legacy default stream.
 * Returns 0 on success, -1 on bad arguments, -2 on a CUDA error. Asynchronous on `stream`. */
TSNE_API int tsne_exact_repulsion_static(const float *Y, int n_point, int low_dim, float *F, double *Z,
                                         void *stream);

/* Measured compute ceilings of the current device (no counterpart in the reference), for the
 * roofline of the non-tensor kernels: FP32 FMA throughput of scalar FFMA and of the paired
 * fma.rn.f32x2 form (TFLOP/s, 2 flops per FMA and lane), and MUFU reciprocals (10^12 per
 * second). Each is the best of five timed launches of a register-resident loop over every SM.
 * 0 on success, -2 on a CUDA error. */
TSNE_API int tsne_measure_compute_peaks(double *ffma_tflops, double *ffma2_tflops, double *rcp_tops);

/* Device memory: workspaces take their buffers from the current device's stream-ordered
 * memory pool, which keeps freed memory for the next workspace (no counterpart in the
 * reference, which allocates on the host). This returns the pool's unused memory to the
 * driver; 0 on success. */
TSNE_API int tsne_release_cached_memory(void);

/* ---- Batched and served jobs (no counterpart in the reference, which runs one embedding
 * per call). A server runs many independent optimisations on the current device: jobs queue
 * in arrival order and start when fewer than max_concurrent run and their device memory
 * estimate fits under hbm_budget_gb next to the running jobs' (a job larger than the budget
 * runs alone). Each job is a workspace with its own stream, so running jobs overlap on the
 * GPU; a job's result is the one it gets alone, bit for bit. */
typedef struct tsne_server tsne_server_t;

typedef struct {
    int job;            /* id returned by tsne_server_submit */
    int status;         /* 0: done; -1: failed or cancelled */
    int n_point, low_dim;
    double latency_s;   /* submission to completion */
    double queue_s;     /* submission to start */
    double run_s;       /* tsne_init_with_P + tsne_run + read-back */
    double kl;          /* final KL divergence */
    double start_s, end_s;   /* steady-clock times of start and completion */
} tsne_job_info_t;

/* NULL on bad arguments or when no CUDA device is current. */
TSNE_API tsne_server_t *tsne_server_create(int max_concurrent, double hbm_budget_gb);
/* Queues one job; takes ownership of P (from sparse_matrix_create) as tsne_init_with_P does,
 * copies params and init_Y. Returns the job id (>= 0) or -1 on bad arguments. */
TSNE_API int tsne_server_submit(tsne_server_t *s, int n_point, int low_dim, const tsne_params_t *params,
                                sparse_matrix_t *P);
/* Blocks until the job ends; Y_out (low_dim x n_point, may be NULL) and info (may be NULL)
 * receive the result, which the server then releases (a second wait returns the info and -1).
 * Returns 0, or -1 when the job failed, was cancelled or was already collected. */
TSNE_API int tsne_server_wait(tsne_server_t *s, int job, DTYPE *Y_out, tsne_job_info_t *info);
/* Jobs queued or running. */
TSNE_API int tsne_server_pending(tsne_server_t *s);
/* Cancels the jobs that have not started, waits for the running ones, frees everything. */
TSNE_API void tsne_server_destroy(tsne_server_t *s);

#ifdef __cplusplus
}
#endif
#endif
