// Launchers of the engine's CUDA kernels (host-callable, stream-ordered, no syncs).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace tsne {

// Device-resident scalars shared by the kernels of one workspace.
struct DevScalars {
    double Z;           // normalisation of the current iteration's repulsion
    double rep_Z;       // Z that goes with the stored repulsive force
    double kl;          // last KL divergence
    double mean[3];     // last centring offset
    double max_change;  // convergence check: largest per-point displacement
    int force_ok;       // the repulsion computed this iteration was applied
    int rep_valid;      // the stored repulsive force is usable
    int bad_z;          // Z <= 0 or non-finite on the H2 path
    int pad0;
};

// Result of an H2 tree build read back by the host (one sync per rebuild).
struct TreeInfo {
    int nonfinite;      // Y held NaN / Inf: the rebuild fails
    int n_node;
    int max_level;
    int max_leaf;       // largest leaf population
    int n_level_nodes[32];
    int level_begin[33];
    int nset_overflow;
    int pad[3];
    double corner[3];
    double radius;
};

// ---- dense per-point kernels (dense.cu) ----
template <int D>
void launch_attr_update(cudaStream_t st, int n, const int *rp, const int *col, const float *val,
                        const void *Y, void *Ynext, void *uY, void *gains, const void *rep,
                        const int *rep_flag, float exag4, float mom, float lr, double *partials);
// the attractive sums alone (into attr), and the update from them (same bits as the fused step)
template <int D>
void launch_attr_grad(cudaStream_t st, int n, const int *rp, const int *col, const float *val, const void *Y,
                      void *attr);
template <int D>
void launch_update(cudaStream_t st, int n, const int *rp, const void *Y, void *Ynext, void *uY, void *gains,
                   const void *rep, const int *rep_flag, const void *attr, float exag4, float mom, float lr,
                   double *partials);
template <int D>
void launch_center(cudaStream_t st, int n, const void *Ynext, void *Ycur, const double *partials,
                   DevScalars *sc, const void *Yprev_conv, double *conv_partials);
template <int D>
void launch_exact_sv(cudaStream_t st, int n, const void *Y, float *s, void *v);
template <int D>
void launch_z_force(cudaStream_t st, int n, const void *Ypts, const float *s, const void *v,
                    const int *perm, void *rep, DevScalars *sc, double *partials, int h2_path,
                    int keep_rep);
template <int D>
void launch_kl(cudaStream_t st, int n, const int *rp, const int *col, const float *val,
               const void *Y, double exag, DevScalars *sc, double *partials);
template <int D>
void launch_attr_only(cudaStream_t st, int n, const int *rp, const int *col, const float *val,
                      const void *Y, double scale, double *grad_soa);
template <int D>
void launch_soa_to_vec(cudaStream_t st, int n, const double *soa, void *vec);
template <int D>
void launch_vec_to_soa(cudaStream_t st, int n, const void *vec, double *soa);
template <int D>
void launch_fill_vec(cudaStream_t st, int n, void *vec, float value);
template <int D>
void launch_permute_vec(cudaStream_t st, int n, const int *ord, const void *src, void *dst);
void launch_permute_int(cudaStream_t st, int n, const int *ord, const int *src, int *dst,
                        int identity_src);
void launch_invert_perm(cudaStream_t st, int n, const int *ord, int *inv);
void launch_row_len(cudaStream_t st, int n, const int *ord, const int *rp_old, int *len_new);
// renumbering of the CSR: new row k = old row ord[k], columns mapped through inv
void launch_row_gather(cudaStream_t st, int n, const int *ord, const int *inv, const int *rp_old,
                       const int *col_old, const float *val_old, const int *rp_new, int *col_new, float *val_new);
void launch_pcal(cudaStream_t st, int n, const int *indptr, const double *dist,
                 double perplexity, double *out);

}  // namespace tsne
