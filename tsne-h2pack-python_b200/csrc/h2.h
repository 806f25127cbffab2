// Device H2 matrix of the repulsive kernel (1 + r^2)^-2: construction (tree, lists,
// proxy-point interpolative decomposition) and the fused product [s | v] = K [1 | Y].
#pragma once

#include <cuda_runtime.h>
#include <functional>
#include <memory>
#include <vector>

#include "kernels.h"

namespace tsne {

struct H2Stats {
    int n_node = 0, max_level = 0, n_far = 0, n_near = 0, max_leaf = 0;
    int rank_max = 0;
    double rank_mean = 0.0;
};

class H2Matrix {
public:
    virtual ~H2Matrix() = default;
    // Build for the points Y (device, point order). Returns 0 on success, -1 when Y holds
    // a non-finite coordinate, -2 when a bounded dependency wait of an earlier launch gave
    // up, 1 when the tree is too shallow for an H2 matrix
    // (max_level <= 2: the caller uses the exact sums). `overlap`, when given, is called
    // once, after the tree and list-count kernels are queued and before the host waits for
    // their counts: work it queues on the stream keeps the GPU busy meanwhile (it must not
    // depend on the tree).
    virtual int build(const void *Y, int leaf_size, double tol, const std::function<void()> *overlap = nullptr) = 0;
    // [s | v] = K [1 | Y] - [1 | Y] (diagonal excluded), tree order; then the Z identity and
    // the force, written in point order into F. keep_rep marks F as the stored force.
    virtual void product_force(void *F, DevScalars *sc, double *partials, int keep_rep) = 0;
    // s (n) and v (D-vectors) in point order on the host, for tests and the C ABI
    virtual void product_host(std::vector<float> &s, std::vector<float> &v) = 0;
    // K x - x for up to four input columns (tree order, 4 floats per point), diagonal excluded
    virtual void product_columns(const std::vector<float> &x_tree, std::vector<float> &y_tree) = 0;
    virtual const int *perm_device() const = 0;           // tree position -> point
    virtual const H2Stats &stats() const = 0;
    virtual void copy_tree(int *perm, double *corner, double *radius) = 0;
    virtual void copy_nodes(int *start, int *end, int *level, int *parent, int *fchild,
                            int *nchild, int *leaf) = 0;
    virtual void copy_lists(int *far_ptr, int *far_idx, int *near_ptr, int *near_idx) = 0;
    virtual void copy_ranks(int *rank) = 0;
    // the bases: node t's U rows are row_off[t] .. row_off[t] + (its leaf's points, or its
    // children's ranks summed) - 1, max_rank floats each (columns past the node's rank
    // unused); skel holds max_rank skeleton points of d floats per node. With U == nullptr
    // only n_rows (= row_off[n_node]) and max_rank are returned. -1 before a build.
    virtual int copy_bases(int *n_rows, int *max_rank, long long *row_off, float *U, float *skel) = 0;
    virtual long long launches() const = 0;
    // 1 when a bounded wait of a dependency-ordered launch gave up since the last build
    // (its results are not to be trusted); synchronises the stream
    virtual int wait_failed() = 0;
    // Test of the failure path: one dependency wait, bounded to `polls` polls, on a node flag
    // that nothing publishes. The wait gives up and records the failure that the next build
    // reports. Returns wait_failed() (1), or -1 before any build.
    virtual int probe_dependency_timeout(int polls) = 0;
    // prints and clears the per-phase device times gathered under TSNE_H2_TIMERS=1
    virtual void flush_timers() = 0;
};

std::unique_ptr<H2Matrix> make_h2_matrix(int d, int n, cudaStream_t st);

}  // namespace tsne
