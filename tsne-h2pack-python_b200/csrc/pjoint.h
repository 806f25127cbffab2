// The joint probabilities P built on the device from a k-NN distance graph.
#pragma once

#include <cuda_runtime.h>

#include "devbuf.h"
#include "../../include/tsne_h2pack.h"

namespace tsne {

// CSR on the device: int32 row pointers and columns, FP64 values
struct DevCSR {
    DevBuf<int> rp, col;
    DevBuf<double> val;
    int n = 0;
    long long nnz = 0;
};

// P = (P_c + P_c^T) / sum from a host k-NN distance graph (rows sorted by column, no self
// entries), P_c the conditional probabilities at `perplexity`. Buffers come from the calling
// thread's allocation stream. 0 on success, -1 on bad input (reported on stderr); throws
// CudaError on a device error. Synchronises `st`.
int joint_P_device(cudaStream_t st, int n, const double *knn_dist, const int *knn_ind, const int *knn_indptr,
                   long long nnz, double perplexity, DevCSR &out);

}  // namespace tsne
