// The 2D attractive pass over row tiles with shared columns (attr_tiles.cu).
#pragma once

#include <cuda_runtime.h>

#include "devbuf.h"

namespace tsne {

struct AttrTiles {
    DevBuf<unsigned short> lidx;   // per padded P entry: index into its tile's column list
    DevBuf<int> ucol;              // the tiles' sorted distinct columns, tile after tile
    DevBuf<int> uptr;              // ntile + 1 offsets into ucol
    int ntile = 0;
    int rows = 64;                 // rows per tile (a multiple of 16)
    int umax = 6144;               // distinct columns the shared-memory stage holds
    int n_unique = 0;
    bool valid = false;
};

// Builds the tile format for the padded CSR (rp, col) of n rows; 0 ok, -1 when P is too large
// for 32-bit entry positions. Buffers come from the calling thread's allocation stream.
int attr_tiles_build(cudaStream_t st, int n, long long padded_nnz, const int *rp, const int *col, int rows, int umax,
                     AttrTiles &out);

// The fused step (attractive sums + gains/momentum update + centring partials in ROW_GRID
// slots) and the sums alone, as launch_attr_update<2> / launch_attr_grad<2> compute them.
void launch_attr_tile_update(cudaStream_t st, int n, const AttrTiles &tl, const int *rp, const int *col,
                             const float *val, const void *Y, void *Ynext, void *uY, void *gains, const void *rep,
                             const int *rep_flag, float exag4, float mom, float lr, double *partials);
void launch_attr_tile_grad(cudaStream_t st, int n, const AttrTiles &tl, const int *rp, const int *col,
                           const float *val, const void *Y, void *attr);

}  // namespace tsne
