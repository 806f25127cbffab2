// Device H2 matrix of the t-SNE repulsive kernel K(x, y) = (1 + |x - y|^2)^-2.
//
// The reference builds and applies its H2 matrix through the H2Pack library
// (src/tsne_h2pack.c:772-953 update_h2_matrix, src/tsne_h2_matmul.c:225-452 fused product),
// which is absent from the reference checkout. This file is the engine's own design:
//
//   tree   : root box = bounding-box midpoint with half-width MIN_HALF_WIDTH * 2^k; 64-bit
//            Morton keys of the points' cells at depth L; stable radix sort -> tree order;
//            nodes split level by level (binary search of the child digit inside each node)
//            while they hold more than leaf_size points. Nodes are numbered level by level
//            in key order.
//   lists  : per-target far / near partners of the symmetric dual-tree traversal, derived
//            level by level from the parent's inadmissible-source set (NSET).
//   bases  : for every node at level >= 2, an interpolative decomposition of K(candidates,
//            proxy points): column-pivoted Gram-Schmidt in shared memory, one CTA per node,
//            candidates = a leaf's points or the children's skeletons (nested bases).
//   product: upward pass (warp per node), far field (warp per compressed target), near
//            field (CTA per leaf, source tiles in shared memory), downward pass, then the Z
//            identity and the force.
// The CPU oracle (oracle/tsne_oracle.c) restates the same design; tree and lists agree bit
// for bit.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "devbuf.h"
#include "h2.h"
#include "kernels.h"

namespace tsne {
namespace {

template <int D> using Vec = typename Dim<D>::vec;

constexpr int IDG_THREADS = 256;     // shared-memory ID kernel (3D, large 2D leaves)
constexpr int IDG_GROUP = 4;         // its threads per candidate row in a Gram-Schmidt step
constexpr int NEAR_THREADS = 128;
constexpr int STACK_CAP = 192;       // leaf-target descent stack (depth * (2^D - 1) + 2^D)

struct TreeView {
    int n, L, leaf_size, cap_node, nset_cap;
    const unsigned long long *keys;
    int *start, *end, *level, *parent, *fchild, *nchild, *leaf, *ix;
    signed char *delta;      // shared leading digits with the previous key (n + 1)
    int *fm;                 // per point: first | last level << 8 of the nodes it starts, or -1
    int *blkcnt, *blkoff;    // per block of TREE_BLOCK points, 2 x 32 counts / offsets
    int *bset, *nid;         // per level l: boundary starts B_l and their node ids (stride cap_node)
    int *btot;               // |B_l|
    TreeInfo *info;
};

__device__ __forceinline__ void fma4(float4 &acc, float w, const float4 &v)
{
    acc.x = fmaf(w, v.x, acc.x); acc.y = fmaf(w, v.y, acc.y);
    acc.z = fmaf(w, v.z, acc.z); acc.w = fmaf(w, v.w, acc.w);
}
__device__ __forceinline__ void add4(float4 &a, const float4 &b) { a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w; }

// ---------------------------------------------------------------------------------
// root box and keys
// ---------------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(256) k_bbox(int n, const Vec<D> *__restrict__ Y, double *__restrict__ part)
{
    float lo[D], hi[D];
    int bad = 0;
    for (int k = 0; k < D; k++) { lo[k] = INFINITY; hi[k] = -INFINITY; }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> y = Y[i];
        for (int k = 0; k < D; k++) {
            const float v = vget(y, k);
            if (!isfinite(v)) { bad++; continue; }
            lo[k] = fminf(lo[k], v);
            hi[k] = fmaxf(hi[k], v);
        }
    }
    __shared__ float sl[256][D], sh[256][D];
    __shared__ int sb[256];
    for (int k = 0; k < D; k++) { sl[threadIdx.x][k] = lo[k]; sh[threadIdx.x][k] = hi[k]; }
    sb[threadIdx.x] = bad;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            for (int k = 0; k < D; k++) {
                sl[threadIdx.x][k] = fminf(sl[threadIdx.x][k], sl[threadIdx.x + s][k]);
                sh[threadIdx.x][k] = fmaxf(sh[threadIdx.x][k], sh[threadIdx.x + s][k]);
            }
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < D; k++) {
            part[(size_t)blockIdx.x * (2 * D + 1) + k] = sl[0][k];
            part[(size_t)blockIdx.x * (2 * D + 1) + D + k] = sh[0][k];
        }
        part[(size_t)blockIdx.x * (2 * D + 1) + 2 * D] = sb[0];
    }
}

// Root box from the bounding box (min / max are exact in any order), then the root node.
template <int D>
__global__ void __launch_bounds__(256) k_root(int n, int L, int nblk, const double *__restrict__ part, TreeView tv)
{
    __shared__ double slo[256][D], shi[256][D], sbad[256];
    double lo[D], hi[D], bad = 0.0;
    for (int k = 0; k < D; k++) { lo[k] = INFINITY; hi[k] = -INFINITY; }
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        for (int k = 0; k < D; k++) {
            lo[k] = fmin(lo[k], part[(size_t)b * (2 * D + 1) + k]);
            hi[k] = fmax(hi[k], part[(size_t)b * (2 * D + 1) + D + k]);
        }
        bad += part[(size_t)b * (2 * D + 1) + 2 * D];
    }
    for (int k = 0; k < D; k++) { slo[threadIdx.x][k] = lo[k]; shi[threadIdx.x][k] = hi[k]; }
    sbad[threadIdx.x] = bad;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            for (int k = 0; k < D; k++) {
                slo[threadIdx.x][k] = fmin(slo[threadIdx.x][k], slo[threadIdx.x + s][k]);
                shi[threadIdx.x][k] = fmax(shi[threadIdx.x][k], shi[threadIdx.x + s][k]);
            }
            sbad[threadIdx.x] += sbad[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    TreeInfo *info = tv.info;
    double ext = 0.0, ctr[D];
    for (int k = 0; k < D; k++) {
        ctr[k] = 0.5 * (slo[0][k] + shi[0][k]);
        const double e = 0.5 * (shi[0][k] - slo[0][k]);
        if (e > ext) ext = e;
    }
    double R = MIN_HALF_WIDTH;
    for (int it = 0; it < 2100 && R < ext; it++) R *= 2.0;
    info->nonfinite = sbad[0] > 0.0 ? 1 : 0;
    info->radius = R;
    for (int k = 0; k < 3; k++) info->corner[k] = k < D ? ctr[k] - R : 0.0;
    info->n_node = 1;
    info->max_level = 0;
    info->max_leaf = 0;
    info->nset_overflow = 0;
    info->pad[0] = 0;   // node-capacity overflow
    for (int l = 0; l < 32; l++) info->n_level_nodes[l] = 0;
    for (int l = 0; l < 33; l++) info->level_begin[l] = 0;
    info->n_level_nodes[0] = 1;
    info->level_begin[1] = 1;
    tv.start[0] = 0; tv.end[0] = n; tv.level[0] = 0; tv.parent[0] = -1;
    tv.fchild[0] = -1; tv.nchild[0] = 0; tv.leaf[0] = 1;
    tv.ix[0] = tv.ix[1] = tv.ix[2] = 0;
}

template <int D>
__global__ void k_keys(int n, int L, const Vec<D> *__restrict__ Y, const TreeInfo *__restrict__ info,
                       unsigned long long *__restrict__ keys, int *__restrict__ idx)
{
    const double R = info->radius;
    const double cell = 2.0 * R / (double)(1LL << L);
    const double qmax = (double)((1LL << L) - 1);
    double corner[D];
    for (int k = 0; k < D; k++) corner[k] = info->corner[k];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> y = Y[i];
        unsigned int q[D];
        for (int k = 0; k < D; k++) {
            const double t = ((double)vget(y, k) - corner[k]) / cell;
            double f;
            if (!(t >= 0.0)) f = 0.0;
            else if (t > qmax) f = qmax;
            else f = floor(t);
            q[k] = (unsigned int)f;
        }
        unsigned long long key = 0;
        for (int b = L - 1; b >= 0; b--)
            for (int k = D - 1; k >= 0; k--) key = (key << 1) | ((q[k] >> b) & 1u);
        keys[i] = key;
        idx[i] = i;
    }
}

// ---------------------------------------------------------------------------------
// tree: all levels at once from the sorted keys.
//
// delta[i] = number of leading base-2^D digits that key[i - 1] and key[i] share (L when equal;
// -1 at i = 0 and at the sentinel i = n). A node of level l is a maximal run of points with
// one l-digit prefix: it starts at a point s with delta[s] < l and ends at the next point
// with delta < l. A node exists when its parent holds more than leaf_size points (and it is
// at most at level L); the counts shrink down the tree, so that is the whole condition.
//
// Point s starts the nodes of levels f_s = delta[s] + 1 .. m_s when the node of level
// delta[s] around it holds more than leaf_size points (E_s); m_s is the first level whose
// node starting at s holds at most leaf_size points (the leaf), capped at L. Nodes are
// numbered level by level in key order; the starts of level l's node boundaries,
// B_l = {E points with f <= l}, give every node's end (the next entry of B_l), parent (the
// entry of B_{l-1} at or before it) and children (the entries of B_{l+1} inside it).
// ---------------------------------------------------------------------------------
constexpr int TREE_BLOCK = 1024;   // points per block of the marking and numbering kernels

template <int D>
__device__ __forceinline__ int shared_digits(unsigned long long a, unsigned long long b, int L)
{
    const unsigned long long x = a ^ b;
    if (x == 0ULL) return L;
    return (__clzll((long long)x) - (64 - D * L)) / D;
}

template <int D>
__device__ __forceinline__ unsigned int key_coord(unsigned long long key, int k, int L)
{
    unsigned int q = 0;
    for (int b = 0; b < L; b++) q |= (unsigned int)((key >> (D * b + k)) & 1ULL) << b;
    return q;
}

// tree-order coordinates, and delta (with its sentinel)
template <int D>
__global__ void k_gather(int n, int L, const int *__restrict__ perm, const Vec<D> *__restrict__ Y,
                         Vec<D> *__restrict__ xt, const unsigned long long *__restrict__ keys,
                         signed char *__restrict__ delta)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        if (i == n) {
            delta[n] = -1;
            continue;
        }
        xt[i] = Y[perm[i]];
        delta[i] = i == 0 ? (signed char)-1 : (signed char)shared_digits<D>(keys[i - 1], keys[i], L);
    }
}

// per point: E, f, m packed in fm (-1: starts no node); per block and level the number of
// node starts and of boundary starts
__device__ __forceinline__ void tree_bits(int fm, int l, bool &bn, bool &bb)
{
    const int f = fm & 0xff, m = fm >> 8;
    bb = fm >= 0 && f <= l;
    bn = bb && l <= m;
}

template <int D>
__global__ void __launch_bounds__(TREE_BLOCK) k_tree_marks(TreeView tv)
{
    __shared__ int wc[2][32][TREE_BLOCK / 32];
    const int n = tv.n, L = tv.L, leaf = tv.leaf_size;
    const signed char *delta = tv.delta;
    const int s = blockIdx.x * TREE_BLOCK + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int fm = -1;
    if (s < n) {
        const int ds = delta[s], f = ds + 1;
        bool E = s == 0;
        if (s > 0) {
            int j = s - 1;
            while (delta[j] >= ds && s - j <= leaf) j--;   // delta[0] = -1 ends the walk
            const int left = s - j;
            if (left > leaf) E = true;
            else {
                int k = s + 1;
                while (k < n && delta[k] >= ds && left + (k - s) <= leaf) k++;
                E = left + (k - s) > leaf;
            }
        }
        if (f > L) E = false;
        if (E) {
            int mu = L + 1;
            const int last = min(s + leaf, n);
            for (int j = s + 1; j <= last && mu >= f; j++) mu = min(mu, (int)delta[j]);
            const int m = min(L, max(f, mu + 1));
            fm = f | (m << 8);
        }
        tv.fm[s] = fm;
    }
    for (int l = 0; l <= L; l++) {
        bool bn, bb;
        tree_bits(fm, l, bn, bb);
        const unsigned vn = __ballot_sync(0xffffffffu, bn), vb = __ballot_sync(0xffffffffu, bb);
        if (lane == 0) { wc[0][l][w] = __popc(vn); wc[1][l][w] = __popc(vb); }
    }
    __syncthreads();
    if (threadIdx.x < 64) {
        const int arr = threadIdx.x >> 5, l = threadIdx.x & 31;
        int c = 0;
        if (l <= L)
            for (int k = 0; k < TREE_BLOCK / 32; k++) c += wc[arr][l][k];
        tv.blkcnt[((size_t)blockIdx.x * 2 + arr) * 32 + l] = c;
    }
}

// one CTA: block offsets per level (exclusive scans over the blocks), level table, totals
// Exclusive scans of the 64 per-block count columns (a CTA per column; each thread takes a
// contiguous run of blocks, then a block-wide scan of the runs). Column totals: the node
// counts per level (columns 0-31) into btot[32 + l], the boundary counts |B_l| (columns 32-63)
// into btot[l]; k_tree_levels turns the level counts into the node table's level ranges.
constexpr int TREE_SCAN_THREADS = 1024;

__global__ void __launch_bounds__(TREE_SCAN_THREADS) k_tree_scan(int nblk, TreeView tv)
{
    __shared__ int wsum[TREE_SCAN_THREADS / 32];
    const int col = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int per = (nblk + TREE_SCAN_THREADS - 1) / TREE_SCAN_THREADS;
    const int b0 = min(nblk, tid * per), b1 = min(nblk, b0 + per);
    auto at = [&](int b) { return ((size_t)b * 2 + (col >> 5)) * 32 + (col & 31); };
    int own = 0;
    for (int b = b0; b < b1; b++) own += tv.blkcnt[at(b)];
    int x = own;   // inclusive scan of the runs: warps, then the warp totals
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        wsum[lane] = t;
    }
    __syncthreads();
    int run = x - own + (w > 0 ? wsum[w - 1] : 0);
    for (int b = b0; b < b1; b++) {
        const int v = tv.blkcnt[at(b)];
        tv.blkoff[at(b)] = run;
        run += v;
    }
    if (tid == TREE_SCAN_THREADS - 1) {
        const int total = wsum[31];
        if (col < 32) tv.btot[32 + col] = total;
        else tv.btot[col - 32] = (col - 32) <= tv.L ? total : 0;
    }
}

__global__ void k_tree_levels(TreeView tv)
{
    if (threadIdx.x != 0) return;
    TreeInfo *info = tv.info;
    int acc = 0, maxl = 0;
    for (int l = 0; l < 32; l++) {
        const int c = l <= tv.L ? tv.btot[32 + l] : 0;
        info->level_begin[l] = acc;
        info->n_level_nodes[l] = c;
        if (c > 0) maxl = l;
        acc += c;
    }
    info->level_begin[32] = acc;
    info->n_node = acc;
    info->max_level = maxl;
    if (acc > tv.cap_node) {   // node table full: the host regrows it; nothing downstream runs
        info->pad[0] = 1;
        info->n_node = 0;
        info->max_level = 0;
        for (int l = 0; l < 32; l++) info->n_level_nodes[l] = 0;
    }
}

// numbers the nodes and writes their start, level, leaf flag, box index and first child;
// end, parent and child count are stored as positions in the boundary lists for k_tree_finish
template <int D>
__global__ void __launch_bounds__(TREE_BLOCK) k_tree_emit(TreeView tv)
{
    __shared__ int wo[2][32][TREE_BLOCK / 32];
    const TreeInfo *info = tv.info;
    if (info->pad[0]) return;
    const int n = tv.n, L = tv.L;
    const int s = blockIdx.x * TREE_BLOCK + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int fm = s < n ? tv.fm[s] : -1;
    for (int l = 0; l <= L; l++) {
        bool bn, bb;
        tree_bits(fm, l, bn, bb);
        const unsigned vn = __ballot_sync(0xffffffffu, bn), vb = __ballot_sync(0xffffffffu, bb);
        if (lane == 0) { wo[0][l][w] = __popc(vn); wo[1][l][w] = __popc(vb); }
    }
    __syncthreads();
    __shared__ int sboff[2][32], slb[32];
    if (threadIdx.x < 64) {   // exclusive scan over the warps, per array and level
        const int arr = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l <= L) {
            int run = 0;
            for (int k = 0; k < TREE_BLOCK / 32; k++) { const int c = wo[arr][l][k]; wo[arr][l][k] = run; run += c; }
        }
        // the block's level offsets, read once (not once per level by every warp)
        sboff[arr][l] = l <= L ? tv.blkoff[((size_t)blockIdx.x * 2 + arr) * 32 + l] : 0;
        if (arr == 0) slb[l] = info->level_begin[l];
    }
    __syncthreads();
    const size_t cap = (size_t)tv.cap_node;
    const unsigned long long key = s < n ? tv.keys[s] : 0ULL;
    const int f = fm & 0xff, m = fm >> 8;
    int prev_br = 0, prev_id = -1;
    for (int l = 0; l <= L; l++) {
        bool bn, bb;
        tree_bits(fm, l, bn, bb);
        const unsigned vn = __ballot_sync(0xffffffffu, bn), vb = __ballot_sync(0xffffffffu, bb);
        const int br = sboff[1][l] + wo[1][l][w] + __popc(vb & lt);
        if (bb) {
            int id = -1;
            if (bn) {
                const int nr = sboff[0][l] + wo[0][l][w] + __popc(vn & lt);
                id = slb[l] + nr;
                tv.start[id] = s;
                tv.level[id] = l;
                tv.leaf[id] = l == m ? 1 : 0;
                for (int k = 0; k < 3; k++)
                    tv.ix[(size_t)id * 3 + k] = k < D ? (int)(key_coord<D>(key, k, L) >> (L - l)) : 0;
                tv.end[id] = br;
                tv.parent[id] = l == 0 ? -1 : (f <= l - 1 ? prev_br : prev_br - 1);
                tv.fchild[id] = -1;
                tv.nchild[id] = 0;
                if (prev_id >= 0) { tv.fchild[prev_id] = id; tv.nchild[prev_id] = br; }
            }
            tv.bset[(size_t)l * cap + br] = s;
            tv.nid[(size_t)l * cap + br] = id;
            prev_id = id;
        }
        prev_br = br;
    }
}

// end, parent and child count of every node from the boundary lists; the largest leaf
template <int D>
__global__ void k_tree_finish(TreeView tv)
{
    TreeInfo *info = tv.info;
    if (info->pad[0]) return;
    const int n_node = info->n_node;
    const size_t cap = (size_t)tv.cap_node;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_node; t += gridDim.x * blockDim.x) {
        const int l = tv.level[t], s = tv.start[t], pos = tv.end[t];
        const int e = pos + 1 < tv.btot[l] ? tv.bset[(size_t)l * cap + pos + 1] : tv.n;
        tv.end[t] = e;
        if (l > 0) tv.parent[t] = tv.nid[(size_t)(l - 1) * cap + tv.parent[t]];
        if (tv.leaf[t]) {
            atomicMax(&info->max_leaf, e - s);
        } else {
            const int c0 = tv.nchild[t], lim = tv.btot[l + 1];
            int c = 0;
            while (c0 + c < lim && tv.bset[(size_t)(l + 1) * cap + c0 + c] < e) c++;
            tv.nchild[t] = c;
        }
    }
}

// ---------------------------------------------------------------------------------
// dependency-ordered launches
//
// A kernel that processes the nodes of several levels in one launch takes its work items from
// a ticket counter, so items start in ticket order whatever order the hardware dispatches
// blocks in. An item waits only for items with smaller tickets, which are held by running
// blocks or finished, so every wait ends. The waits are bounded all the same: after
// DEP_WAIT_LIMIT polls the waiting thread records the failure (the host reports it) and goes on.
// ---------------------------------------------------------------------------------
constexpr int DEP_WAIT_LIMIT = 1 << 22;

struct DepArgs {
    int *flag;      // per node: epoch of the last launch that finished it
    int *ticket;    // work-item counter, zeroed before the launch
    int *err;       // set when a wait gave up
    int epoch;
    int limit = DEP_WAIT_LIMIT;   // polls before a wait gives up
    int *flag2 = nullptr;         // a second per-node flag (launches that publish twice)
};

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// one thread: poll until node's flag holds this launch's epoch (bounded)
__device__ __forceinline__ void dep_wait(const DepArgs &dp, int node)
{
    const int *f = dp.flag + node;
    for (int it = 0; it < dp.limit; it++) {
        if (ld_acquire_gpu(f) == dp.epoch) return;
        __nanosleep(100);
    }
    atomicExch(dp.err, 1);
}
// one thread, after a block barrier that follows every write of the item
__device__ __forceinline__ void dep_publish(const DepArgs &dp, int node)
{
    __threadfence();
    st_release_gpu(dp.flag + node, dp.epoch);
}

// the second flag of a node (launches that publish twice: the bases publish the skeleton and
// rank first, the upward coefficients last)
__device__ __forceinline__ void dep_wait_y0(const DepArgs &dp, int node)
{
    DepArgs d2 = dp;
    d2.flag = dp.flag2;
    dep_wait(d2, node);
}
__device__ __forceinline__ void dep_publish_y0(const DepArgs &dp, int node)
{
    __threadfence();
    st_release_gpu(dp.flag2 + node, dp.epoch);
}

// one bounded wait for `node` (the failure path of the dependency-ordered launches, for tests)
__global__ void k_dep_probe(DepArgs dp, int node)
{
    if (threadIdx.x == 0) dep_wait(dp, node);
}

// ---------------------------------------------------------------------------------
// interaction lists
// ---------------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ bool admissible(const TreeView &tv, int t, int s)
{
    const long long wt = 1LL << (tv.L - tv.level[t]);
    const long long ws = 1LL << (tv.L - tv.level[s]);
    long long dist = 0;
    for (int k = 0; k < D; k++) {
        const long long ct = 2LL * tv.ix[(size_t)t * 3 + k] * wt + wt;
        const long long cs = 2LL * tv.ix[(size_t)s * 3 + k] * ws + ws;
        const long long df = ct > cs ? ct - cs : cs - ct;
        dist = df > dist ? df : dist;
    }
    return dist >= wt + ws + (long long)ADM_EXTRA * (wt < ws ? wt : ws);
}

// 2D: the count pass also parks each target's entries in fixed slots of LIST_SLOT entries, so
// that the list write is a compaction; a target with more entries sets slot_over and the build
// falls back to the traversing write pass
constexpr int LIST_SLOT = 128;

struct ListOut {
    int *far_cnt, *near_cnt;             // count pass
    const int *far_ptr, *near_ptr;       // write pass
    int *far_idx, *near_idx;
    int *nset, *nset_cnt;
    int *far_slot, *near_slot;           // count pass (2D): LIST_SLOT entries per target, or null
    int *slot_over;
    int write;
};

__device__ __forceinline__ void emit(int *idx, const int *ptr, int t, int &c, int v, int write,
                                     int *slot = nullptr, int *over = nullptr)
{
    if (write) idx[ptr[t] + c] = v;
    else if (slot != nullptr) {
        if (c < LIST_SLOT) slot[(size_t)t * LIST_SLOT + c] = v;
        else *over = 1;
    }
    c++;
}

// leaf target t against the subtree of c (c neither admissible nor a leaf)
template <int D>
__device__ void descend(const TreeView &tv, ListOut &lo, int t, int c, int &fc, int &nc)
{
    int stk[STACK_CAP];
    int sp = 0;
    for (int k = tv.nchild[c] - 1; k >= 0; k--) stk[sp++] = tv.fchild[c] + k;
    while (sp > 0) {
        const int s = stk[--sp];
        if (admissible<D>(tv, t, s)) { emit(lo.far_idx, lo.far_ptr, t, fc, s, lo.write, lo.far_slot, lo.slot_over); continue; }
        if (tv.leaf[s]) { emit(lo.near_idx, lo.near_ptr, t, nc, s, lo.write, lo.near_slot, lo.slot_over); continue; }
        if (sp + tv.nchild[s] > STACK_CAP) { atomicExch(&tv.info->nset_overflow, 1); return; }
        for (int k = tv.nchild[s] - 1; k >= 0; k--) stk[sp++] = tv.fchild[s] + k;
    }
}

template <int D>
__device__ void process_target(const TreeView &tv, ListOut &lo, int t)
{
    int fc = 0, nc = 0, ns = 0;
    if (t == 0) {
        if (tv.leaf[0]) emit(lo.near_idx, lo.near_ptr, 0, nc, 0, lo.write, lo.near_slot, lo.slot_over);
        else if (!lo.write) { lo.nset[0] = 0; ns = 1; }
    } else {
        const int p = tv.parent[t];
        const int pn = lo.nset_cnt[p];
        for (int a = 0; a < pn; a++) {
            const int s = lo.nset[(size_t)p * tv.nset_cap + a];
            const int c0 = tv.leaf[s] ? s : tv.fchild[s];
            const int c1 = tv.leaf[s] ? s + 1 : tv.fchild[s] + tv.nchild[s];
            for (int c = c0; c < c1; c++) {
                if (c == t) {
                    if (tv.leaf[t]) emit(lo.near_idx, lo.near_ptr, t, nc, t, lo.write, lo.near_slot, lo.slot_over);
                    else if (!lo.write) {
                        if (ns < tv.nset_cap) lo.nset[(size_t)t * tv.nset_cap + ns] = c;
                        ns++;
                    }
                } else if (admissible<D>(tv, t, c)) {
                    emit(lo.far_idx, lo.far_ptr, t, fc, c, lo.write, lo.far_slot, lo.slot_over);
                } else if (tv.leaf[t]) {
                    if (tv.leaf[c]) emit(lo.near_idx, lo.near_ptr, t, nc, c, lo.write, lo.near_slot, lo.slot_over);
                    else descend<D>(tv, lo, t, c, fc, nc);
                } else if (!lo.write) {
                    if (ns < tv.nset_cap) lo.nset[(size_t)t * tv.nset_cap + ns] = c;
                    ns++;
                }
            }
        }
    }
    if (!lo.write) {
        lo.far_cnt[t] = fc;
        lo.near_cnt[t] = nc;
        if (ns > tv.nset_cap) { atomicExch(&tv.info->nset_overflow, 1); ns = tv.nset_cap; }
        lo.nset_cnt[t] = ns;
    } else if (D == 2) {
        // ascending partners (insertion sort of this target's short segments; 3D lists are
        // longer and are sorted afterwards by a segmented sort)
        int *f = lo.far_idx + lo.far_ptr[t];
        for (int a = 1; a < fc; a++) { const int v = f[a]; int z = a - 1; while (z >= 0 && f[z] > v) { f[z + 1] = f[z]; z--; } f[z + 1] = v; }
        int *g = lo.near_idx + lo.near_ptr[t];
        for (int a = 1; a < nc; a++) { const int v = g[a]; int z = a - 1; while (z >= 0 && g[z] > v) { g[z + 1] = g[z]; z--; } g[z + 1] = v; }
    }
}

// count pass of the internal targets of every level in one dependency-ordered launch
// (persistent warps; a warp per target, in increasing node id, so a target's parent comes
// first). For target t the lanes take the entries a of the parent's inadmissible set, each
// with its candidate children c (the entry itself when it is a leaf): c goes to the far list
// when c != t and (t, c) is admissible, else to t's inadmissible set, which is written in
// (a, c) order, as process_target does.
template <int D>
__global__ void __launch_bounds__(256) k_lists_internal(TreeView tv, ListOut lo, DepArgs dp)
{
    constexpr int NCH = 1 << D;
    const int lane = threadIdx.x & 31;
    const int n_node = tv.info->n_node;
    const int cap = tv.nset_cap;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(dp.ticket, 1);
        const int t = __shfl_sync(0xffffffffu, item, 0);
        if (t >= n_node) break;
        if (tv.leaf[t]) continue;
        int nf = 0, ns = 0, nf_run = 0;
        if (t == 0) {
            if (lane == 0) lo.nset[0] = 0;
            ns = 1;
        } else {
            const int p = tv.parent[t];
            if (lane == 0) dep_wait(dp, p);
            __syncwarp();
            const int pn = __ldcg(lo.nset_cnt + p);
            for (int a0 = 0; a0 < pn; a0 += 32) {
                const int a = a0 + lane;
                int c0 = 0, c1 = 0, nn = 0;
                if (a < pn) {
                    const int src = __ldcg(lo.nset + (size_t)p * cap + a);
                    const bool sl = tv.leaf[src] != 0;
                    c0 = sl ? src : tv.fchild[src];
                    c1 = sl ? src + 1 : tv.fchild[src] + tv.nchild[src];
                }
                int nfl = 0;
#pragma unroll
                for (int k = 0; k < NCH; k++) {
                    const int c = c0 + k;
                    if (c < c1) {
                        if (c != t && admissible<D>(tv, t, c)) nfl++;
                        else nn++;
                    }
                }
                int inc = nn, incf = nfl;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, inc, o);
                    const int yf = __shfl_up_sync(0xffffffffu, incf, o);
                    if (lane >= o) { inc += y; incf += yf; }
                }
                int w = ns + inc - nn, wf = nf_run + incf - nfl;
#pragma unroll
                for (int k = 0; k < NCH; k++) {
                    const int c = c0 + k;
                    if (c < c1) {
                        if (!(c != t && admissible<D>(tv, t, c))) {
                            if (w < cap) lo.nset[(size_t)t * cap + w] = c;
                            w++;
                        } else if (lo.far_slot != nullptr) {
                            if (wf < LIST_SLOT) lo.far_slot[(size_t)t * LIST_SLOT + wf] = c;
                            else *lo.slot_over = 1;
                            wf++;
                        }
                    }
                }
                ns += __shfl_sync(0xffffffffu, inc, 31);
                nf_run += __shfl_sync(0xffffffffu, incf, 31);
                nf += nfl;
            }
        }
        nf = warp_sum(nf);
        if (lane == 0) {
            lo.far_cnt[t] = nf;
            lo.near_cnt[t] = 0;
            if (ns > cap) { atomicExch(&tv.info->nset_overflow, 1); ns = cap; }
            lo.nset_cnt[t] = ns;
        }
        __syncwarp();
        if (lane == 0) dep_publish(dp, t);
    }
}

// count pass, every leaf target (leaves need only their parent's NSET)
template <int D>
__global__ void __launch_bounds__(128) k_lists_leaves(TreeView tv, ListOut lo)
{
    const int n_node = tv.info->n_node;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_node; t += gridDim.x * blockDim.x)
        if (tv.leaf[t]) process_target<D>(tv, lo, t);
}

template <int D>
__global__ void __launch_bounds__(128) k_lists_write(int n_node, TreeView tv, ListOut lo)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_node; t += gridDim.x * blockDim.x)
        process_target<D>(tv, lo, t);
}

// the list write from the count pass's slots: a warp per target copies its entries to its
// list segment and sorts them ascending (the traversing write pass emits the same set and
// sorts it the same way)
__device__ __forceinline__ void warp_copy_sorted(const int *slot, int cnt, int *dst, int lane)
{
    // rank of each entry among the segment's (distinct) entries
    for (int a = lane; a < cnt; a += 32) {
        const int v = slot[a];
        int r = 0;
        for (int b = 0; b < cnt; b++) r += slot[b] < v;
        dst[r] = v;
    }
}

__global__ void __launch_bounds__(256) k_lists_compact(TreeView tv, ListOut lo)
{
    const int n_node = tv.info->n_node;
    const int lane = threadIdx.x & 31;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < n_node; t += (gridDim.x * blockDim.x) >> 5) {
        warp_copy_sorted(lo.far_slot + (size_t)t * LIST_SLOT, lo.far_cnt[t], lo.far_idx + lo.far_ptr[t], lane);
        warp_copy_sorted(lo.near_slot + (size_t)t * LIST_SLOT, lo.near_cnt[t], lo.near_idx + lo.near_ptr[t], lane);
    }
}

// rows of each node's interpolation matrix: a leaf's points, or (upper bound) the
// children's skeletons; nodes above MIN_ADM_LEVEL are not compressed
// iflag / lflag / bflag: 1 for the internal nodes / leaves of at most LEAF_SMALL (3D:
// ID3_TINY_LEAF) points / larger leaves at level >= MIN_ADM_LEVEL (the items of the basis
// launches)
constexpr int LEAF_SMALL = 64;
constexpr int ID3_TINY_LEAF = 32;   // 3D: the leaves of the smallest basis CTAs
template <int D>
__global__ void k_rowcap(TreeView tv, int *__restrict__ rowcap, int *__restrict__ iflag, int *__restrict__ lflag,
                         int *__restrict__ bflag)
{
    constexpr int NCH = 1 << D;
    const int n_node = tv.info->n_node;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_node; t += gridDim.x * blockDim.x) {
        int r = 0;
        const bool adm = tv.level[t] >= MIN_ADM_LEVEL;
        if (adm) r = tv.leaf[t] ? tv.end[t] - tv.start[t] : NCH * Dim<D>::MAXR;
        rowcap[t] = r;
        iflag[t] = adm && !tv.leaf[t];
        const int small = D == 2 ? LEAF_SMALL : ID3_TINY_LEAF;
        lflag[t] = adm && tv.leaf[t] && r <= small;
        bflag[t] = adm && tv.leaf[t] && r > small;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { rowcap[n_node] = 0; iflag[n_node] = 0; lflag[n_node] = 0; bflag[n_node] = 0; }
}

// ids of the flagged nodes in increasing order
__global__ void k_flag_list(const int *__restrict__ n_node_p, const int *__restrict__ flag,
                            const int *__restrict__ pos, int *__restrict__ list)
{
    const int n_node = *n_node_p;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_node; t += gridDim.x * blockDim.x)
        if (flag[t]) list[pos[t]] = t;
}

// ---------------------------------------------------------------------------------
// proxy points (shells |y - c|_inf = rho h around a box of half-width h)
// ---------------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void proxy_point(int p, double h, float *out)
{
    if constexpr (D == 2) {
        const int sh = p / SHELL_PTS_2D, k = p % SHELL_PTS_2D;
        const double rad = shell_rho(sh) * h;
        const double off = (sh & 1) ? 0.0 : 0.5;
        const double u = ((double)k + off) * (8.0 / SHELL_PTS_2D);
        const int side = (int)(u * 0.5);
        const double a = u - 2.0 * side - 1.0;
        double x, y;
        switch (side) {
            case 0: x = a; y = -1.0; break;
            case 1: x = 1.0; y = a; break;
            case 2: x = -a; y = 1.0; break;
            default: x = -1.0; y = -a; break;
        }
        out[0] = (float)(x * rad);
        out[1] = (float)(y * rad);
    } else {
        constexpr int g = SHELL_GRID_3D, per = 6 * g * g;
        const int sh = p / per, r = p % per, f = r / (g * g), ij = r % (g * g), i = ij / g, j = ij % g;
        const double rad = shell_rho(sh) * h;
        const int ax = f >> 1;
        const double sgn = (f & 1) ? 1.0 : -1.0;
        const double a = ((double)i + 0.5) * (2.0 / g) - 1.0;
        const double b = ((double)j + 0.5) * (2.0 / g) - 1.0;
        double c[3];
        c[ax] = sgn;
        c[(ax + 1) % 3] = a;
        c[(ax + 2) % 3] = b;
        for (int k = 0; k < 3; k++) out[k] = (float)(c[k] * rad);
    }
}

struct IdArgs {
    TreeView tv;
    const void *xt;
    void *skel;
    int *rank;
    const long long *rowoff;
    float *U;
    float *gA, *gnrm;
    int *gsel;
    void *gcand;
    int mcap;      // candidate rows that fit the launch's shared memory
    float tol2;
    float4 *y0;    // upward-pass coefficients of [1 | Y], computed right after the basis
};

template <int D>
constexpr size_t id_smem_bytes(int mcap)
{
    constexpr int P = Dim<D>::NPROXY, MAXR = Dim<D>::MAXR;
    return sizeof(float) * (size_t)P * D                 // proxies
           + sizeof(Vec<D>) * (size_t)mcap               // candidates
           + sizeof(float) * (size_t)mcap                // residual norms
           + sizeof(int) * (size_t)mcap                  // pivot position per row (-1: not selected)
           + sizeof(int) * (size_t)MAXR                  // pivot rows
           + sizeof(float) * (size_t)mcap * (P + 1);     // the matrix (row stride P + 1)
}

// Interpolative decomposition of one node (one CTA): A = K(candidates - c, proxies),
// column-pivoted Gram-Schmidt over the rows of A until the largest residual row norm is
// <= tol * the largest initial one; U = [I ; R11^-1 R12]^T in candidate order.
// The dot products of every step go to the node's U rows (R12), and the column of R11 that
// a step produces is stored in the pivot row of A, which no later step reads.
// LEAVES = true: every leaf at level >= 2 (leaves depend on nothing), blockIdx.x counts
// from the first node of level 2; false: the internal nodes of one level.
// One Gram-Schmidt step over the candidate rows of A (row stride PP): every unselected row a
// loses its component along the unit pivot row q; its dot product goes to U[a][r] and its new
// squared norm to nrm[a]. G threads per row, each over every G-th proxy.
template <int G, int P, int PP>
__device__ __forceinline__ void gs_rows(float *A, const float *q, int m, int tid, const int *selpos, float *nrm,
                                        float *U, int MAXR, int r)
{
    static_assert(P % G == 0, "proxies split evenly over a row's threads");
    for (int a0 = 0; a0 < m; a0 += IDG_THREADS / G) {
        const int a = a0 + tid / G, gl = tid % G;
        const bool act = a < m && selpos[a] < 0;
        float *row = A + (size_t)(act ? a : 0) * PP;
        float d2[2] = {0.f, 0.f};
        if (act) {
#pragma unroll 6
            for (int i = 0; i < P / G; i++) {
                const int p = gl + i * G;
                d2[i & 1] = fmaf(q[p], row[p], d2[i & 1]);
            }
        }
        float dot = d2[0] + d2[1];
        for (int o = 1; o < G; o <<= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
        float z2[2] = {0.f, 0.f};
        if (act) {
#pragma unroll 6
            for (int i = 0; i < P / G; i++) {
                const int p = gl + i * G;
                const float v = fmaf(-dot, q[p], row[p]);
                row[p] = v;
                z2[i & 1] = fmaf(v, v, z2[i & 1]);
            }
        }
        float s2 = z2[0] + z2[1];
        for (int o = 1; o < G; o <<= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        if (act && gl == 0) {
            nrm[a] = s2;
            U[(size_t)a * MAXR + r] = dot;
        }
    }
}

// items != nullptr: the internal nodes of every level in one dependency-ordered launch (items
// in increasing node id, taken deepest first; a node waits for its internal children's flags);
// otherwise the nodes of `level` (or every leaf). Children's ranks, skeletons and coefficients
// are read through L2.
template <int D, bool LEAVES>
__global__ void __launch_bounds__(IDG_THREADS) k_id(int level, IdArgs g, int n_item, const int *__restrict__ items,
                                                    DepArgs dp)
{
    constexpr int P = Dim<D>::NPROXY, PP = P + 1, MAXR = Dim<D>::MAXR, NCH = 1 << D;
    extern __shared__ __align__(16) unsigned char smraw[];
    const TreeView &tv = g.tv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    __shared__ int s_item;
    __shared__ int s_coff[NCH + 1];   // children's first candidate row
    __shared__ float4 s_part[IDG_THREADS];
    int t;
    if (items != nullptr) {
        if (tid == 0) s_item = atomicAdd(dp.ticket, 1);
        __syncthreads();
        if (s_item >= n_item) return;
        t = items[n_item - 1 - s_item];
        if (!LEAVES && tid < tv.nchild[t] && !tv.leaf[tv.fchild[t] + tid]) dep_wait(dp, tv.fchild[t] + tid);
        __syncthreads();
    } else {
        t = tv.info->level_begin[LEAVES ? MIN_ADM_LEVEL : level] + blockIdx.x;
        if (LEAVES ? !tv.leaf[t] : tv.leaf[t] != 0) return;
    }
    const int lvl = tv.level[t];
    const Vec<D> *xt = (const Vec<D> *)g.xt;
    Vec<D> *skel = (Vec<D> *)g.skel;

    unsigned char *ptr = smraw;
    float *prox = (float *)ptr; ptr += sizeof(float) * P * D;
    Vec<D> *cand_s = (Vec<D> *)ptr; ptr += sizeof(Vec<D>) * g.mcap;
    float *nrm_s = (float *)ptr; ptr += sizeof(float) * g.mcap;
    int *selpos_s = (int *)ptr; ptr += sizeof(int) * g.mcap;
    int *sel = (int *)ptr; ptr += sizeof(int) * MAXR;
    float *A_s = (float *)ptr;

    __shared__ float s_bv[IDG_THREADS / 32];
    __shared__ int s_bi[IDG_THREADS / 32];
    __shared__ int s_best, s_stop;
    __shared__ float s_n0;

    int m = 0;
    if (LEAVES) m = tv.end[t] - tv.start[t];
    else {
        if (tid == 0) {
            int acc = 0;
            for (int c = 0; c < tv.nchild[t]; c++) {
                s_coff[c] = acc;
                acc += __ldcg(g.rank + tv.fchild[t] + c);
            }
            s_coff[tv.nchild[t]] = acc;
        }
        __syncthreads();
        m = s_coff[tv.nchild[t]];
    }
    const long long roff = g.rowoff[t];
    const bool glob = m > g.mcap;
    float *A = glob ? g.gA + roff * PP : A_s;
    float *nrm = glob ? g.gnrm + roff : nrm_s;
    int *selpos = glob ? g.gsel + roff : selpos_s;
    Vec<D> *cand = glob ? (Vec<D> *)g.gcand + roff : cand_s;
    float *U = g.U + roff * MAXR;

    const double h = tv.info->radius / (double)(1LL << lvl);
    for (int p = tid; p < P; p += IDG_THREADS) proxy_point<D>(p, h, prox + p * D);
    float ctr[D];
    for (int k = 0; k < D; k++)
        ctr[k] = (float)(tv.info->corner[k] + (double)(2 * tv.ix[(size_t)t * 3 + k] + 1) * h);
    if (LEAVES) {
        for (int a = tid; a < m; a += IDG_THREADS) cand[a] = xt[tv.start[t] + a];
    } else {
        for (int a = tid; a < m; a += IDG_THREADS) {
            int c = 0;
            while (a >= s_coff[c + 1]) c++;
            cand[a] = __ldcg(skel + (size_t)(tv.fchild[t] + c) * MAXR + (a - s_coff[c]));
        }
    }
    __syncthreads();

    float lmax = 0.f;
    for (int a = tid; a < m; a += IDG_THREADS) {
        const Vec<D> x = cand[a];
        float rel[D];
        for (int k = 0; k < D; k++) rel[k] = vget(x, k) - ctr[k];
        float s2 = 0.f;
        float *row = A + (size_t)a * PP;
        for (int p = 0; p < P; p++) {
            float r2 = 0.f;
            for (int k = 0; k < D; k++) { const float df = rel[k] - prox[p * D + k]; r2 = fmaf(df, df, r2); }
            const float w = rkernel(r2);
            row[p] = w;
            s2 = fmaf(w, w, s2);
        }
        nrm[a] = s2;
        selpos[a] = -1;
        lmax = fmaxf(lmax, s2);
    }
    for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if (lane == 0) s_bv[wid] = lmax;
    __syncthreads();
    if (tid == 0) {
        float v = 0.f;
        for (int w = 0; w < IDG_THREADS / 32; w++) v = fmaxf(v, s_bv[w]);
        s_n0 = v;
    }
    __syncthreads();
    const float stop2 = g.tol2 * s_n0;
    const int rmax = min(min(m, P), MAXR);
    int r = 0;
    while (r < rmax) {
        float bv = -1.f;
        int bi = INT_MAX;
        for (int a = tid; a < m; a += IDG_THREADS)
            if (selpos[a] < 0 && (nrm[a] > bv)) { bv = nrm[a]; bi = a; }
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) { s_bv[wid] = bv; s_bi[wid] = bi; }
        __syncthreads();
        if (tid == 0) {
            float v = s_bv[0];
            int i = s_bi[0];
            for (int w = 1; w < IDG_THREADS / 32; w++)
                if (s_bv[w] > v || (s_bv[w] == v && s_bi[w] < i)) { v = s_bv[w]; i = s_bi[w]; }
            s_best = i;
            s_stop = (i == INT_MAX) || !(v > stop2) || !(v > 0.f);
        }
        __syncthreads();
        if (s_stop) break;
        const int best = s_best;
        const float rr = sqrtf(nrm[best]);
        const float inv = 1.0f / rr;
        float *q = A + (size_t)best * PP;
        for (int p = tid; p < P; p += IDG_THREADS) {
            const float v = q[p] * inv;
            q[p] = v;
            if (glob) A_s[p] = v;   // the shared-memory matrix area is free for a global-memory node
        }
        if (tid == 0) { selpos[best] = r; sel[r] = best; }
        __syncthreads();
        // G threads per row, each over every G-th proxy; the partial sums meet by shuffles inside
        // the group (whole warps take part in them). A matrix in global memory uses G = 8 and the
        // pivot row staged in shared memory, for more loads in flight per row.
        if (glob) gs_rows<8, P, PP>(A, A_s, m, tid, selpos, nrm, U, MAXR, r);
        else gs_rows<IDG_GROUP, P, PP>(A, q, m, tid, selpos, nrm, U, MAXR, r);
        __syncthreads();
        // column r of R11 (R[0..r-1][best] from the earlier steps, then the norm) into the
        // pivot row, which is dead from now on
        for (int k = tid; k <= r; k += IDG_THREADS) q[k] = k < r ? U[(size_t)best * MAXR + k] : rr;
        r++;
    }
    __syncthreads();
    for (int k = tid; k < r; k += IDG_THREADS) skel[(size_t)t * MAXR + k] = cand[sel[k]];
    if (tid == 0) g.rank[t] = r;
    // R11[k][j] = A[sel[j]][k]; a node whose matrix lives in global memory first copies R11 into
    // the (unused) shared-memory matrix area, column j at j (j + 1) / 2
    const float *R11 = A;
    if (glob) {
        float *R = A_s;
        for (int idx = tid; idx < r * r; idx += IDG_THREADS) {
            const int j = idx / r, k = idx % r;
            if (k <= j) R[j * (j + 1) / 2 + k] = A[(size_t)sel[j] * PP + k];
        }
        __syncthreads();
        R11 = R;
    }
    for (int a = tid; a < m; a += IDG_THREADS) {
        float *u = U + (size_t)a * MAXR;
        const int pos = selpos[a];
        if (pos >= 0) {
            for (int k = 0; k < r; k++) u[k] = (k == pos) ? 1.f : 0.f;
        } else if (glob) {
            for (int k = r - 1; k >= 0; k--) {
                float acc = u[k];
                for (int j = k + 1; j < r; j++) acc = fmaf(-R11[j * (j + 1) / 2 + k], u[j], acc);
                u[k] = acc / R11[k * (k + 1) / 2 + k];
            }
        } else {
            for (int k = r - 1; k >= 0; k--) {
                float acc = u[k];
                for (int j = k + 1; j < r; j++) acc = fmaf(-R11[(size_t)sel[j] * PP + k], u[j], acc);
                u[k] = acc / R11[(size_t)sel[k] * PP + k];
            }
        }
    }
    // upward pass of this node: y0[t] = U^T (the leaf's [1 | x] | the children's y0), groups of
    // RG threads over k and IDG_THREADS / RG groups over the rows, summed in a fixed order
    __syncthreads();
    {
        const int RG = r <= 16 ? 16 : (r <= 32 ? 32 : 64);
        const int C = IDG_THREADS / RG, kk = tid % RG, cg = tid / RG;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        if (kk < r) {
            for (int a = cg; a < m; a += C) {
                const float w = U[(size_t)a * MAXR + kk];
                if (LEAVES) {
                    const Vec<D> x = cand[a];
                    acc.x += w;
                    acc.y = fmaf(w, vget(x, 0), acc.y);
                    acc.z = fmaf(w, vget(x, 1), acc.z);
                    if (D == 3) acc.w = fmaf(w, vget(x, 2), acc.w);
                } else {
                    int c = 0;
                    while (a >= s_coff[c + 1]) c++;
                    fma4(acc, w, __ldcg(g.y0 + (size_t)(tv.fchild[t] + c) * MAXR + (a - s_coff[c])));
                }
            }
        }
        s_part[tid] = acc;
        __syncthreads();
        if (tid < r) {
            float4 y = s_part[tid];
            for (int c = 1; c < C; c++) add4(y, s_part[c * RG + tid]);
            g.y0[(size_t)t * MAXR + tid] = y;
        }
    }
    if (items != nullptr && !LEAVES) {
        __syncthreads();
        if (tid == 0) dep_publish(dp, t);
    }
}



// Warp argmax of (norm, row): the largest norm, ties to the lowest row. Norms are >= 0 or -1
// (no candidate), so their bit patterns order like the values.
__device__ __forceinline__ void warp_argmax(float &bv, int &bi)
{
    const int key = __float_as_int(bv);
    const int mx = __reduce_max_sync(0xffffffffu, key);
    bi = __reduce_min_sync(0xffffffffu, key == mx ? bi : INT_MAX);
    bv = __int_as_float(mx);
}

// Interpolative decompositions of the 2D nodes at level >= 2, one CTA of THREADS threads per
// node, thread `tid` owning candidate row tid (its row of A = K(candidate - c, proxies) in
// registers). LEAVES: every leaf (candidates = its points; CTAs of 64 threads for leaves of at
// most 64 points, which fit seven to an SM, and of 128 for the others). Otherwise every
// internal node in one dependency-ordered launch (candidates = the children's skeletons):
// items in decreasing node id (deepest level first), so a node's internal children come
// before it; it waits for their first flags (skeleton and rank, published right after their
// Gram-Schmidt steps) and, before its own upward sums, for their second flags (coefficients,
// published last), and reads all of these through L2 (CTAs of 128 threads). When the children's ranks add up to more than 128, thread
// tid also owns row 128 + tid, kept in global memory (in the node's first U rows, unused until
// the end).
// Column-pivoted Gram-Schmidt until the largest residual row norm is <= tol * the largest
// initial one (ties: the lower row); the dot products of every step are kept in shared
// memory (row-major, stride MAXR + 1), R11 is gathered from the pivot rows into shared
// memory, and the back substitution U = [I ; R11^-1 R12]^T runs there. Then U goes out to
// global memory, with the skeleton and the rank, and the upward coefficients
// y0 = U^T (the leaf's [1 | x] | the children's y0) are summed by all threads in a fixed order.
constexpr int ID2_THREADS = 128;                  // internal nodes and leaves of 65..128 points
constexpr int ID2_SMALL = 64;                     // leaves of at most 64 points
constexpr int ID2_DSTRIDE = Dim<2>::MAXR + 1;
constexpr size_t id2_smem(int threads) { return sizeof(float) * threads * ID2_DSTRIDE; }   // dot products

template <bool LEAVES, int THREADS>
__global__ void __launch_bounds__(THREADS, THREADS == ID2_SMALL ? 7 : 4)
k_id2d(int n_item, const int *__restrict__ items, IdArgs g, DepArgs dp)
{
    constexpr int P = Dim<2>::NPROXY, MAXR = Dim<2>::MAXR, NW = THREADS / 32;
    constexpr int ROWS = LEAVES ? THREADS : 2 * THREADS;   // candidate rows a CTA can hold
    static_assert(LEAVES || (ROWS >= 4 * MAXR && P == MAXR), "overflow rows reuse U rows of MAXR floats");
    extern __shared__ float dots[];            // [THREADS][ID2_DSTRIDE]
    __shared__ float prox[P * 2];
    __shared__ float qsh[P];
    __shared__ float rdiag[MAXR];
    __shared__ int piv[MAXR];
    __shared__ float R11[MAXR * (MAXR + 1) / 2];   // column jj at jj (jj + 1) / 2
    __shared__ float4 sin_[ROWS];
    __shared__ float4 part[THREADS];
    __shared__ float2 sxy[ROWS];
    __shared__ float s_bv[2][NW];
    __shared__ int s_bi[2][NW];
    __shared__ float s_lmax[NW];
    __shared__ int s_crank[4], s_item;
    const TreeView &tv = g.tv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    // internal nodes by level (items == nullptr): one launch per level, node n_item + block,
    // its children finished by the launches before, so nothing waits or publishes
    const bool bylevel = !LEAVES && items == nullptr;
    if (!LEAVES && !bylevel && tid == 0) s_item = atomicAdd(dp.ticket, 1);
    __syncthreads();
    int t;
    if (bylevel) {
        t = n_item + (int)blockIdx.x;
        if (tv.leaf[t]) return;   // uniform over the CTA
    } else {
        const int item = LEAVES ? (int)blockIdx.x : s_item;
        if (item >= n_item) return;
        t = items[LEAVES ? item : n_item - 1 - item];
    }
    const int lvl = tv.level[t];
    const float2 *xt = (const float2 *)g.xt;
    float2 *skel = (float2 *)g.skel;
    const int cfirst = tv.fchild[t], nch = LEAVES ? 0 : tv.nchild[t];
    if (!LEAVES && tid < nch) {
        if (!bylevel && !tv.leaf[cfirst + tid]) dep_wait(dp, cfirst + tid);   // leaves: the launch before
        s_crank[tid] = __ldcg(g.rank + cfirst + tid);
    }
    __syncthreads();
    int m = 0;
    if (LEAVES) m = tv.end[t] - tv.start[t];
    else for (int c = 0; c < nch; c++) m += s_crank[c];
    const int s0 = tv.start[t];
    const long long roff = g.rowoff[t];
    float *U = g.U + roff * MAXR;
    const double h = tv.info->radius / (double)(1LL << lvl);
    for (int p = tid; p < P; p += THREADS) proxy_point<2>(p, h, prox + p * 2);
    const float cx = (float)(tv.info->corner[0] + (double)(2 * tv.ix[(size_t)t * 3 + 0] + 1) * h);
    const float cy = (float)(tv.info->corner[1] + (double)(2 * tv.ix[(size_t)t * 3 + 1] + 1) * h);
    // candidates and the upward-pass inputs
    for (int q = 0; q < 2; q++) {
        const int a = tid + THREADS * q;
        if (a >= m) break;
        float2 pt;
        if (LEAVES) {
            pt = xt[s0 + a];
            sin_[a] = make_float4(1.f, pt.x, pt.y, 0.f);
        } else {
            int c = 0, aa = a;
            while (aa >= s_crank[c]) { aa -= s_crank[c]; c++; }
            pt = __ldcg(skel + (size_t)(cfirst + c) * MAXR + aa);
            if (bylevel) sin_[a] = __ldcg(g.y0 + (size_t)(cfirst + c) * MAXR + aa);
        }
        sxy[a] = pt;
    }
    __syncthreads();

    const bool valid = tid < m;
    const bool big = !LEAVES && m > THREADS;   // uniform over the block
    const bool xvalid = big && THREADS + tid < m;
    float row[P];
    int pos = valid ? -1 : -2, xpos = xvalid ? -1 : -2;
    float nrm = -1.f, xnrm = -1.f, lmax = 0.f;
    {
        const float2 x = valid ? sxy[tid] : make_float2(0.f, 0.f);
        const float rx = x.x - cx, ry = x.y - cy;
        float s4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int p = 0; p < P; p++) {
            const float dx = rx - prox[2 * p], dy = ry - prox[2 * p + 1];
            const float w = valid ? rkernel(fmaf(dx, dx, dy * dy)) : 0.f;
            row[p] = w;
            s4[p & 3] = fmaf(w, w, s4[p & 3]);
        }
        if (valid) nrm = (s4[0] + s4[1]) + (s4[2] + s4[3]);
        lmax = fmaxf(lmax, fmaxf(nrm, 0.f));
    }
    float *xr = U + (size_t)tid * MAXR;   // overflow row, in the node's first U rows
    if (xvalid) {
        const float2 xx = sxy[THREADS + tid];
        const float qx = xx.x - cx, qy = xx.y - cy;
        float z2 = 0.f;
        for (int p = 0; p < P; p++) {
            const float dx = qx - prox[2 * p], dy = qy - prox[2 * p + 1];
            const float w = rkernel(fmaf(dx, dx, dy * dy));
            xr[p] = w;
            z2 = fmaf(w, w, z2);
        }
        xnrm = z2;
        lmax = fmaxf(lmax, z2);
    }
    float bv = nrm;
    int bi = valid ? tid : INT_MAX;
    if (xnrm > bv) { bv = xnrm; bi = THREADS + tid; }
    lmax = __int_as_float(__reduce_max_sync(0xffffffffu, __float_as_int(lmax)));
    warp_argmax(bv, bi);
    if (lane == 0) { s_lmax[wid] = lmax; s_bv[0][wid] = bv; s_bi[0][wid] = bi; }
    __syncthreads();
    float n0 = 0.f;
    for (int w = 0; w < NW; w++) n0 = fmaxf(n0, s_lmax[w]);
    const float stop2 = g.tol2 * n0;
    const int rmax = min(min(m, P), MAXR);
    float *drow = dots + (size_t)tid * ID2_DSTRIDE;
    int r = 0, buf = 0;
    while (r < rmax) {
        float v = s_bv[buf][0];
        int best = s_bi[buf][0];
        for (int w = 1; w < NW; w++)
            if (s_bv[buf][w] > v || (s_bv[buf][w] == v && s_bi[buf][w] < best)) { v = s_bv[buf][w]; best = s_bi[buf][w]; }
        if (best == INT_MAX || !(v > stop2) || !(v > 0.f)) break;
        if (best == tid) {
            const float rr = sqrtf(nrm);
            const float inv = 1.0f / rr;
#pragma unroll
            for (int p = 0; p < P; p++) qsh[p] = row[p] * inv;
            rdiag[r] = rr;
            piv[r] = best;
            pos = r;
            nrm = -1.f;
        } else if (best == THREADS + tid) {
            const float rr = sqrtf(xnrm);
            const float inv = 1.0f / rr;
            for (int p = 0; p < P; p++) qsh[p] = xr[p] * inv;
            rdiag[r] = rr;
            piv[r] = best;
            xpos = r;
            xnrm = -1.f;
        }
        __syncthreads();
        bv = -1.f;
        bi = INT_MAX;
        if (pos == -1) {
            float d4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int p = 0; p < P; p++) d4[p & 3] = fmaf(qsh[p], row[p], d4[p & 3]);
            const float dot = (d4[0] + d4[1]) + (d4[2] + d4[3]);
            asm volatile("" ::: "memory");   // reload q below instead of holding 64 more registers
            float s4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int p = 0; p < P; p++) {
                row[p] = fmaf(-dot, qsh[p], row[p]);
                s4[p & 3] = fmaf(row[p], row[p], s4[p & 3]);
            }
            nrm = (s4[0] + s4[1]) + (s4[2] + s4[3]);
            drow[r] = dot;
            bv = nrm;
            bi = tid;
        }
        if (xpos == -1) {
            float dot = 0.f;
            for (int p = 0; p < P; p++) dot = fmaf(qsh[p], xr[p], dot);
            float s2 = 0.f;
            for (int p = 0; p < P; p++) {
                const float y = fmaf(-dot, qsh[p], xr[p]);
                xr[p] = y;
                s2 = fmaf(y, y, s2);
            }
            xnrm = s2;
            U[(size_t)(THREADS + tid) * MAXR + r] = dot;
            if (s2 > bv) { bv = s2; bi = THREADS + tid; }
        }
        warp_argmax(bv, bi);
        buf ^= 1;
        if (lane == 0) { s_bv[buf][wid] = bv; s_bi[buf][wid] = bi; }
        r++;
        __syncthreads();
    }
    __syncthreads();
    // skeleton and rank; R11 from the pivot rows' dot products (column jj: its entries k < jj)
    if (pos >= 0) skel[(size_t)t * MAXR + pos] = sxy[tid];
    if (xpos >= 0) skel[(size_t)t * MAXR + xpos] = sxy[THREADS + tid];
    if (tid == 0) g.rank[t] = r;
    for (int idx = tid; idx < r * r; idx += THREADS) {
        const int jj = idx / r, k = idx % r;
        if (k > jj) continue;
        const int pr = piv[jj];
        R11[jj * (jj + 1) / 2 + k] = k == jj ? rdiag[jj]
                                             : (pr < THREADS ? dots[(size_t)pr * ID2_DSTRIDE + k]
                                                                 : U[(size_t)pr * MAXR + k]);
    }
    __syncthreads();
    // the skeleton and the rank are what the parent's decomposition needs: published here;
    // the children's upward coefficients, published last, are waited for before the sums
    if (!LEAVES && !bylevel) {
        if (tid == 0) dep_publish(dp, t);
        if (tid < nch && !tv.leaf[cfirst + tid]) dep_wait_y0(dp, cfirst + tid);
        __syncthreads();
        for (int q = 0; q < 2; q++) {
            const int a = tid + THREADS * q;
            if (a >= m) break;
            int c = 0, aa = a;
            while (aa >= s_crank[c]) { aa -= s_crank[c]; c++; }
            sin_[a] = __ldcg(g.y0 + (size_t)(cfirst + c) * MAXR + aa);
        }
    }
    // back substitution of the non-pivot rows, column by column (independent updates)
    if (pos == -1) {
        for (int k = r - 1; k >= 0; k--) {
            const float *col = R11 + k * (k + 1) / 2;
            const float uk = drow[k] / col[k];
            drow[k] = uk;
            for (int i = 0; i < k; i++) drow[i] = fmaf(-col[i], uk, drow[i]);
        }
    }
    if (xpos == -1) {
        float *u = U + (size_t)(THREADS + tid) * MAXR;
        for (int k = r - 1; k >= 0; k--) {
            float acc = u[k];
            for (int jj = k + 1; jj < r; jj++) acc = fmaf(-R11[jj * (jj + 1) / 2 + k], u[jj], acc);
            u[k] = acc / R11[k * (k + 1) / 2 + k];
        }
    }
    __syncthreads();
    // pivot rows are rows of the identity
    if (pos >= 0)
        for (int k = 0; k < r; k++) drow[k] = k == pos ? 1.f : 0.f;
    if (xpos >= 0)
        for (int k = 0; k < r; k++) U[(size_t)(THREADS + tid) * MAXR + k] = k == xpos ? 1.f : 0.f;
    __syncthreads();
    // U rows 0 .. min(m, THREADS) - 1 out of shared memory (over the overflow rows' scratch)
    const int mm = min(m, THREADS);
    for (int idx = tid; idx < mm * r; idx += THREADS) {
        const int a = idx / r, k = idx % r;
        U[(size_t)a * MAXR + k] = dots[(size_t)a * ID2_DSTRIDE + k];
    }
    // y0[k] = sum_a U[a][k] in[a]: groups of RG threads over k, C = THREADS / RG groups over a
    const int RG = r <= 16 ? 16 : (r <= 32 ? 32 : 64);
    const int C = THREADS / RG, kk = tid % RG, cg = tid / RG;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (kk < r) {
        for (int a = cg; a < m; a += C) {
            const float w = a < THREADS ? dots[(size_t)a * ID2_DSTRIDE + kk] : U[(size_t)a * MAXR + kk];
            fma4(acc, w, sin_[a]);
        }
    }
    part[tid] = acc;
    __syncthreads();
    if (tid < r) {
        float4 y = part[tid];
        for (int c = 1; c < C; c++) add4(y, part[c * RG + tid]);
        g.y0[(size_t)t * MAXR + tid] = y;
    }
    if (!LEAVES && !bylevel) {
        __syncthreads();
        if (tid == 0) dep_publish_y0(dp, t);
    }
}

// ---------------------------------------------------------------------------------
// 3D interpolative decompositions with recomputed rows
// ---------------------------------------------------------------------------------
// The 3D proxy matrix has 216 columns and up to 512 candidate rows (eight children of rank
// <= 64): 442 KB in FP32, more than one SM holds. Its entries are cheap to recompute, one
// reciprocal each in the expanded form (1 + |x|^2 + |p|^2 - 2 x.p)^-2 (x: candidate relative
// to the node's centre, p: proxy), so no row is stored: the column-pivoted Gram-Schmidt runs
// left-looking. Step r takes the row b of the largest residual norm and orthonormalises it
// against the earlier directions q_0..q_{r-1} by classical Gram-Schmidt applied twice (the
// first pass from b's stored projections, the second recomputed, so the directions stay
// orthonormal to rounding); every other row a then recomputes its entries once for its dot
// product c = a . q_r (= its residual's, as q_r is orthogonal to the earlier directions),
// kept in shared memory as R12, with its squared residual norm downdated in FP64 by c^2.
// R11's column r is b's projections on q_0..q_{r-1} and its residual norm. The stop rule, tie
// rule, back substitution U = [I ; R11^-1 R12]^T and the upward coefficients are those of k_id.
//
// One CTA per node, in three sizes (THREADS, ROWS = the most candidate rows it takes): 512
// threads and 512 rows (internal nodes, leaves above 128 points; one CTA per SM), 256 and 128
// (leaves of 33..128 points; two per SM), 128 and 32 (leaves of at most 32 points, four per
// SM). The proxies are held in pairs (2j, 2j + 1) for the paired FP32 instructions; a row is
// split over S adjacent lanes (the largest S <= 16 with THREADS / S >= rows, else 2), lane
// `sub` taking the pairs j = sub mod S, and lane group g = tid / S covers the rows
// g + (THREADS / S) k; the S partial sums of a row meet by butterfly shuffles, which give
// every lane of the group the same value.
//
// Internal nodes run in one dependency-ordered launch: a node waits for its internal
// children's skeletons and ranks (flag), published right after their pivot loop, and, before
// its upward coefficients, for their coefficients (second flag, published last).
constexpr int ID3_P = Dim<3>::NPROXY;
constexpr int ID3_ROWS = 8 * Dim<3>::MAXR;   // candidate rows of an internal node
constexpr int ID3_QS = 220;                  // row stride of the directions (16-byte rows,
                                             // conflict-free for 4 lanes x 8 directions)
constexpr int ID3_TINY = 32;                 // leaves of the 128-thread CTAs
constexpr int ID3_SMALL = 128;               // leaves of the 256-thread CTAs
static_assert(ID3_TINY == ID3_TINY_LEAF, "the small-leaf list is the 128-thread launch's");
static_assert(ID3_P % 8 == 0 && ID3_QS >= ID3_P && ID3_QS % 4 == 0, "proxy pairs, 16-byte rows");

template <int THREADS, int ROWS>
struct Id3 {
    static constexpr int QR = ROWS < Dim<3>::MAXR ? ROWS : Dim<3>::MAXR;   // rank bound
    static constexpr int CS = QR + 1;                                      // row stride of R12 / U
    static constexpr int NW = THREADS / 32;
    static constexpr int NKMAX = 2 * ROWS > THREADS ? 2 * ROWS / THREADS : 1;   // rows per lane group
    static constexpr int SMIN = THREADS >= 2 * ROWS ? THREADS / ROWS : 2;       // smallest lane split
    static_assert(NKMAX <= 2 && THREADS >= 4 * QR, "row groups, four lanes per direction");
    struct Smem {
        float Q[QR * ID3_QS];                  // directions q_0..q_{r-1}; at the end: y0 partials
        float C[ROWS * CS];                    // R12 (the rows' dots), then U
        float4 pa[ID3_P / 2];                  // proxy pairs: (-2x, -2x', -2y, -2y')
        float4 pb[ID3_P / 2];                  //              (-2z, -2z', |p|^2, |p'|^2)
        float4 cand[ROWS];                     // candidates: (x, y, z) - centre, 1 + |.|^2
        float R11[QR * (QR + 1) / 2];          // column j at j (j + 1) / 2
        float res[ID3_P];                      // the pivot's residual
        float dc[QR];                          // its second-pass projections
        int piv[QR];
        int selpos[ROWS];                      // pivot position of each row, or -1
        float bv[2][NW];
        int bi[2][NW];
        float red[NW];
        int coff[9];
        int item;
    };
    static_assert(QR * ID3_QS * sizeof(float) >= THREADS * sizeof(float4), "y0 partials in the directions");
};

// entry of proxy p (scalar form of the paired arithmetic below: the same operations in the
// same order, so both give the same value)
template <typename SM>
__device__ __forceinline__ float id3_entry(const SM &s, const float4 &c, int p)
{
    const float4 A = s.pa[p >> 1], B = s.pb[p >> 1];
    const bool o = p & 1;
    const float mx = o ? A.y : A.x, my = o ? A.w : A.z, mz = o ? B.y : B.x, e = o ? B.w : B.z;
    const float d = fmaf(c.z, mz, fmaf(c.y, my, fmaf(c.x, mx, c.w + e)));
    const float w = fast_rcp(d);
    return w * w;
}

// Over the lane's share of the proxies (pairs sub, sub + S, ...), for its NK rows
// g + RPG k: NORM: sum of squared entries (FP64); otherwise the dot product with v (FP32,
// two partial sums per row).
template <int S, int NK, bool NORM, typename SM>
__device__ __forceinline__ void id3_rows(const SM &s, const float *v, int g, int rpg, int sub, double (&out)[2])
{
    F2 cx[NK], cy[NK], cz[NK], cw[NK], acc[NK];
    double dn[NK];
#pragma unroll
    for (int k = 0; k < NK; k++) {
        const float4 c = s.cand[g + rpg * k];
        cx[k] = f2_pack(c.x, c.x); cy[k] = f2_pack(c.y, c.y); cz[k] = f2_pack(c.z, c.z); cw[k] = f2_pack(c.w, c.w);
        acc[k] = f2_pack(0.f, 0.f);
        dn[k] = 0.0;
    }
#pragma unroll 2
    for (int j = sub; j < ID3_P / 2; j += S) {
        const float4 A = s.pa[j], B = s.pb[j];
        const F2 mx = f2_pack(A.x, A.y), my = f2_pack(A.z, A.w), mz = f2_pack(B.x, B.y), e = f2_pack(B.z, B.w);
        F2 vv;
        if (!NORM) {
            const float2 v2 = *reinterpret_cast<const float2 *>(v + 2 * j);
            vv = f2_pack(v2.x, v2.y);
        }
#pragma unroll
        for (int k = 0; k < NK; k++) {
            const F2 d = f2_fma(cz[k], mz, f2_fma(cy[k], my, f2_fma(cx[k], mx, f2_add(cw[k], e))));
            float d0, d1;
            f2_unpack(d, d0, d1);
            const F2 w = f2_pack(fast_rcp(d0), fast_rcp(d1));
            const F2 w2 = f2_mul(w, w);
            if (NORM) {
                float a0, a1;
                f2_unpack(w2, a0, a1);
                dn[k] = fma((double)a0, (double)a0, dn[k]);
                dn[k] = fma((double)a1, (double)a1, dn[k]);
            } else {
                acc[k] = f2_fma(w2, vv, acc[k]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < NK; k++) {
        if (NORM) out[k] = dn[k];
        else {
            float a0, a1;
            f2_unpack(acc[k], a0, a1);
            out[k] = (double)(a0 + a1);
        }
    }
}

// the lane group's row sums (every lane of the group gets the same values)
template <bool NORM, int SMIN, int NKMAX, typename SM>
__device__ __forceinline__ void id3_rows_any(const SM &s, const float *v, int S, int g, int rpg, int sub, int nk,
                                             double (&out)[2])
{
    out[0] = out[1] = 0.0;
    if (nk > 0) {
        if (S == 16) id3_rows<16, 1, NORM>(s, v, g, rpg, sub, out);
        else if (S == 8) id3_rows<8, 1, NORM>(s, v, g, rpg, sub, out);
        else if (SMIN <= 4 && S == 4) id3_rows<4, 1, NORM>(s, v, g, rpg, sub, out);
        else if constexpr (SMIN <= 2) {
            if (NKMAX >= 2 && nk == 2) id3_rows<2, (NKMAX >= 2 ? 2 : 1), NORM>(s, v, g, rpg, sub, out);
            else id3_rows<2, 1, NORM>(s, v, g, rpg, sub, out);
        }
    }
    for (int o = 1; o < S; o <<= 1) {
        out[0] += __shfl_xor_sync(0xffffffffu, out[0], o);
        out[1] += __shfl_xor_sync(0xffffffffu, out[1], o);
    }
}

// d[j] = q_j . res for the directions j < r (four lanes per direction, 54 proxies each)
template <typename SM>
__device__ __forceinline__ void id3_proj(SM &s, int r, int tid, float *d)
{
    const int j = tid >> 2, sub = tid & 3;
    float d0 = 0.f, d1 = 0.f;
    if (j < r) {
        const float *qj = s.Q + j * ID3_QS;
#pragma unroll
        for (int i = 0; i < ID3_P / 8; i++) {
            const int p = sub + 8 * i;
            d0 = fmaf(qj[p], s.res[p], d0);
            d1 = fmaf(qj[p + 4], s.res[p + 4], d1);
        }
    }
    float x = d0 + d1;
    x += __shfl_xor_sync(0xffffffffu, x, 1);
    x += __shfl_xor_sync(0xffffffffu, x, 2);
    if (sub == 0 && j < r) d[j] = x;
}

// v - sum_{j < r} d[j] q_j[p]
__device__ __forceinline__ float id3_sub(const float *Q, int r, int p, const float *d, float v)
{
    float a0 = v, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    int j = 0;
    for (; j + 3 < r; j += 4) {
        a0 = fmaf(-d[j], Q[j * ID3_QS + p], a0);
        a1 = fmaf(-d[j + 1], Q[(j + 1) * ID3_QS + p], a1);
        a2 = fmaf(-d[j + 2], Q[(j + 2) * ID3_QS + p], a2);
        a3 = fmaf(-d[j + 3], Q[(j + 3) * ID3_QS + p], a3);
    }
    for (; j < r; j++) a0 = fmaf(-d[j], Q[j * ID3_QS + p], a0);
    return (a0 + a1) + (a2 + a3);
}

template <int THREADS>
constexpr int id3_min_blocks() { return THREADS >= 512 ? 1 : (THREADS >= 256 ? 2 : 4); }

// LEAVES: the leaves of `items` with mlo < points <= ROWS (others are another launch's).
template <bool LEAVES, int THREADS, int ROWS>
__global__ void __launch_bounds__(THREADS, id3_min_blocks<THREADS>())
k_id3(int n_item, const int *__restrict__ items, int mlo, IdArgs g, DepArgs dp)
{
    using K = Id3<THREADS, ROWS>;
    using SM = typename K::Smem;
    constexpr int P = ID3_P, MAXR = Dim<3>::MAXR, QR = K::QR, CS = K::CS, NW = K::NW;
    constexpr int PPT = (P + THREADS - 1) / THREADS;   // proxies per thread in the pivot's steps
    extern __shared__ __align__(16) unsigned char smraw[];
    SM &s = *reinterpret_cast<SM *>(smraw);
    const TreeView &tv = g.tv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (!LEAVES && tid == 0) s.item = atomicAdd(dp.ticket, 1);
    __syncthreads();
    const int item = LEAVES ? (int)blockIdx.x : s.item;
    if (item >= n_item) return;
    const int t = items[LEAVES ? item : n_item - 1 - item];
    if (LEAVES) {
        const int mm = tv.end[t] - tv.start[t];
        if (mm <= mlo || mm > ROWS) return;   // uniform over the CTA
    }
    const int cfirst = tv.fchild[t], nch = LEAVES ? 0 : tv.nchild[t];
    if (!LEAVES && tid < nch && !tv.leaf[cfirst + tid]) dep_wait(dp, cfirst + tid);
    __syncthreads();
    if (tid == 0) {
        int acc = 0;
        for (int c = 0; c < nch; c++) {
            s.coff[c] = acc;
            acc += __ldcg(g.rank + cfirst + c);
        }
        s.coff[nch] = acc;
    }
    __syncthreads();
    const int m = LEAVES ? tv.end[t] - tv.start[t] : s.coff[nch];
    const int s0 = tv.start[t];
    const int lvl = tv.level[t];
    const long long roff = g.rowoff[t];
    float *U = g.U + roff * MAXR;
    const float4 *xt = (const float4 *)g.xt;
    float4 *skel = (float4 *)g.skel;
    const double h = tv.info->radius / (double)(1LL << lvl);
    float ctr[3];
    for (int k = 0; k < 3; k++)
        ctr[k] = (float)(tv.info->corner[k] + (double)(2 * tv.ix[(size_t)t * 3 + k] + 1) * h);
    for (int j = tid; j < P / 2; j += THREADS) {
        float p0[3], p1[3];
        proxy_point<3>(2 * j, h, p0);
        proxy_point<3>(2 * j + 1, h, p1);
        s.pa[j] = make_float4(-2.f * p0[0], -2.f * p1[0], -2.f * p0[1], -2.f * p1[1]);
        s.pb[j] = make_float4(-2.f * p0[2], -2.f * p1[2], fmaf(p0[0], p0[0], fmaf(p0[1], p0[1], p0[2] * p0[2])),
                              fmaf(p1[0], p1[0], fmaf(p1[1], p1[1], p1[2] * p1[2])));
    }
    for (int a = tid; a < m; a += THREADS) {
        float4 x;
        if (LEAVES) x = xt[s0 + a];
        else {
            int c = 0;
            while (a >= s.coff[c + 1]) c++;
            x = __ldcg(skel + (size_t)(cfirst + c) * MAXR + (a - s.coff[c]));
        }
        const float rx = x.x - ctr[0], ry = x.y - ctr[1], rz = x.z - ctr[2];
        s.cand[a] = make_float4(rx, ry, rz, 1.f + fmaf(rx, rx, fmaf(ry, ry, rz * rz)));
        s.selpos[a] = -1;
    }
    __syncthreads();

    int S = 2;   // uniform over the CTA
    while (S < 16 && THREADS / (2 * S) >= m) S <<= 1;
    const int rpg = THREADS / S, sub = tid & (S - 1), rb = tid / S;
    const int nk = max(0, min(K::NKMAX, (m - rb + rpg - 1) / rpg));   // rows rb + rpg k < m
    double nrm[2];
    int pos[2];   // -1: open row, -2: no row, >= 0: pivot position
    id3_rows_any<true, K::SMIN, K::NKMAX>(s, nullptr, S, rb, rpg, sub, nk, nrm);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        pos[k] = k < nk ? -1 : -2;
        if (pos[k] == -2) nrm[k] = -1.0;
    }
    float bv = -1.f, lmax = 0.f;
    int bi = INT_MAX;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float v = (float)nrm[k];
        if (pos[k] == -1 && sub == 0 && v > bv) { bv = v; bi = rb + rpg * k; }
        lmax = fmaxf(lmax, v);
    }
    lmax = __int_as_float(__reduce_max_sync(0xffffffffu, __float_as_int(lmax)));
    warp_argmax(bv, bi);
    if (lane == 0) { s.red[wid] = lmax; s.bv[0][wid] = bv; s.bi[0][wid] = bi; }
    __syncthreads();
    float n0 = 0.f;
    for (int w = 0; w < NW; w++) n0 = fmaxf(n0, s.red[w]);
    const float stop2 = g.tol2 * n0;
    const int rmax = min(min(m, P), QR);
    int r = 0, buf = 0;
    while (r < rmax) {
        float v = s.bv[buf][0];
        int best = s.bi[buf][0];
        for (int w = 1; w < NW; w++)
            if (s.bv[buf][w] > v || (s.bv[buf][w] == v && s.bi[buf][w] < best)) { v = s.bv[buf][w]; best = s.bi[buf][w]; }
        if (best == INT_MAX || !(v > stop2) || !(v > 0.f)) break;
        // the pivot's residual: thread tid takes the proxies tid + THREADS i
        const float *cb = s.C + best * CS;   // the pivot's projections on q_0..q_{r-1}
        float rv[PPT];
#pragma unroll
        for (int i = 0; i < PPT; i++) {
            const int p = tid + THREADS * i;
            rv[i] = 0.f;
            if (p < P) {
                rv[i] = id3_sub(s.Q, r, p, cb, id3_entry(s, s.cand[best], p));
                s.res[p] = rv[i];
            }
        }
        __syncthreads();
        if (r > 0) id3_proj(s, r, tid, s.dc);   // uniform
        __syncthreads();
        float sq = 0.f;
#pragma unroll
        for (int i = 0; i < PPT; i++) {
            const int p = tid + THREADS * i;
            if (p < P) {
                rv[i] = id3_sub(s.Q, r, p, s.dc, rv[i]);
                s.res[p] = rv[i];
                sq = fmaf(rv[i], rv[i], sq);
            }
        }
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if (lane == 0) s.red[wid] = sq;
        __syncthreads();
        float rr2 = 0.f;
        for (int w = 0; w < NW; w++) rr2 += s.red[w];
        const float rr = sqrtf(rr2);
        if (!(rr > 0.f) || !(rr < INFINITY)) break;   // uniform: every thread sums the same values
        const float inv = 1.0f / rr;
#pragma unroll
        for (int i = 0; i < PPT; i++)
            if (tid + THREADS * i < P) s.Q[r * ID3_QS + tid + THREADS * i] = rv[i] * inv;
        if (tid < r) s.R11[r * (r + 1) / 2 + tid] = cb[tid] + s.dc[tid];
        if (tid == r) s.R11[r * (r + 1) / 2 + r] = rr;
        if (tid == 0) { s.piv[r] = best; s.selpos[best] = r; }
#pragma unroll
        for (int k = 0; k < 2; k++)
            if (pos[k] == -1 && rb + rpg * k == best) { pos[k] = r; nrm[k] = -1.0; }
        // every open row: c = a . q_r (from the unscaled residual), its R12 entry; squared
        // residual norm -= c^2
        double part[2];
        id3_rows_any<false, K::SMIN, K::NKMAX>(s, s.res, S, rb, rpg, sub, nk, part);
        bv = -1.f;
        bi = INT_MAX;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const float c = (float)part[k] * inv;
            if (pos[k] == -1) {
                nrm[k] = fmax(nrm[k] - (double)c * (double)c, 0.0);
                if (sub == 0) {
                    s.C[(rb + rpg * k) * CS + r] = c;
                    const float nv = (float)nrm[k];
                    if (nv > bv) { bv = nv; bi = rb + rpg * k; }
                }
            }
        }
        warp_argmax(bv, bi);
        buf ^= 1;
        if (lane == 0) { s.bv[buf][wid] = bv; s.bi[buf][wid] = bi; }
        r++;
        __syncthreads();
    }
    __syncthreads();
    // skeleton and rank, published before the rest (the parent's candidates)
    for (int k = tid; k < r; k += THREADS) {
        const int a = s.piv[k];
        float4 x;
        if (LEAVES) x = xt[s0 + a];
        else {
            int c = 0;
            while (a >= s.coff[c + 1]) c++;
            x = __ldcg(skel + (size_t)(cfirst + c) * MAXR + (a - s.coff[c]));
        }
        skel[(size_t)t * MAXR + k] = x;
    }
    if (tid == 0) g.rank[t] = r;
    if (!LEAVES) {
        __syncthreads();
        if (tid == 0) dep_publish(dp, t);
    }
    // U = R12 times R11^-1 for the open rows (back substitution, one thread per row), the
    // pivot rows rows of the identity
    for (int a = tid; a < m; a += THREADS) {
        float *u = s.C + a * CS;
        const int sp = s.selpos[a];
        if (sp >= 0) {
            for (int i = 0; i < r; i++) u[i] = i == sp ? 1.f : 0.f;
        } else {
            for (int k = r - 1; k >= 0; k--) {
                const float *col = s.R11 + k * (k + 1) / 2;
                const float uk = u[k] / col[k];
                u[k] = uk;
                for (int i = 0; i < k; i++) u[i] = fmaf(-col[i], uk, u[i]);
            }
        }
    }
    if (!LEAVES && tid < nch && !tv.leaf[cfirst + tid]) dep_wait_y0(dp, cfirst + tid);
    __syncthreads();
    for (int idx = tid; idx < m * r; idx += THREADS) {
        const int a = idx / r, k = idx - a * r;
        U[(size_t)a * MAXR + k] = s.C[a * CS + k];
    }
    // upward coefficients y0 = U^T (the leaf's [1 | x] | the children's y0): groups of RG
    // threads over k and THREADS / RG groups over the rows, summed in a fixed order
    {
        float4 *part = reinterpret_cast<float4 *>(s.Q);
        const int RG = r <= 16 ? 16 : (r <= 32 ? 32 : 64);
        const int C = THREADS / RG, kk = tid % RG, cg = tid / RG;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        if (kk < r) {
            for (int a = cg; a < m; a += C) {
                const float w = s.C[a * CS + kk];
                if (LEAVES) {
                    const float4 x = xt[s0 + a];
                    acc.x += w;
                    acc.y = fmaf(w, x.x, acc.y);
                    acc.z = fmaf(w, x.y, acc.z);
                    acc.w = fmaf(w, x.z, acc.w);
                } else {
                    int c = 0;
                    while (a >= s.coff[c + 1]) c++;
                    fma4(acc, w, __ldcg(g.y0 + (size_t)(cfirst + c) * MAXR + (a - s.coff[c])));
                }
            }
        }
        part[tid] = acc;
        __syncthreads();
        if (tid < r) {
            float4 y = part[tid];
            for (int c = 1; c < C; c++) add4(y, part[c * RG + tid]);
            g.y0[(size_t)t * MAXR + tid] = y;
        }
    }
    if (!LEAVES) {
        __syncthreads();
        if (tid == 0) dep_publish_y0(dp, t);
    }
}

// ---------------------------------------------------------------------------------
// product kernels
// ---------------------------------------------------------------------------------
struct ProdArgs {
    TreeView tv;
    const void *xt;
    const void *skel;
    const int *rank;
    const long long *rowoff;
    const float *U;
    float4 *y0, *y1, *yp;
    const int *far_ptr, *far_idx, *near_ptr, *near_idx;
    const float4 *xin;   // input columns in tree order, or null for [1 | coordinates]
};

template <int D>
__device__ __forceinline__ float4 input_at(const ProdArgs &g, const typename Dim<D>::vec *xt, int j);

template <int D>
__device__ __forceinline__ float4 with_one(const Vec<D> &x)
{
    if constexpr (D == 2) return make_float4(1.f, x.x, x.y, 0.f);
    else return make_float4(1.f, x.x, x.y, x.z);
}
template <int D>
__device__ __forceinline__ float4 input_at(const ProdArgs &g, const typename Dim<D>::vec *xt, int j)
{
    return g.xin ? g.xin[j] : with_one<D>(xt[j]);
}

// upward pass, one warp per node of `level`: y0[t] = U_t^T (leaf points | children's y0)
template <int D>
__global__ void __launch_bounds__(256) k_up(int level, ProdArgs g)
{
    constexpr int MAXR = Dim<D>::MAXR;
    const TreeView &tv = g.tv;
    const Vec<D> *xt = (const Vec<D> *)g.xt;
    const int lb = tv.info->level_begin[level], nl = tv.info->n_level_nodes[level];
    const int lane = threadIdx.x & 31;
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nl; j += (gridDim.x * blockDim.x) >> 5) {
        const int t = lb + j;
        const int r = g.rank[t];
        const float *U = g.U + g.rowoff[t] * MAXR;
        float4 acc[MAXR / 32];
        for (int h = 0; h < MAXR / 32; h++) acc[h] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (tv.leaf[t]) {
            const int m = tv.end[t] - tv.start[t];
            for (int a = 0; a < m; a++) {
                const float4 in = input_at<D>(g, xt, tv.start[t] + a);
                for (int h = 0; h < MAXR / 32; h++) {
                    const int k = lane + 32 * h;
                    if (k < r) fma4(acc[h], U[(size_t)a * MAXR + k], in);
                }
            }
        } else {
            int a = 0;
            for (int c = tv.fchild[t]; c < tv.fchild[t] + tv.nchild[t]; c++) {
                for (int kk = 0; kk < g.rank[c]; kk++, a++) {
                    const float4 in = g.y0[(size_t)c * MAXR + kk];
                    for (int h = 0; h < MAXR / 32; h++) {
                        const int k = lane + 32 * h;
                        if (k < r) fma4(acc[h], U[(size_t)a * MAXR + k], in);
                    }
                }
            }
        }
        for (int h = 0; h < MAXR / 32; h++) {
            const int k = lane + 32 * h;
            if (k < r) g.y0[(size_t)t * MAXR + k] = acc[h];
        }
    }
}

// far field onto compressed targets, one warp per node at level >= 2:
//   same-level partner  : y1[t] += K(J_t, J_s) y0[s]
//   coarser leaf partner: y1[t] += K(J_t, X_s) [1 | x_s]
template <int D>
__global__ void __launch_bounds__(256) k_far_c(int first, int n_node, ProdArgs g)
{
    constexpr int MAXR = Dim<D>::MAXR;
    const TreeView &tv = g.tv;
    const Vec<D> *xt = (const Vec<D> *)g.xt;
    const Vec<D> *skel = (const Vec<D> *)g.skel;
    const int lane = threadIdx.x & 31;
    for (int t = first + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); t < n_node;
         t += (gridDim.x * blockDim.x) >> 5) {
        const int r = g.rank[t], lt = tv.level[t];
        if (r <= 32) {
            // rank <= 32: groups of rp lanes (rp = r rounded up to a power of two) take one
            // target slot each and the warp's 32 / rp groups split the sources; the group sums
            // meet by shuffles in a fixed order
            int rp = 1;
            while (rp < r) rp <<= 1;
            const int S = 32 / rp, k = lane % rp, sub = lane / rp;
            const Vec<D> Jk = skel[(size_t)t * MAXR + (k < r ? k : 0)];
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int e = g.far_ptr[t]; e < g.far_ptr[t + 1]; e++) {
                const int s = g.far_idx[e];
                const int ls = tv.level[s];
                if (ls == lt) {
                    const int rs = g.rank[s];
                    for (int b = sub; b < rs; b += S)
                        fma4(acc, rkernel(dist2(Jk, skel[(size_t)s * MAXR + b])), g.y0[(size_t)s * MAXR + b]);
                } else if (ls < lt) {
                    for (int j = tv.start[s] + sub; j < tv.end[s]; j += S)
                        fma4(acc, rkernel(dist2(Jk, xt[j])), input_at<D>(g, xt, j));
                }
            }
            for (int o = rp; o < 32; o <<= 1) {
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
                acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
                acc.w += __shfl_xor_sync(0xffffffffu, acc.w, o);
            }
            if (sub == 0 && k < r) g.y1[(size_t)t * MAXR + k] = acc;
            continue;
        }
        Vec<D> J[MAXR / 32];
        float4 acc[MAXR / 32];
        for (int h = 0; h < MAXR / 32; h++) {
            const int k = lane + 32 * h;
            J[h] = skel[(size_t)t * MAXR + (k < r ? k : 0)];
            acc[h] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        for (int e = g.far_ptr[t]; e < g.far_ptr[t + 1]; e++) {
            const int s = g.far_idx[e];
            const int ls = tv.level[s];
            if (ls == lt) {
                const int rs = g.rank[s];
                for (int b = 0; b < rs; b++) {
                    const Vec<D> js = skel[(size_t)s * MAXR + b];
                    const float4 y = g.y0[(size_t)s * MAXR + b];
                    for (int h = 0; h < MAXR / 32; h++) fma4(acc[h], rkernel(dist2(J[h], js)), y);
                }
            } else if (ls < lt) {
                for (int j = tv.start[s]; j < tv.end[s]; j++) {
                    const Vec<D> x = xt[j];
                    const float4 y = input_at<D>(g, xt, j);
                    for (int h = 0; h < MAXR / 32; h++) fma4(acc[h], rkernel(dist2(J[h], x)), y);
                }
            }
        }
        for (int h = 0; h < MAXR / 32; h++) {
            const int k = lane + 32 * h;
            if (k < r) g.y1[(size_t)t * MAXR + k] = acc[h];
        }
    }
}

// near field onto a leaf's points (one CTA per leaf, sources tiled through shared memory):
//   near partner           : yp[i] += sum_{j != i} K(x_i, x_j) [1 | x_j]
//   finer far partner (s)  : yp[i] += K(x_i, J_s) y0[s]
// NC = number of accumulated columns (3 in 2D for [1 | x y], 4 in 3D or for general inputs);
// only the leaf's own tiles test for the diagonal.
template <int NC>
__device__ __forceinline__ void acc_cols(float4 &acc, float w, const float4 &v)
{
    acc.x = fmaf(w, v.x, acc.x);
    acc.y = fmaf(w, v.y, acc.y);
    acc.z = fmaf(w, v.z, acc.z);
    if (NC == 4) acc.w = fmaf(w, v.w, acc.w);
}

// Parts of the leaf targets' sums: NEAR_ALL = the near blocks and the far entries whose source
// is finer than the leaf (through the source's skeleton and upward coefficients), assigned;
// NEAR_BLOCKS = the near blocks alone (tree, points and lists only: no basis), assigned;
// NEAR_FINE = the finer far entries alone, added.
constexpr int NEAR_ALL = 0, NEAR_BLOCKS = 1, NEAR_FINE = 2;

// whether leaf t has a far entry whose source is finer (every thread computes the same)
__device__ __forceinline__ bool has_fine_far(const ProdArgs &g, int t, int lt)
{
    for (int e = g.far_ptr[t]; e < g.far_ptr[t + 1]; e++)
        if (g.tv.level[g.far_idx[e]] > lt) return true;
    return false;
}

template <int D, int NC, int PART = NEAR_ALL>
__global__ void __launch_bounds__(NEAR_THREADS) k_near(ProdArgs g)
{
    constexpr int MAXR = Dim<D>::MAXR;
    const TreeView &tv = g.tv;
    const int t = blockIdx.x;
    if (!tv.leaf[t]) return;
    const Vec<D> *xt = (const Vec<D> *)g.xt;
    const Vec<D> *skel = (const Vec<D> *)g.skel;
    __shared__ Vec<D> sx[NEAR_THREADS];
    __shared__ float4 sxin[NEAR_THREADS];
    __shared__ float4 sy[MAXR];
    const int s0 = tv.start[t], cnt = tv.end[t] - s0, lt = tv.level[t];
    if (PART == NEAR_FINE && !has_fine_far(g, t, lt)) return;
    for (int chunk = 0; chunk < cnt; chunk += NEAR_THREADS) {
        const int i = s0 + chunk + threadIdx.x;
        const bool valid = chunk + (int)threadIdx.x < cnt;
        const Vec<D> xi = xt[valid ? i : s0];
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int e = g.near_ptr[t]; PART != NEAR_FINE && e < g.near_ptr[t + 1]; e++) {
            const int s = g.near_idx[e];
            const int ss = tv.start[s], sc = tv.end[s] - ss;
            for (int tile = 0; tile < sc; tile += NEAR_THREADS) {
                __syncthreads();
                if ((int)threadIdx.x < sc - tile) {
                    sx[threadIdx.x] = xt[ss + tile + threadIdx.x];
                    sxin[threadIdx.x] = input_at<D>(g, xt, ss + tile + threadIdx.x);
                }
                __syncthreads();
                const int lim = min(NEAR_THREADS, sc - tile);
                if (s == t) {
                    const int self = i - (ss + tile);
                    for (int j = 0; j < lim; j++) {
                        float w = rkernel(dist2(xi, sx[j]));
                        w = (j == self) ? 0.f : w;
                        acc_cols<NC>(acc, w, sxin[j]);
                    }
                } else {
#pragma unroll 4
                    for (int j = 0; j < lim; j++) acc_cols<NC>(acc, rkernel(dist2(xi, sx[j])), sxin[j]);
                }
            }
        }
        for (int e = g.far_ptr[t]; PART != NEAR_BLOCKS && e < g.far_ptr[t + 1]; e++) {
            const int s = g.far_idx[e];
            if (tv.level[s] <= lt) continue;
            const int rs = g.rank[s];
            __syncthreads();
            for (int b = threadIdx.x; b < rs; b += NEAR_THREADS) {
                sx[b] = skel[(size_t)s * MAXR + b];
                sy[b] = g.y0[(size_t)s * MAXR + b];
            }
            __syncthreads();
            for (int b = 0; b < rs; b++) acc_cols<NC>(acc, rkernel(dist2(xi, sx[b])), sy[b]);
        }
        if (valid) {
            if (PART == NEAR_FINE) add4(acc, g.yp[i]);
            g.yp[i] = acc;
        }
    }
}

// Near field of the 2D force product ([1 | x y] columns), two targets per thread with the
// paired FP32 instructions: thread `tid` owns the leaf's points tid and tid + NEAR2_THREADS of
// each chunk of 2 * NEAR2_THREADS. Sources are staged with each coordinate duplicated
// ((x, x), (y, y)), so one shared-memory load feeds both targets; per source and target pair
// the kernel issues 5 arithmetic instructions and 2 reciprocals instead of 10 and 2.
// Same sums, same order of sources, as k_near.
constexpr int NEAR2_THREADS = 64;
constexpr int NEAR2_TILE = 2 * NEAR2_THREADS;

template <int PART = NEAR_ALL>
__global__ void __launch_bounds__(NEAR2_THREADS) k_near2d(ProdArgs g)
{
    constexpr int MAXR = Dim<2>::MAXR;
    const TreeView &tv = g.tv;
    const int t = blockIdx.x;
    if (!tv.leaf[t]) return;
    const float2 *xt = (const float2 *)g.xt;
    const float2 *skel = (const float2 *)g.skel;
    __shared__ float4 sxy[NEAR2_TILE];      // (x, x, y, y)
    __shared__ float4 sw01[MAXR];           // (w0, w0, w1, w1) of a skeleton source
    __shared__ float2 sw2[MAXR];            // (w2, w2)
    const int tid = threadIdx.x;
    const int s0 = tv.start[t], cnt = tv.end[t] - s0, lt = tv.level[t];
    if (PART == NEAR_FINE && !has_fine_far(g, t, lt)) return;
    for (int chunk = 0; chunk < cnt; chunk += NEAR2_TILE) {
        const int a0 = chunk + tid, a1 = a0 + NEAR2_THREADS;
        const float2 x0 = xt[s0 + (a0 < cnt ? a0 : 0)], x1 = xt[s0 + (a1 < cnt ? a1 : 0)];
        const F2 ax = f2_pack(x0.x, x1.x), ay = f2_pack(x0.y, x1.y);
        F2 acc0 = f2_pack(0.f, 0.f), accx = acc0, accy = acc0;
        for (int e = g.near_ptr[t]; PART != NEAR_FINE && e < g.near_ptr[t + 1]; e++) {
            const int s = g.near_idx[e];
            const int ss = tv.start[s], sc = tv.end[s] - ss;
            for (int tile = 0; tile < sc; tile += NEAR2_TILE) {
                __syncthreads();
                for (int b = tid; b < NEAR2_TILE && b < sc - tile; b += NEAR2_THREADS) {
                    const float2 p = xt[ss + tile + b];
                    sxy[b] = make_float4(p.x, p.x, p.y, p.y);
                }
                __syncthreads();
                const int lim = min(NEAR2_TILE, sc - tile);
                if (s == t) {
                    const int self0 = a0 - tile, self1 = a1 - tile;
                    for (int j = 0; j < lim; j++) {
                        const float4 q = sxy[j];
                        const F2 sx = f2_pack(q.x, q.y), sy = f2_pack(q.z, q.w);
                        F2 w = f2_rkernel(ax, ay, sx, sy);
                        float w0, w1;
                        f2_unpack(w, w0, w1);
                        w = f2_pack(j == self0 ? 0.f : w0, j == self1 ? 0.f : w1);
                        acc0 = f2_add(acc0, w);
                        accx = f2_fma(w, sx, accx);
                        accy = f2_fma(w, sy, accy);
                    }
                } else {
#pragma unroll 4
                    for (int j = 0; j < lim; j++) {
                        const float4 q = sxy[j];
                        const F2 sx = f2_pack(q.x, q.y), sy = f2_pack(q.z, q.w);
                        const F2 w = f2_rkernel(ax, ay, sx, sy);
                        acc0 = f2_add(acc0, w);
                        accx = f2_fma(w, sx, accx);
                        accy = f2_fma(w, sy, accy);
                    }
                }
            }
        }
        for (int e = g.far_ptr[t]; PART != NEAR_BLOCKS && e < g.far_ptr[t + 1]; e++) {
            const int s = g.far_idx[e];
            if (tv.level[s] <= lt) continue;
            const int rs = g.rank[s];
            __syncthreads();
            for (int b = tid; b < rs; b += NEAR2_THREADS) {
                const float2 p = skel[(size_t)s * MAXR + b];
                const float4 y = g.y0[(size_t)s * MAXR + b];
                sxy[b] = make_float4(p.x, p.x, p.y, p.y);
                sw01[b] = make_float4(y.x, y.x, y.y, y.y);
                sw2[b] = make_float2(y.z, y.z);
            }
            __syncthreads();
            for (int b = 0; b < rs; b++) {
                const float4 q = sxy[b];
                const float4 y01 = sw01[b];
                const float2 y2 = sw2[b];
                const F2 w = f2_rkernel(ax, ay, f2_pack(q.x, q.y), f2_pack(q.z, q.w));
                acc0 = f2_fma(w, f2_pack(y01.x, y01.y), acc0);
                accx = f2_fma(w, f2_pack(y01.z, y01.w), accx);
                accy = f2_fma(w, f2_pack(y2.x, y2.y), accy);
            }
        }
        float c00, c01, cx0, cx1, cy0, cy1;
        f2_unpack(acc0, c00, c01);
        f2_unpack(accx, cx0, cx1);
        f2_unpack(accy, cy0, cy1);
        float4 o0 = make_float4(c00, cx0, cy0, 0.f), o1 = make_float4(c01, cx1, cy1, 0.f);
        if (PART == NEAR_FINE) {
            if (a0 < cnt) add4(o0, g.yp[s0 + a0]);
            if (a1 < cnt) add4(o1, g.yp[s0 + a1]);
        }
        if (a0 < cnt) g.yp[s0 + a0] = o0;
        if (a1 < cnt) g.yp[s0 + a1] = o1;
    }
}

// downward pass of node t (one warp): the node's y1 through U onto its leaf points (yp) or
// its children's y1. y1 is staged in the warp's slice of shared memory (sy, MAXR entries); lane
// a takes candidate row a and reads its U row four entries at a time. FRESH: y1 is read
// through L2 (written in the same launch).
template <int D, bool FRESH>
__device__ __forceinline__ void down_node(const ProdArgs &g, int t, int lane, float4 *sy)
{
    constexpr int MAXR = Dim<D>::MAXR;
    const TreeView &tv = g.tv;
    const int r = g.rank[t];
    const float *U = g.U + g.rowoff[t] * MAXR;
    for (int k = lane; k < r; k += 32) {
        const float4 *src = g.y1 + (size_t)t * MAXR + k;
        sy[k] = FRESH ? __ldcg(src) : *src;
    }
    __syncwarp();
    const bool isleaf = tv.leaf[t] != 0;
    int m = 0;
    if (isleaf) m = tv.end[t] - tv.start[t];
    else for (int c = tv.fchild[t]; c < tv.fchild[t] + tv.nchild[t]; c++) m += g.rank[c];
    const int r4 = r & ~3;
    for (int a0 = 0; a0 < m; a0 += 32) {
        const int a = a0 + lane;
        if (a >= m) break;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        const float *u = U + (size_t)a * MAXR;
        for (int k = 0; k < r4; k += 4) {
            const float4 w = *reinterpret_cast<const float4 *>(u + k);
            fma4(acc, w.x, sy[k]);
            fma4(acc, w.y, sy[k + 1]);
            fma4(acc, w.z, sy[k + 2]);
            fma4(acc, w.w, sy[k + 3]);
        }
        for (int k = r4; k < r; k++) fma4(acc, u[k], sy[k]);
        if (isleaf) {
            float4 o = g.yp[tv.start[t] + a];
            add4(o, acc);
            g.yp[tv.start[t] + a] = o;
        } else {
            int c = tv.fchild[t], aa = a;
            while (aa >= g.rank[c]) { aa -= g.rank[c]; c++; }
            float4 *dst = g.y1 + (size_t)c * MAXR + aa;
            float4 o = FRESH ? __ldcg(dst) : *dst;
            add4(o, acc);
            *dst = o;
        }
    }
    __syncwarp();
}

// downward pass of every internal node at level >= 2 in one dependency-ordered launch
// (persistent warps, items in increasing node id): a node waits for its parent's push
template <int D>
__global__ void __launch_bounds__(256) k_down_internal(int n_item, const int *__restrict__ items, ProdArgs g,
                                                        DepArgs dp)
{
    __shared__ float4 sy[256 / 32][Dim<D>::MAXR];
    const int lane = threadIdx.x & 31;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(dp.ticket, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n_item) break;
        const int t = items[item];
        const int p = g.tv.parent[t];
        if (lane == 0 && g.tv.level[p] >= MIN_ADM_LEVEL) dep_wait(dp, p);
        __syncwarp();
        down_node<D, true>(g, t, lane, sy[threadIdx.x >> 5]);
        __syncwarp();
        if (lane == 0) dep_publish(dp, t);
    }
}

// downward pass of every leaf at level >= 2 (after the internal nodes)
template <int D>
__global__ void __launch_bounds__(256) k_down_leaves(ProdArgs g)
{
    __shared__ float4 sy[256 / 32][Dim<D>::MAXR];
    const TreeView &tv = g.tv;
    const int lb = tv.info->level_begin[MIN_ADM_LEVEL];
    const int nl = tv.info->n_node - lb;
    const int lane = threadIdx.x & 31;
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nl; j += (gridDim.x * blockDim.x) >> 5) {
        const int t = lb + j;
        if (tv.leaf[t]) down_node<D, false>(g, t, lane, sy[threadIdx.x >> 5]);
    }
}

template <int D>
__global__ void k_split_out(int n, const float4 *__restrict__ yp, float *__restrict__ s, Vec<D> *__restrict__ v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = yp[i];
        s[i] = a.x;
        Vec<D> o;
        if constexpr (D == 2) o = make_float2(a.y, a.z);
        else o = make_float4(a.y, a.z, a.w, 0.f);
        v[i] = o;
    }
}

inline int grid_for(long long work, int block, int cap = 148 * 16)
{
    long long g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------
template <int D>
class H2Impl final : public H2Matrix {
public:
    ~H2Impl() override
    {
        if (counts_ev_) cudaEventDestroy(counts_ev_);
        if (st2_) {
            cudaStreamSynchronize(st2_);
            cudaStreamDestroy(st2_);
        }
        if (fork_ev_) cudaEventDestroy(fork_ev_);
        if (near_ev_) cudaEventDestroy(near_ev_);
        if (lists_ev_) cudaEventDestroy(lists_ev_);
    }

    H2Impl(int n, cudaStream_t st) : n_(n), st_(st)
    {
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st2_, cudaStreamNonBlocking));
        TSNE_CUDA_CHECK(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
        TSNE_CUDA_CHECK(cudaEventCreateWithFlags(&near_ev_, cudaEventDisableTiming));
        TSNE_CUDA_CHECK(cudaEventCreateWithFlags(&lists_ev_, cudaEventDisableTiming));
        keys_in_.exact(n); keys_.exact(n); idx_in_.exact(n); perm_.exact(n); xt_.exact(n);
        yp_.exact(n); s_.exact(n); v_.exact(n);
        bbox_part_.exact((size_t)BBOX_BLOCKS * (2 * D + 1));
        delta_.exact((size_t)n + 1);
        fm_.exact(n);
        blkcnt_.exact((size_t)ceil_div(n, TREE_BLOCK) * 64);
        blkoff_.exact((size_t)ceil_div(n, TREE_BLOCK) * 64);
        btot_.exact(64);
        ticket_.exact(1);
        info_.exact(1);
        TSNE_CUDA_CHECK(cudaMemsetAsync(info_.p, 0, sizeof(TreeInfo), st_));
        TSNE_CUDA_CHECK(cudaEventCreateWithFlags(&counts_ev_, cudaEventDisableTiming));
        size_t b1 = 0, b2 = 0;
        TSNE_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, b1, keys_in_.p, keys_.p, idx_in_.p,
                                                        perm_.p, n, 0, D * Dim<D>::L, st_));
        TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(nullptr, b2, (int *)nullptr, (int *)nullptr,
                                                      n + 1, st_));
        sort_bytes_ = b1;
        cub_tmp_.exact(std::max(b1, b2) + 256);
        cap_node_ = std::max(1024, 4 * (n / 16) + 1024);
        nset_cap_ = Dim<D>::NSET;
        alloc_nodes();
        TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_id<D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)id_smem_bytes<D>(id_mcap())));
        TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_id<D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)id_smem_bytes<D>(id_mcap())));
        TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_id2d<true, ID2_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)id2_smem(ID2_SMALL)));
        TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_id2d<true, ID2_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)id2_smem(ID2_THREADS)));
        TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_id2d<false, ID2_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)id2_smem(ID2_THREADS)));
        if (D == 3) {
            id3_attr<false, 512, ID3_ROWS>();
            id3_attr<true, 512, ID3_ROWS>();
            id3_attr<true, 256, ID3_SMALL>();
            id3_attr<true, 128, ID3_TINY>();
        }
    }

    int build(const void *Y, int leaf_size, double tol, const std::function<void()> *overlap) override
    {
        join_near();   // the side stream's near field reads the tree this build rewrites
        leaf_size_ = leaf_size;
        const int L = Dim<D>::L;
        cudaEvent_t t_tree = mark_begin();
        sec_begin();
        // One batch: root box, keys, sort, the whole tree (four kernels over the points, no level
        // loop) and the counting pass of the interaction lists (kernels read the level and node
        // counts on the device; scans run over the node capacity, whose unused tail counts are
        // zero), then a single synchronisation reads the tree, the list totals and the basis
        // rows. A full node table or a full inadmissible-source set are caught there and redone.
        bool tree_ok = false;
        for (int attempt = 0; attempt < 12; attempt++) {
            if (!tree_ok) {
                const int nblk = ceil_div(n_, TREE_BLOCK);
                k_bbox<D><<<BBOX_BLOCKS, 256, 0, st_>>>(n_, (const Vec<D> *)Y, bbox_part_.p);
                k_root<D><<<1, 256, 0, st_>>>(n_, L, BBOX_BLOCKS, bbox_part_.p, view());
                k_keys<D><<<grid_for(n_, 256), 256, 0, st_>>>(n_, L, (const Vec<D> *)Y, info_.p, keys_in_.p, idx_in_.p);
                size_t bytes = sort_bytes_;
                TSNE_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(cub_tmp_.p, bytes, keys_in_.p, keys_.p, idx_in_.p,
                                                                perm_.p, n_, 0, D * L, st_));
                k_gather<D><<<grid_for(n_ + 1, 256), 256, 0, st_>>>(n_, L, perm_.p, (const Vec<D> *)Y,
                                                                     (Vec<D> *)xt_.p, keys_.p, delta_.p);
                k_tree_marks<D><<<nblk, TREE_BLOCK, 0, st_>>>(view());
                k_tree_scan<<<64, TREE_SCAN_THREADS, 0, st_>>>(nblk, view());
                k_tree_levels<<<1, 32, 0, st_>>>(view());
                k_tree_emit<D><<<nblk, TREE_BLOCK, 0, st_>>>(view());
                k_tree_finish<D><<<grid_for(cap_node_, 256, 148 * 8), 256, 0, st_>>>(view());
                launches_ += 10 + 4;
                tree_ok = true;
            }
            launch_list_counts();
            TSNE_CUDA_CHECK(cudaMemcpyAsync(hinfo_.p, info_.p, sizeof(TreeInfo), cudaMemcpyDeviceToHost, st_));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(&htot_[0], far_ptr_.p + cap_node_, sizeof(int), cudaMemcpyDeviceToHost, st_));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(&htot_[1], near_ptr_.p + cap_node_, sizeof(int), cudaMemcpyDeviceToHost, st_));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(&hrows_, rowoff_.p + cap_node_, sizeof(long long), cudaMemcpyDeviceToHost, st_));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(&hint_, ipos_.p + cap_node_, sizeof(int), cudaMemcpyDeviceToHost, st_));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(&hleaf_, lpos_.p + cap_node_, sizeof(int), cudaMemcpyDeviceToHost, st_));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(&hbig_, bpos_.p + cap_node_, sizeof(int), cudaMemcpyDeviceToHost, st_));
            TSNE_CUDA_CHECK(cudaEventRecord(counts_ev_, st_));
            if (overlap != nullptr && *overlap) {
                (*overlap)();
                overlap = nullptr;
            }
            TSNE_CUDA_CHECK(cudaEventSynchronize(counts_ev_));
            const TreeInfo &I = *hinfo_.p;
            if (I.nonfinite) return -1;
            if (I.pad[1]) {   // a dependency wait of an earlier launch gave up
                fprintf(stderr, "tsne_h2pack: an H2 kernel gave up waiting for a tree dependency\n");
                return -2;
            }
            if (I.pad[0]) {   // node table full: grow and start over
                cap_node_ *= 2;
                alloc_nodes();
                tree_ok = false;
                continue;
            }
            if (I.nset_overflow) {   // inadmissible-source set full: grow, recount
                nset_cap_ *= 2;
                alloc_lists();
                if (attempt < 11) continue;
            }
            break;
        }
        mark_end(t_tree, 0);
        sec_end("tree+counts");
        const TreeInfo &I = *hinfo_.p;
        n_node_ = I.n_node;
        max_level_ = I.max_level;
        last_max_level_ = max_level_;
        stats_.n_node = n_node_;
        stats_.max_level = max_level_;
        stats_.max_leaf = I.max_leaf;
        if (max_level_ <= 2) { built_ = false; return 1; }

        // The list write (and in 3D the segmented sort of each target's entries) needs only the
        // count pass, and the bases read no list, so it runs on the side stream beside the leaf
        // bases; the near blocks follow it there. Its buffers are allocated first, in the
        // workspace stream's order (the stream-ordered pool), and the side stream starts from
        // that point. Readers on the workspace stream join it first (join_lists).
        stats_.n_far = htot_[0];
        stats_.n_near = htot_[1];
        far_idx_.ensure(std::max(1, htot_[0]));
        near_idx_.ensure(std::max(1, htot_[1]));
        if (D == 3) {
            sort_reserve(far_idx_, far_alt_, htot_[0], far_ptr_.p);
            sort_reserve(near_idx_, near_alt_, htot_[1], near_ptr_.p);
        }
        {
            TSNE_CUDA_CHECK(cudaEventRecord(fork_ev_, st_));
            TSNE_CUDA_CHECK(cudaStreamWaitEvent(st2_, fork_ev_, 0));
            cudaEvent_t t_lists = mark_begin(st2_);
            ListOut lo = list_out(1);
            if (D == 2 && !I.pad[2]) {
                k_lists_compact<<<grid_for((long long)n_node_ * 32, 256, 148 * 8), 256, 0, st2_>>>(view(), lo);
            } else {
                k_lists_write<D><<<grid_for(n_node_, 128, 148 * 8), 128, 0, st2_>>>(n_node_, view(), lo);
            }
            launches_++;
            if (D == 3) {
                sort_segments(far_idx_, far_alt_, htot_[0], far_ptr_.p, st2_);
                sort_segments(near_idx_, near_alt_, htot_[1], near_ptr_.p, st2_);
            }
            mark_end(t_lists, 1, st2_);
            TSNE_CUDA_CHECK(cudaEventRecord(lists_ev_, st2_));
            lists_pending_ = true;
        }

        // bases, bottom-up
        cudaEvent_t t_bases = mark_begin();
        constexpr int MAXR = Dim<D>::MAXR, P = Dim<D>::NPROXY;
        rank_.exact(n_node_);
        TSNE_CUDA_CHECK(cudaMemsetAsync(rank_.p, 0, sizeof(int) * n_node_, st_));
        skel_.ensure((size_t)n_node_ * MAXR);
        y0_.ensure((size_t)n_node_ * MAXR);
        y1_.ensure((size_t)n_node_ * MAXR);
        U_.ensure((size_t)std::max<long long>(hrows_, 1) * MAXR);
        const int mcap = id_mcap();
        const bool id3_path = D == 3 && id3_;   // no stored matrix, except for leaves above ID3_ROWS
        const bool need_glob = id3_path ? stats_.max_leaf > ID3_ROWS : stats_.max_leaf > mcap || (1 << D) * MAXR > mcap;
        if (need_glob) {
            gA_.ensure((size_t)std::max<long long>(hrows_, 1) * (P + 1));
            gnrm_.ensure(std::max<long long>(hrows_, 1));
            gsel_.ensure(std::max<long long>(hrows_, 1));
            gcand_.ensure(std::max<long long>(hrows_, 1));
        }
        const float tol2 = (float)((tol * ID_TOL_FACTOR) * (tol * ID_TOL_FACTOR));
        // leaves: one launch, shared memory sized for the largest leaf
        const int mleaf = std::max(1, std::min(stats_.max_leaf, mcap));
        IdArgs il{view(), xt_.p, skel_.p, rank_.p, rowoff_.p, U_.p, gA_.p, gnrm_.p, gsel_.p, gcand_.p, mleaf, tol2,
                  y0_.p};
        const int first = I.level_begin[MIN_ADM_LEVEL];
        if (D == 2 && stats_.max_leaf <= ID2_THREADS) {
            // leaves in one launch, then the internal nodes of every level in one
            // dependency-ordered launch
            DepArgs dp{flag_.p, ticket_.p, &info_.p->pad[1], ++epoch_};
            if (hleaf_ > 0)
                k_id2d<true, ID2_SMALL><<<hleaf_, ID2_SMALL, id2_smem(ID2_SMALL), st_>>>(hleaf_, llist_.p, il, dp);
            if (hbig_ > 0)
                k_id2d<true, ID2_THREADS><<<hbig_, ID2_THREADS, id2_smem(ID2_THREADS), st_>>>(hbig_, blist_.p, il, dp);
            mark_end(t_bases, 2);
            t_bases = mark_begin();
            near_fork_point();
            if (hint_ > 0 && id_by_level_) {
                // one launch per level, deepest first (TSNE_ID_BYLEVEL=1)
                for (int l = max_level_; l >= MIN_ADM_LEVEL; l--) {
                    const int nl = I.n_level_nodes[l];
                    if (nl <= 0) continue;
                    k_id2d<false, ID2_THREADS><<<nl, ID2_THREADS, id2_smem(ID2_THREADS), st_>>>(
                        I.level_begin[l], nullptr, il, dp);
                    launches_++;
                }
            } else if (hint_ > 0) {
                TSNE_CUDA_CHECK(cudaMemsetAsync(ticket_.p, 0, sizeof(int), st_));
                DepArgs d2 = dp;
                d2.flag2 = flag2_.p;
                k_id2d<false, ID2_THREADS><<<hint_, ID2_THREADS, id2_smem(ID2_THREADS), st_>>>(hint_, ilist_.p, il, d2);
            }
            launches_ += 2;
            near_launch_side();
            mark_end(t_bases, 7);
            if (timing_) TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
            sec_end("lists+bases");
            built_ = true;
            y0_from_build_ = true;
            rank_stats_valid_ = false;
            return 0;
        }
        DepArgs dp{flag_.p, ticket_.p, &info_.p->pad[1], ++epoch_};
        if (D == 3 && id3_) {
            // recomputed-row decompositions: leaves by size (llist: at most ID3_TINY points;
            // blist: the others, up to ID3_ROWS; larger leaves, only at the depth limit, take
            // k_id), then the internal nodes in one dependency-ordered launch
            if (stats_.max_leaf <= ID3_ROWS) {
                if (hleaf_ > 0) id3_launch<true, 128, ID3_TINY>(hleaf_, llist_.p, 0, il, dp);
                if (hbig_ > 0) {
                    id3_launch<true, 256, ID3_SMALL>(hbig_, blist_.p, ID3_TINY, il, dp);
                    if (stats_.max_leaf > ID3_SMALL) id3_launch<true, 512, ID3_ROWS>(hbig_, blist_.p, ID3_SMALL, il, dp);
                }
            } else {
                k_id<D, true><<<n_node_ - first, IDG_THREADS, id_smem_bytes<D>(mleaf), st_>>>(MIN_ADM_LEVEL, il, 0,
                                                                                              nullptr, dp);
                launches_++;
            }
            mark_end(t_bases, 2);
            t_bases = mark_begin();
            near_fork_point();
            if (hint_ > 0) {
                TSNE_CUDA_CHECK(cudaMemsetAsync(ticket_.p, 0, sizeof(int), st_));
                DepArgs d2 = dp;
                d2.flag2 = flag2_.p;
                id3_launch<false, 512, ID3_ROWS>(hint_, ilist_.p, 0, il, d2);
            }
            near_launch_side();
            mark_end(t_bases, 7);
            if (timing_) TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
            sec_end("lists+bases");
            built_ = true;
            y0_from_build_ = true;
            rank_stats_valid_ = false;
            return 0;
        }
        k_id<D, true><<<n_node_ - first, IDG_THREADS, id_smem_bytes<D>(mleaf), st_>>>(MIN_ADM_LEVEL, il, 0, nullptr, dp);
        launches_++;
        mark_end(t_bases, 2);
        t_bases = mark_begin();
        // internal nodes of every level in one dependency-ordered launch (their candidates are
        // the children's skeletons)
        IdArgs ia = il;
        ia.mcap = mcap;
        if (hint_ > 0) {
            TSNE_CUDA_CHECK(cudaMemsetAsync(ticket_.p, 0, sizeof(int), st_));
            k_id<D, false><<<hint_, IDG_THREADS, id_smem_bytes<D>(mcap), st_>>>(0, ia, hint_, ilist_.p, dp);
            launches_++;
        }
        mark_end(t_bases, 7);
        if (timing_) TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        sec_end("lists+bases");
        built_ = true;
        y0_from_build_ = true;
        rank_stats_valid_ = false;
        return 0;
    }

    // counting pass of the lists (internal targets, then every leaf target), the pointer
    // scans and the basis row offsets, all over the node capacity
    void launch_list_counts()
    {
        TSNE_CUDA_CHECK(cudaMemsetAsync(far_cnt_.p, 0, sizeof(int) * (cap_node_ + 1), st_));
        TSNE_CUDA_CHECK(cudaMemsetAsync(near_cnt_.p, 0, sizeof(int) * (cap_node_ + 1), st_));
        TSNE_CUDA_CHECK(cudaMemsetAsync(rowcap_.p, 0, sizeof(int) * (cap_node_ + 1), st_));
        TSNE_CUDA_CHECK(cudaMemsetAsync(&info_.p->nset_overflow, 0, sizeof(int), st_));
        TSNE_CUDA_CHECK(cudaMemsetAsync(&info_.p->pad[2], 0, sizeof(int), st_));
        ListOut lo = list_out(0);
        TSNE_CUDA_CHECK(cudaMemsetAsync(ticket_.p, 0, sizeof(int), st_));
        DepArgs dp{flag_.p, ticket_.p, &info_.p->pad[1], ++epoch_};
        k_lists_internal<D><<<148 * 4, 256, 0, st_>>>(view(), lo, dp);
        k_lists_leaves<D><<<148 * 8, 128, 0, st_>>>(view(), lo);
        launches_ += 2;
        TSNE_CUDA_CHECK(cudaMemsetAsync(iflag_.p, 0, sizeof(int) * (cap_node_ + 1), st_));
        TSNE_CUDA_CHECK(cudaMemsetAsync(lflag_.p, 0, sizeof(int) * (cap_node_ + 1), st_));
        TSNE_CUDA_CHECK(cudaMemsetAsync(bflag_.p, 0, sizeof(int) * (cap_node_ + 1), st_));
        k_rowcap<D><<<148 * 4, 256, 0, st_>>>(view(), rowcap_.p, iflag_.p, lflag_.p, bflag_.p);
        scan_exclusive(far_cnt_.p, far_ptr_.p, cap_node_);
        scan_exclusive(near_cnt_.p, near_ptr_.p, cap_node_);
        scan_exclusive_ll(rowcap_.p, rowoff_.p, cap_node_);
        scan_exclusive(iflag_.p, ipos_.p, cap_node_);
        scan_exclusive(lflag_.p, lpos_.p, cap_node_);
        scan_exclusive(bflag_.p, bpos_.p, cap_node_);
        k_flag_list<<<148 * 4, 256, 0, st_>>>(&info_.p->n_node, iflag_.p, ipos_.p, ilist_.p);
        k_flag_list<<<148 * 4, 256, 0, st_>>>(&info_.p->n_node, lflag_.p, lpos_.p, llist_.p);
        k_flag_list<<<148 * 4, 256, 0, st_>>>(&info_.p->n_node, bflag_.p, bpos_.p, blist_.p);
        launches_ += 12;
    }

    void alloc_lists()
    {
        const size_t c = cap_node_;
        nset_.exact(c * nset_cap_);
        nset_cnt_.exact(c + 1);
        far_cnt_.exact(c + 1); near_cnt_.exact(c + 1);
        far_ptr_.exact(c + 2); near_ptr_.exact(c + 2);
        rowcap_.exact(c + 1);
        iflag_.exact(c + 1); ipos_.exact(c + 2); ilist_.exact(c + 1);
        lflag_.exact(c + 1); lpos_.exact(c + 2); llist_.exact(c + 1);
        bflag_.exact(c + 1); bpos_.exact(c + 2); blist_.exact(c + 1);
        rowoff_.exact(c + 2);
        if (D == 2) {
            far_slot_.exact(c * LIST_SLOT);
            near_slot_.exact(c * LIST_SLOT);
        }
    }

    void product_force(void *F, DevScalars *sc, double *partials, int keep_rep) override
    {
        run_product();
        cudaEvent_t t_force = mark_begin();
        k_split_out<D><<<grid_for(n_, 256), 256, 0, st_>>>(n_, yp_.p, s_.p, (Vec<D> *)v_.p);
        launch_z_force<D>(st_, n_, xt_.p, s_.p, v_.p, perm_.p, F, sc, partials, 1, keep_rep);
        launches_ += 3;
        mark_end(t_force, 6);
    }

    void product_host(std::vector<float> &s, std::vector<float> &v) override
    {
        run_product();
        k_split_out<D><<<grid_for(n_, 256), 256, 0, st_>>>(n_, yp_.p, s_.p, (Vec<D> *)v_.p);
        std::vector<float> st(n_);
        std::vector<Vec<D>> vt(n_);
        std::vector<int> perm(n_);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(st.data(), s_.p, sizeof(float) * n_, cudaMemcpyDeviceToHost, st_));
        TSNE_CUDA_CHECK(cudaMemcpyAsync(vt.data(), v_.p, sizeof(Vec<D>) * n_, cudaMemcpyDeviceToHost, st_));
        TSNE_CUDA_CHECK(cudaMemcpyAsync(perm.data(), perm_.p, sizeof(int) * n_, cudaMemcpyDeviceToHost, st_));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        s.assign(n_, 0.f);
        v.assign((size_t)n_ * D, 0.f);
        for (int k = 0; k < n_; k++) {
            const int i = perm[k];
            s[i] = st[k];
            const float *vv = reinterpret_cast<const float *>(&vt[k]);
            for (int c = 0; c < D; c++) v[(size_t)c * n_ + i] = vv[c];
        }
    }

    void product_columns(const std::vector<float> &x_tree, std::vector<float> &y_tree) override
    {
        xin_.exact(n_);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(xin_.p, x_tree.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice, st_));
        run_product(xin_.p);
        y_tree.assign((size_t)n_ * 4, 0.f);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(y_tree.data(), yp_.p, sizeof(float4) * n_, cudaMemcpyDeviceToHost, st_));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
    }

    const int *perm_device() const override { return perm_.p; }

    const H2Stats &stats() const override
    {
        if (!rank_stats_valid_ && built_) {
            std::vector<int> r(n_node_);
            cudaStreamSynchronize(st_);
            cudaMemcpy(r.data(), rank_.p, sizeof(int) * n_node_, cudaMemcpyDeviceToHost);
            int mx = 0; double sum = 0; int cnt = 0;
            for (int x : r) if (x > 0) { mx = std::max(mx, x); sum += x; cnt++; }
            stats_.rank_max = mx;
            stats_.rank_mean = cnt ? sum / cnt : 0.0;
            rank_stats_valid_ = true;
        }
        return stats_;
    }

    void copy_tree(int *perm, double *corner, double *radius) override
    {
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        TSNE_CUDA_CHECK(cudaMemcpy(perm, perm_.p, sizeof(int) * n_, cudaMemcpyDeviceToHost));
        TreeInfo I;
        TSNE_CUDA_CHECK(cudaMemcpy(&I, info_.p, sizeof(TreeInfo), cudaMemcpyDeviceToHost));
        for (int k = 0; k < D; k++) corner[k] = I.corner[k];
        *radius = I.radius;
    }

    void copy_nodes(int *start, int *end, int *level, int *parent, int *fchild, int *nchild, int *leaf) override
    {
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        const size_t b = sizeof(int) * n_node_;
        TSNE_CUDA_CHECK(cudaMemcpy(start, start_.p, b, cudaMemcpyDeviceToHost));
        TSNE_CUDA_CHECK(cudaMemcpy(end, end_.p, b, cudaMemcpyDeviceToHost));
        TSNE_CUDA_CHECK(cudaMemcpy(level, level_.p, b, cudaMemcpyDeviceToHost));
        TSNE_CUDA_CHECK(cudaMemcpy(parent, parent_.p, b, cudaMemcpyDeviceToHost));
        TSNE_CUDA_CHECK(cudaMemcpy(fchild, fchild_.p, b, cudaMemcpyDeviceToHost));
        TSNE_CUDA_CHECK(cudaMemcpy(nchild, nchild_.p, b, cudaMemcpyDeviceToHost));
        TSNE_CUDA_CHECK(cudaMemcpy(leaf, leaf_.p, b, cudaMemcpyDeviceToHost));
    }

    void copy_lists(int *far_ptr, int *far_idx, int *near_ptr, int *near_idx) override
    {
        join_lists();
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        TSNE_CUDA_CHECK(cudaMemcpy(far_ptr, far_ptr_.p, sizeof(int) * (n_node_ + 1), cudaMemcpyDeviceToHost));
        TSNE_CUDA_CHECK(cudaMemcpy(near_ptr, near_ptr_.p, sizeof(int) * (n_node_ + 1), cudaMemcpyDeviceToHost));
        if (stats_.n_far) TSNE_CUDA_CHECK(cudaMemcpy(far_idx, far_idx_.p, sizeof(int) * stats_.n_far, cudaMemcpyDeviceToHost));
        if (stats_.n_near) TSNE_CUDA_CHECK(cudaMemcpy(near_idx, near_idx_.p, sizeof(int) * stats_.n_near, cudaMemcpyDeviceToHost));
    }

    void copy_ranks(int *rank) override
    {
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        if (built_) TSNE_CUDA_CHECK(cudaMemcpy(rank, rank_.p, sizeof(int) * n_node_, cudaMemcpyDeviceToHost));
        else for (int i = 0; i < n_node_; i++) rank[i] = 0;
    }

    int copy_bases(int *n_rows, int *max_rank, long long *row_off, float *U, float *skel) override
    {
        constexpr int MAXR = Dim<D>::MAXR;
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        if (!built_) return -1;
        *n_rows = (int)hrows_;
        *max_rank = MAXR;
        if (U == nullptr) return 0;
        TSNE_CUDA_CHECK(cudaMemcpy(row_off, rowoff_.p, sizeof(long long) * (n_node_ + 1), cudaMemcpyDeviceToHost));
        if (hrows_ > 0)
            TSNE_CUDA_CHECK(cudaMemcpy(U, U_.p, sizeof(float) * (size_t)hrows_ * MAXR, cudaMemcpyDeviceToHost));
        std::vector<Vec<D>> sk((size_t)n_node_ * MAXR);
        TSNE_CUDA_CHECK(cudaMemcpy(sk.data(), skel_.p, sizeof(Vec<D>) * sk.size(), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < sk.size(); i++) {
            const float *f = reinterpret_cast<const float *>(&sk[i]);   // x, y (, z)
            for (int k = 0; k < D; k++) skel[i * D + k] = f[k];
        }
        return 0;
    }

    long long launches() const override { return launches_; }

    int probe_dependency_timeout(int polls) override
    {
        if (n_node_ <= 0) return -1;
        // an epoch that no launch has published: the wait runs out after `polls` polls
        DepArgs dp{flag_.p, ticket_.p, &info_.p->pad[1], epoch_ + (1 << 24), polls};
        k_dep_probe<<<1, 32, 0, st_>>>(dp, 0);
        launches_++;
        return wait_failed();
    }

    int wait_failed() override
    {
        TreeInfo I;
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        TSNE_CUDA_CHECK(cudaMemcpy(&I, info_.p, sizeof(TreeInfo), cudaMemcpyDeviceToHost));
        return I.pad[1] != 0;
    }

    // TSNE_H2_TIMERS=1: device time per phase (CUDA events on the stream), summed over builds
    // and products until flush_timers() prints them
    void flush_timers() override
    {
        if (!timing_) return;
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st_));
        static const char *names[N_PHASE] = {"tree", "lists", "leaf_bases", "far", "near", "down", "force",
                                             "internal_bases"};
        for (auto &m : marks_) {
            float ms = 0.f;
            TSNE_CUDA_CHECK(cudaEventElapsedTime(&ms, m.a, m.b));
            phase_ms_[m.phase] += ms;
            cudaEventDestroy(m.a);
            cudaEventDestroy(m.b);
        }
        marks_.clear();
        printf("H2TIMERS");
        for (int i = 0; i < N_PHASE; i++) printf(" %s=%.3f", names[i], phase_ms_[i] * 1e-3);
        printf(" (s)\n");
        fflush(stdout);
        for (double &x : phase_ms_) x = 0.0;
    }

private:
    static constexpr int BBOX_BLOCKS = 148 * 2;
    static constexpr int N_PHASE = 8;
    struct Mark { cudaEvent_t a, b; int phase; };
    bool timing_ = getenv("TSNE_H2_TIMERS") && atoi(getenv("TSNE_H2_TIMERS")) != 0;
    bool id_by_level_ = getenv("TSNE_ID_BYLEVEL") && atoi(getenv("TSNE_ID_BYLEVEL")) != 0;
    // 3D bases: recomputed rows (k_id3, default) or rows held in memory (k_id, TSNE_ID3=0)
    bool id3_ = !(getenv("TSNE_ID3") && atoi(getenv("TSNE_ID3")) == 0);
    std::vector<Mark> marks_;
    double phase_ms_[N_PHASE] = {0, 0, 0, 0, 0, 0, 0, 0};
    cudaEvent_t mark_begin(cudaStream_t st = nullptr)
    {
        cudaEvent_t e = nullptr;
        if (!timing_) return e;
        TSNE_CUDA_CHECK(cudaEventCreate(&e));
        TSNE_CUDA_CHECK(cudaEventRecord(e, st ? st : st_));
        return e;
    }
    // host wall time of one build section; sections slower than 10 ms are reported
    std::chrono::steady_clock::time_point sec_t0_;
    void sec_begin() { if (timing_) sec_t0_ = std::chrono::steady_clock::now(); }
    void sec_end(const char *name)
    {
        if (!timing_) return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - sec_t0_).count();
        if (ms > 10.0) printf("H2SLOW %s %.1f ms (n_node %d, max_leaf %d, far %d, near %d, nset_cap %d, cap_node %d)\n", name, ms,
                              n_node_, stats_.max_leaf, htot_[0], htot_[1], nset_cap_, cap_node_);
        sec_t0_ = std::chrono::steady_clock::now();
    }
    void mark_end(cudaEvent_t a, int phase, cudaStream_t st = nullptr)
    {
        if (!timing_) return;
        cudaEvent_t b;
        TSNE_CUDA_CHECK(cudaEventCreate(&b));
        TSNE_CUDA_CHECK(cudaEventRecord(b, st ? st : st_));
        marks_.push_back({a, b, phase});
    }

    template <bool LEAVES, int THREADS, int ROWS>
    static void id3_attr()
    {
        TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_id3<LEAVES, THREADS, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(typename Id3<THREADS, ROWS>::Smem)));
    }
    template <bool LEAVES, int THREADS, int ROWS>
    void id3_launch(int n_item, const int *items, int mlo, const IdArgs &a, const DepArgs &dp)
    {
        k_id3<LEAVES, THREADS, ROWS><<<n_item, THREADS, sizeof(typename Id3<THREADS, ROWS>::Smem), st_>>>(
            n_item, items, mlo, a, dp);
        launches_++;
    }

    static int id_mcap()
    {
        // shared-memory rows of the ID: every internal node of the 2D tree (4 * MAXR rows)
        // and leaves up to that size; the 3D bound keeps the CTA under 227 KB
        return D == 2 ? (1 << D) * Dim<D>::MAXR : 240;
    }

    void alloc_nodes()
    {
        const size_t c = cap_node_;
        start_.exact(c); end_.exact(c); level_.exact(c); parent_.exact(c); fchild_.exact(c);
        nchild_.exact(c); leaf_.exact(c); ix_.exact(3 * c);
        bset_.exact(c * (Dim<D>::L + 1));
        flag_.exact(c);
        TSNE_CUDA_CHECK(cudaMemsetAsync(flag_.p, 0, sizeof(int) * c, st_));
        flag2_.exact(c);
        TSNE_CUDA_CHECK(cudaMemsetAsync(flag2_.p, 0, sizeof(int) * c, st_));
        nid_.exact(c * (Dim<D>::L + 1));
        alloc_lists();
    }

    TreeView view()
    {
        TreeView v;
        v.n = n_; v.L = Dim<D>::L; v.leaf_size = leaf_size_; v.cap_node = cap_node_; v.nset_cap = nset_cap_;
        v.keys = keys_.p; v.start = start_.p; v.end = end_.p; v.level = level_.p; v.parent = parent_.p;
        v.fchild = fchild_.p; v.nchild = nchild_.p; v.leaf = leaf_.p; v.ix = ix_.p;
        v.delta = delta_.p; v.fm = fm_.p; v.blkcnt = blkcnt_.p; v.blkoff = blkoff_.p;
        v.bset = bset_.p; v.nid = nid_.p; v.btot = btot_.p; v.info = info_.p;
        return v;
    }

    ListOut list_out(int write)
    {
        ListOut lo;
        lo.far_cnt = far_cnt_.p; lo.near_cnt = near_cnt_.p;
        lo.far_ptr = far_ptr_.p; lo.near_ptr = near_ptr_.p;
        lo.far_idx = far_idx_.p; lo.near_idx = near_idx_.p;
        lo.nset = nset_.p; lo.nset_cnt = nset_cnt_.p;
        lo.far_slot = D == 2 ? far_slot_.p : nullptr;
        lo.near_slot = D == 2 ? near_slot_.p : nullptr;
        lo.slot_over = &info_.p->pad[2];
        lo.write = write;
        return lo;
    }

    // out[0] = 0, out[i + 1] = in[0] + ... + in[i]
    void scan_exclusive(const int *in, int *out, int count)
    {
        TSNE_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(int), st_));
        size_t need = 0;
        TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(nullptr, need, in, out + 1, count, st_));
        if (need > cub_tmp_.cap) cub_tmp_.exact(need + 256);
        size_t bytes = cub_tmp_.cap;
        TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(cub_tmp_.p, bytes, in, out + 1, count, st_));
    }
    void sort_reserve(DevBuf<int> &idx, DevBuf<int> &alt, int count, const int *ptr)
    {
        if (count <= 1) return;
        alt.ensure(count);
        cub::DoubleBuffer<int> keys(idx.p, alt.p);
        size_t need = 0;
        TSNE_CUDA_CHECK(cub::DeviceSegmentedSort::SortKeys(nullptr, need, keys, count, n_node_, ptr, ptr + 1, st_));
        if (need > cub_tmp_.cap) cub_tmp_.exact(need + 256);
    }
    // ascending order inside every node's segment [ptr[t], ptr[t + 1]) of idx (count entries)
    // (sort_reserve allocates its partner buffer and scratch beforehand)
    void sort_segments(DevBuf<int> &idx, DevBuf<int> &alt, int count, const int *ptr, cudaStream_t st)
    {
        if (count <= 1) return;
        cub::DoubleBuffer<int> keys(idx.p, alt.p);
        size_t bytes = cub_tmp_.cap;
        TSNE_CUDA_CHECK(cub::DeviceSegmentedSort::SortKeys(cub_tmp_.p, bytes, keys, count, n_node_, ptr, ptr + 1, st));
        if (keys.Current() != idx.p) idx.swap(alt);
        launches_ += 2;
    }
    void scan_exclusive_ll(const int *in, long long *out, int count)
    {
        TSNE_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(long long), st_));
        size_t need = 0;
        TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(nullptr, need, in, out + 1, count, st_));
        if (need > cub_tmp_.cap) cub_tmp_.exact(need + 256);
        size_t bytes = cub_tmp_.cap;
        TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(cub_tmp_.p, bytes, in, out + 1, count, st_));
    }

    ProdArgs prod_args(const float4 *xin)
    {
        ProdArgs g;
        g.xin = xin;
        g.tv = view(); g.xt = xt_.p; g.skel = skel_.p; g.rank = rank_.p; g.rowoff = rowoff_.p; g.U = U_.p;
        g.y0 = y0_.p; g.y1 = y1_.p; g.yp = yp_.p;
        g.far_ptr = far_ptr_.p; g.far_idx = far_idx_.p; g.near_ptr = near_ptr_.p; g.near_idx = near_idx_.p;
        return g;
    }
    template <int PART>
    void launch_near(const ProdArgs &g, cudaStream_t st)
    {
        if (D == 2 && g.xin == nullptr) k_near2d<PART><<<n_node_, NEAR2_THREADS, 0, st>>>(g);
        else k_near<D, 4, PART><<<n_node_, NEAR_THREADS, 0, st>>>(g);
        launches_++;
    }
    // The near blocks of the force product ([1 | Y] columns) need only the tree, the points and
    // the near lists, so a build runs them on a side stream beside the internal bases, whose
    // dependency chain leaves SMs idle. The fork point follows the leaf bases (which fill the
    // GPU by themselves); the internal bases are queued before the near blocks, so their CTAs
    // are dispatched first. The product joins the side stream before the first kernel that
    // adds to their output (the leaves' far entries with finer sources, which read the bases,
    // then k_down_leaves).
    void near_fork_point() { TSNE_CUDA_CHECK(cudaEventRecord(fork_ev_, st_)); }
    void near_launch_side()
    {
        TSNE_CUDA_CHECK(cudaStreamWaitEvent(st2_, fork_ev_, 0));
        launch_near<NEAR_BLOCKS>(prod_args(nullptr), st2_);
        TSNE_CUDA_CHECK(cudaEventRecord(near_ev_, st2_));
        near_pending_ = true;
    }
    void join_lists()
    {
        if (!lists_pending_) return;
        TSNE_CUDA_CHECK(cudaStreamWaitEvent(st_, lists_ev_, 0));
        lists_pending_ = false;
    }
    void join_near()
    {
        join_lists();
        if (!near_pending_) return;
        TSNE_CUDA_CHECK(cudaStreamWaitEvent(st_, near_ev_, 0));
        near_pending_ = false;
    }

    void run_product(const float4 *xin = nullptr)
    {
        const bool near_done = near_pending_ && xin == nullptr;   // the side stream's near field
        if (!near_done) join_near();                              // other columns rewrite it
        else join_lists();
        const ProdArgs g = prod_args(xin);
        const TreeInfo &I = *hinfo_.p;
        if (xin != nullptr || !y0_from_build_) {
            for (int l = max_level_; l >= MIN_ADM_LEVEL; l--) {
                const int nl = I.n_level_nodes[l];
                if (nl > 0) { k_up<D><<<grid_for((long long)nl * 32, 256), 256, 0, st_>>>(l, g); launches_++; }
            }
        }
        y0_from_build_ = y0_from_build_ && xin == nullptr;
        const int first = I.level_begin[MIN_ADM_LEVEL];
        cudaEvent_t t_far = mark_begin();
        k_far_c<D><<<grid_for((long long)(n_node_ - first) * 32, 256), 256, 0, st_>>>(first, n_node_, g);
        mark_end(t_far, 3);
        launches_++;
        cudaEvent_t t_near = mark_begin();
        if (!near_done) launch_near<NEAR_ALL>(g, st_);
        mark_end(t_near, 4);
        cudaEvent_t t_down = mark_begin();
        if (hint_ > 0) {
            TSNE_CUDA_CHECK(cudaMemsetAsync(ticket_.p, 0, sizeof(int), st_));
            DepArgs dp{flag_.p, ticket_.p, &info_.p->pad[1], ++epoch_};
            k_down_internal<D><<<grid_for((long long)hint_ * 32, 256, 148 * 8), 256, 0, st_>>>(hint_, ilist_.p, g, dp);
            launches_++;
        }
        if (near_done) {
            join_near();
            launch_near<NEAR_FINE>(g, st_);
        }
        k_down_leaves<D><<<grid_for((long long)(n_node_ - first) * 32, 256), 256, 0, st_>>>(g);
        launches_++;
        mark_end(t_down, 5);
    }

    int n_;
    cudaStream_t st_;
    int leaf_size_ = 100;
    int cap_node_ = 0, nset_cap_ = 0;
    int n_node_ = 0, max_level_ = 0, last_max_level_ = 0;
    bool built_ = false;
    bool y0_from_build_ = false;   // y0 holds U^T [1 | Y] of the last build
    mutable bool rank_stats_valid_ = false;
    mutable H2Stats stats_;
    long long launches_ = 0;
    size_t sort_bytes_ = 0;
    int htot_[2] = {0, 0};
    long long hrows_ = 0;

    DevBuf<unsigned long long> keys_in_, keys_;
    DevBuf<int> idx_in_, perm_;
    DevBuf<Vec<D>> xt_;
    DevBuf<unsigned char> cub_tmp_;
    DevBuf<double> bbox_part_;
    DevBuf<TreeInfo> info_;
    HostPinned<TreeInfo> hinfo_;
    DevBuf<int> start_, end_, level_, parent_, fchild_, nchild_, leaf_, ix_;
    DevBuf<signed char> delta_;
    DevBuf<int> fm_, blkcnt_, blkoff_, bset_, nid_, btot_;
    DevBuf<int> flag_, ticket_;   // dependency-ordered launches
    DevBuf<int> flag2_;           // second flags (bases: upward coefficients final)
    cudaStream_t st2_ = nullptr;  // side stream: the list write and the near field beside the bases
    cudaEvent_t fork_ev_ = nullptr, near_ev_ = nullptr, lists_ev_ = nullptr;
    bool near_pending_ = false, lists_pending_ = false;
    DevBuf<int> far_slot_, near_slot_;   // 2D: list entries parked by the count pass
    int epoch_ = 0;
    DevBuf<int> nset_, nset_cnt_, far_cnt_, near_cnt_, far_ptr_, near_ptr_, far_idx_, near_idx_;
    DevBuf<int> far_alt_, near_alt_;   // segmented-sort partners of the 3D lists
    DevBuf<int> rowcap_;
    DevBuf<int> iflag_, ipos_, ilist_;   // internal nodes at level >= 2, in increasing id
    DevBuf<int> lflag_, lpos_, llist_;   // leaves at level >= 2 of at most LEAF_SMALL points
    DevBuf<int> bflag_, bpos_, blist_;   // the larger leaves at level >= 2
    int hint_ = 0, hleaf_ = 0, hbig_ = 0;
    cudaEvent_t counts_ev_ = nullptr;   // end of a build's count batch (host waits on it)
    DevBuf<long long> rowoff_;
    DevBuf<int> rank_;
    DevBuf<Vec<D>> skel_;
    DevBuf<float4> y0_, y1_, yp_, xin_;
    DevBuf<float> U_, s_;
    DevBuf<Vec<D>> v_;
    DevBuf<float> gA_, gnrm_;
    DevBuf<int> gsel_;
    DevBuf<Vec<D>> gcand_;
};

}  // namespace

std::unique_ptr<H2Matrix> make_h2_matrix(int d, int n, cudaStream_t st)
{
    if (d == 2) return std::unique_ptr<H2Matrix>(new H2Impl<2>(n, st));
    return std::unique_ptr<H2Matrix>(new H2Impl<3>(n, st));
}

}  // namespace tsne
