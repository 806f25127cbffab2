// The optimisation engine behind the C ABI (include/tsne_h2pack.h): one workspace per
// embedding, all state resident on the current CUDA device, the reference's schedule
// (src/tsne_h2pack.c:1652-2102) driven from the host with one stream per workspace.
#include <functional>
#include <cstring>
#include <thread>
#include <mutex>
#include <sys/mman.h>
#include <cub/cub.cuh>

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "devbuf.h"
#include "h2.h"
#include "kernels.h"
#include "attr_tiles.h"
#include "pjoint.h"
#include "../../include/tsne_h2pack.h"

using namespace tsne;

namespace {

int env_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return (v != nullptr && *v != '\0') ? atoi(v) : dflt;
}

double wall_sec()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// CSR rows padded to a multiple of 4 entries (column = the row itself, value 0) so that the
// attractive pass reads 4 entries per 128-bit load.
__global__ void k_pad_len(int n, const int *__restrict__ rp, int *__restrict__ len)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        len[i] = (rp[i + 1] - rp[i] + 3) & ~3;
}
template <typename V>
__global__ void k_pad_copy(int n, const int *__restrict__ rp, const int *__restrict__ ci, const V *__restrict__ pv,
                           const int *__restrict__ rpp, int *__restrict__ col, float *__restrict__ val)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarp = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < n; i += nwarp) {
        const int b = rp[i], len = rp[i + 1] - b, o = rpp[i], plen = rpp[i + 1] - o;
        for (int e = lane; e < plen; e += 32) {
            col[o + e] = e < len ? ci[b + e] : i;
            val[o + e] = e < len ? (float)pv[b + e] : 0.f;
        }
    }
}
__global__ void k_conv_check(int n, const float *__restrict__ Y, const float *__restrict__ Yprev, int d,
                             int vec_stride, double *__restrict__ out_max)
{
    __shared__ double sh[256];
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < d; k++) {
            const double df = (double)Y[(size_t)i * vec_stride + k] - (double)Yprev[(size_t)i * vec_stride + k];
            s += df * df;
        }
        m = fmax(m, sqrt(s));
    }
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out_max[blockIdx.x] = sh[0];
}

}  // namespace

extern "C" TSNE_API int tsne_release_cached_memory(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return -1;
    if (cudaDeviceSynchronize() != cudaSuccess) return -1;
    return cudaMemPoolTrimTo(pool, 0) == cudaSuccess ? 0 : -1;
}

namespace tsne {
void keep_pool_memory()
{
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        unsigned long long keep = ~0ULL;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done[dev] = true;
}
}  // namespace tsne

struct tsne_workspace {
    tsne_params_t params{};
    std::string prof_file;
    int n = 0, d = 0, pt_dim = 0;
    double lr = 200.0;
    sparse_matrix_t *P = nullptr;   // host P (owned, as in the reference)
    size_t vbytes = 0;              // bytes per point of the device vectors

    cudaStream_t st = nullptr;
    DevBuf<int> rp, col, rp2, col2, len, inv, order, order2;
    long long padded_nnz = 0;
    DevBuf<float> val, val2;
    DevBuf<unsigned char> Y, Yn, uY, gains, rep, frc, tmpv, Yconv;
    DevBuf<unsigned char> attr;     // attractive sums of a rebuild iteration (computed during the build)
    DevBuf<float> s;
    DevBuf<unsigned char> v;
    DevBuf<DevScalars> sc;
    HostPinned<DevScalars> hsc;
    DevBuf<double> part, zpart, klpart, convpart;
    DevBuf<unsigned char> cub_tmp;
    AttrTiles tiles;                // 2D attractive pass over shared-column row tiles
    std::unique_ptr<H2Matrix> h2;
    bool h2_valid = false;
    bool has_order = false;
    bool rep_valid_host = false;
    int next_reorder = 0;
    int n_rebuild = 0;
    long long n_launch = 0;
    double kl = 0.0;
    int convergence_count = 0, converged = 0;
    std::vector<double> iter_times;
    profiling_data_t *prof = nullptr;
    // device timing of the last run (CUDA events on the workspace stream)
    double last_run_ms = 0.0, attr_ms = 0.0;
    int attr_launches = 0;
};

struct tsne_h2_matrix {
    tsne_workspace *ws;
};

namespace {

template <int D> size_t vec_bytes() { return sizeof(typename Dim<D>::vec); }

// Host staging of P's upload: two pinned buffers (process-wide, one upload at a time) are
// filled by host threads with a chunk of column indices and values rounded to float (the
// rounding the device applies), while the previous chunk is copied to the device. This sends
// 8 bytes per entry at DMA speed instead of 12 bytes per entry through the driver's pageable
// path.
struct PinnedStage {
    std::mutex mu;
    int *col[2] = {nullptr, nullptr};
    float *val[2] = {nullptr, nullptr};
    size_t cap = 0;   // entries per buffer
};
PinnedStage &pinned_stage()
{
    static PinnedStage s;
    return s;
}

// A column index outside [0, n) in the caller's P: the device would gather out of bounds, so
// the upload stops and tsne_init_with_P returns NULL, leaving P with the caller (as on a
// wrong shape).
struct BadColumn {};

// Copies one chunk of P into the staging buffers (values rounded to float) and checks every
// column index against [0, n) on the way; false if one is out of range.
bool fill_chunk(const int *ci, const double *pv, size_t count, int n, int *col, float *val)
{
    const size_t per = size_t(1) << 20;
    const int nth = (int)std::max<size_t>(1, std::min<size_t>({(size_t)8, (size_t)std::max(1u, std::thread::hardware_concurrency()),
                                                             (count + per - 1) / per}));
    std::vector<unsigned char> bad(nth, 0);
    auto work = [&](int k) {
        const size_t b = count * k / nth, e = count * (k + 1) / nth;
        unsigned int out = 0;
        for (size_t i = b; i < e; i++) {
            const int c = ci[i];
            out |= (unsigned int)c >= (unsigned int)n;
            col[i] = c;
        }
        for (size_t i = b; i < e; i++) val[i] = (float)pv[i];
        bad[k] = out != 0;
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nth; k++) th.emplace_back(work, k);
    work(0);
    for (auto &t : th) t.join();
    for (unsigned char b : bad)
        if (b) return false;
    return true;
}

// Row pointers of the caller's P: start at 0 and never decrease (so every row range lies in
// [0, nnz)), arrays present when there are entries.
bool csr_rows_valid(const sparse_matrix_t *P)
{
    const int n = P->n_rows;
    if (P->row_ptr == nullptr || P->row_ptr[0] != 0) return false;
    for (int i = 0; i < n; i++)
        if (P->row_ptr[i + 1] < P->row_ptr[i]) return false;
    return P->row_ptr[n] == 0 || (P->col_idx != nullptr && P->values != nullptr);
}

template <typename V>
void pad_P(tsne_workspace *ws, const int *rp0, const int *ci0, const V *pv0);

void upload_P(tsne_workspace *ws)
{
    const int n = ws->n, nnz = ws->P->row_ptr[n];
    cudaStream_t st = ws->st;
    DevBuf<int> rp0, ci0;
    DevBuf<float> pv0;
    rp0.exact(n + 1);
    ci0.exact(std::max(nnz, 1));
    pv0.exact(std::max(nnz, 1));
    const bool tm = env_int("TSNE_E2E_TIMERS", 0) != 0;
    double t0 = wall_sec();
    TSNE_CUDA_CHECK(cudaMemcpyAsync(rp0.p, ws->P->row_ptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
    if (nnz > 0) {
        PinnedStage &ps = pinned_stage();
        std::lock_guard<std::mutex> lock(ps.mu);
        constexpr size_t CHUNK = size_t(8) << 20;   // entries per staging buffer
        if (ps.cap < CHUNK) {
            for (int b = 0; b < 2; b++) {
                TSNE_CUDA_CHECK(cudaHostAlloc(&ps.col[b], sizeof(int) * CHUNK, cudaHostAllocPortable));
                TSNE_CUDA_CHECK(cudaHostAlloc(&ps.val[b], sizeof(float) * CHUNK, cudaHostAllocPortable));
            }
            ps.cap = CHUNK;
        }
        cudaEvent_t ev[2];
        for (int b = 0; b < 2; b++) TSNE_CUDA_CHECK(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
        size_t i = 0;
        bool cols_ok = true;
        for (size_t c0 = 0; c0 < (size_t)nnz; c0 += CHUNK, i++) {
            const int b = (int)(i & 1);
            if (i >= 2) TSNE_CUDA_CHECK(cudaEventSynchronize(ev[b]));
            const size_t cnt = std::min(CHUNK, (size_t)nnz - c0);
            if (!fill_chunk(ws->P->col_idx + c0, ws->P->values + c0, cnt, n, ps.col[b], ps.val[b])) {
                cols_ok = false;
                break;
            }
            TSNE_CUDA_CHECK(cudaMemcpyAsync(ci0.p + c0, ps.col[b], sizeof(int) * cnt, cudaMemcpyHostToDevice, st));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(pv0.p + c0, ps.val[b], sizeof(float) * cnt, cudaMemcpyHostToDevice, st));
            TSNE_CUDA_CHECK(cudaEventRecord(ev[b], st));
        }
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        for (int b = 0; b < 2; b++) cudaEventDestroy(ev[b]);
        if (!cols_ok) throw BadColumn();
    }
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    if (tm) printf("E2E upload_P: alloc + copies %.1f ms\n", 1e3 * (wall_sec() - t0));
    pad_P(ws, rp0.p, ci0.p, pv0.p);
}

// The workspace's padded single-precision CSR from a device CSR (row pointers rp0, columns
// ci0, values pv0 of type V)
template <typename V>
void pad_P(tsne_workspace *ws, const int *rp0, const int *ci0, const V *pv0)
{
    const int n = ws->n;
    cudaStream_t st = ws->st;
    ws->len.exact(n + 1);
    ws->rp.exact(n + 2);
    k_pad_len<<<ceil_div(n, 256), 256, 0, st>>>(n, rp0, ws->len.p);
    TSNE_CUDA_CHECK(cudaMemsetAsync(ws->rp.p, 0, sizeof(int), st));
    size_t bytes = 0;
    TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(nullptr, bytes, ws->len.p, ws->rp.p + 1, n, st));
    ws->cub_tmp.ensure(bytes + 256);
    bytes = ws->cub_tmp.cap;
    TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(ws->cub_tmp.p, bytes, ws->len.p, ws->rp.p + 1, n, st));
    int padded = 0;
    TSNE_CUDA_CHECK(cudaMemcpyAsync(&padded, ws->rp.p + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    ws->col.exact(std::max(padded, 4));
    ws->val.exact(std::max(padded, 4));
    ws->padded_nnz = padded;
    k_pad_copy<V><<<ROW_GRID, ROW_BLOCK, 0, st>>>(n, rp0, ci0, pv0, ws->rp.p, ws->col.p, ws->val.p);
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    ws->n_launch += 3;
}

template <int D>
void soa_to_device(tsne_workspace *ws, const double *soa_host, void *dst)
{
    DevBuf<double> tmp;
    tmp.exact((size_t)ws->n * D);
    TSNE_CUDA_CHECK(cudaMemcpyAsync(tmp.p, soa_host, sizeof(double) * ws->n * D, cudaMemcpyHostToDevice, ws->st));
    launch_soa_to_vec<D>(ws->st, ws->n, tmp.p, dst);
    TSNE_CUDA_CHECK(cudaStreamSynchronize(ws->st));
}

void upload_soa(tsne_workspace *ws, const double *soa_host, void *dst)
{
    if (ws->d == 2) soa_to_device<2>(ws, soa_host, dst);
    else soa_to_device<3>(ws, soa_host, dst);
}

// device vec -> host SoA double, in the caller's point order
void download_soa(tsne_workspace *ws, const void *src, double *out)
{
    const int n = ws->n, d = ws->d;
    DevBuf<double> tmp;
    tmp.exact((size_t)n * d);
    if (d == 2) launch_vec_to_soa<2>(ws->st, n, src, tmp.p);
    else launch_vec_to_soa<3>(ws->st, n, src, tmp.p);
    std::vector<double> h((size_t)n * d);
    TSNE_CUDA_CHECK(cudaMemcpyAsync(h.data(), tmp.p, sizeof(double) * n * d, cudaMemcpyDeviceToHost, ws->st));
    std::vector<int> ord;
    if (ws->has_order) {
        ord.resize(n);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(ord.data(), ws->order.p, sizeof(int) * n, cudaMemcpyDeviceToHost, ws->st));
    }
    TSNE_CUDA_CHECK(cudaStreamSynchronize(ws->st));
    for (int k = 0; k < d; k++)
        for (int j = 0; j < n; j++) out[(size_t)k * n + (ws->has_order ? ord[j] : j)] = h[(size_t)k * n + j];
}

// Rebuild the H2 matrix for the current embedding (reference update_h2_matrix,
// src/tsne_h2pack.c:772-953). 0 ok (h2_valid tells whether an H2 matrix exists), -1 failure.
int rebuild_h2(tsne_workspace *ws, const std::function<void()> *overlap = nullptr)
{
    if (ws->n < 2000) { ws->h2_valid = false; return 0; }
    if (!ws->h2) ws->h2 = make_h2_matrix(ws->d, ws->n, ws->st);
    const int leaf = ws->params.h2_leaf_size > 0 ? ws->params.h2_leaf_size : 100;
    const double tol = ws->params.h2_tol > 0.0 ? ws->params.h2_tol : 1e-6;
    const long long l0 = ws->h2->launches();
    const int rc = ws->h2->build(ws->Y.p, leaf, tol, overlap);
    ws->n_launch += ws->h2->launches() - l0;
    if (rc < 0) {
        if (rc == -1) fprintf(stderr, "ERROR: Y contains NaN or Inf!\n");
        ws->h2_valid = false;
        return -1;
    }
    ws->h2_valid = (rc == 0);
    if (rc == 1 && (ws->params.verbose || ws->params.h2pack_print_level >= 1))
        printf("  Skipping H2 approximation: shallow tree (max_level=%d <= 2), using direct O(N^2) sums\n",
               ws->h2->stats().max_level);
    if (ws->h2_valid && ws->params.h2pack_print_level >= 1) {
        const H2Stats &s = ws->h2->stats();
        printf("  H2 matrix: %d nodes, max level %d, far %d, near %d, rank max %d mean %.1f\n", s.n_node,
               s.max_level, s.n_far, s.n_near, s.rank_max, s.rank_mean);
    }
    return 0;
}

// Renumbering (reference tsne_reorder.c:112-167): new point k = old point ord[k]. New row k
// of P is old row ord[k] with its columns mapped through the inverse permutation, in one
// gather pass (the reference transposes twice, which also sorts every row by its new column;
// the entries of a row are the same here, in their previous order, so the attractive sums
// differ only in rounding). Then every per-point array is permuted and the cumulative order
// updated. No host synchronisation.
template <int D>
void renumber_impl(tsne_workspace *ws, const int *ord_dev)
{
    const int n = ws->n;
    const long long nnz = ws->padded_nnz;
    cudaStream_t st = ws->st;
    ws->inv.exact(n);
    ws->len.exact(n + 1);
    ws->rp2.exact(n + 2);
    launch_invert_perm(st, n, ord_dev, ws->inv.p);
    launch_row_len(st, n, ord_dev, ws->rp.p, ws->len.p);
    TSNE_CUDA_CHECK(cudaMemsetAsync(ws->rp2.p, 0, sizeof(int), st));
    size_t bytes = 0;
    TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(nullptr, bytes, ws->len.p, ws->rp2.p + 1, n, st));
    ws->cub_tmp.ensure(bytes + 256);
    bytes = ws->cub_tmp.cap;
    TSNE_CUDA_CHECK(cub::DeviceScan::InclusiveSum(ws->cub_tmp.p, bytes, ws->len.p, ws->rp2.p + 1, n, st));
    ws->col2.exact(std::max<long long>(nnz, 4));
    ws->val2.exact(std::max<long long>(nnz, 4));
    launch_row_gather(st, n, ord_dev, ws->inv.p, ws->rp.p, ws->col.p, ws->val.p, ws->rp2.p, ws->col2.p, ws->val2.p);
    ws->rp.swap(ws->rp2);
    ws->col.swap(ws->col2);
    ws->val.swap(ws->val2);
    ws->tmpv.exact(ws->vbytes * n);
    DevBuf<unsigned char> *arrs[] = {&ws->Y, &ws->uY, &ws->gains, &ws->rep, ws->Yconv.p ? &ws->Yconv : nullptr};
    for (DevBuf<unsigned char> *a : arrs) {
        if (a == nullptr) continue;
        launch_permute_vec<D>(st, n, ord_dev, a->p, ws->tmpv.p);
        a->swap(ws->tmpv);
    }
    ws->order2.exact(n);
    launch_permute_int(st, n, ord_dev, ws->has_order ? ws->order.p : nullptr, ws->order2.p, ws->has_order ? 0 : 1);
    ws->order.swap(ws->order2);
    ws->has_order = true;
    ws->tiles.valid = false;        // rows changed: the tile format is rebuilt by the caller
    ws->n_launch += 11;
}

void renumber(tsne_workspace *ws, const int *ord_dev)
{
    if (ws->d == 2) renumber_impl<2>(ws, ord_dev);
    else renumber_impl<3>(ws, ord_dev);
}

// exact O(N^2) sums + Z + force into ws->frc (reference tsne_h2pack.c:404-491)
template <int D>
void exact_force(tsne_workspace *ws)
{
    ws->s.exact(ws->n);
    ws->v.exact(ws->vbytes * ws->n);
    ws->frc.exact(ws->vbytes * ws->n);
    launch_exact_sv<D>(ws->st, ws->n, ws->Y.p, ws->s.p, ws->v.p);
    launch_z_force<D>(ws->st, ws->n, ws->Y.p, ws->s.p, ws->v.p, nullptr, ws->frc.p, ws->sc.p, ws->zpart.p, 0, 0);
    ws->n_launch += 3;
}

// the shared-memory window forms (TSNE_ATTR_WINDOW) are off: the CSR kernels that the tile
// form pairs with (the update after a rebuild, the centring) use the ROW_GRID row split
bool window_off()
{
    const char *e = getenv("TSNE_ATTR_WINDOW");
    return e == nullptr || atoi(e) == 0;
}

bool next_reorder_due(tsne_workspace *ws, int iter, const int *iters, int n_reorder)
{
    return ws->next_reorder < n_reorder && iter >= iters[ws->next_reorder];
}

void stage_event(tsne_workspace *ws, std::vector<cudaEvent_t> &pool, size_t &used)
{
    if (used == pool.size()) {
        cudaEvent_t e;
        TSNE_CUDA_CHECK(cudaEventCreate(&e));
        pool.push_back(e);
    }
    TSNE_CUDA_CHECK(cudaEventRecord(pool[used++], ws->st));
}

template <int D>
int run_range_impl(tsne_workspace *ws, int it_begin, int it_end)
{
    const tsne_params_t &p = ws->params;
    const int n = ws->n, n_iter = p.n_iter;
    const int verbose = p.verbose, print_freq = p.print_freq > 0 ? p.print_freq : 50;
    const int sklearn = p.sklearn_compatible;
    const int rep_reuse = env_int("TSNE_REP_REUSE", 1) && n >= 2000;
    int reorder_iters[16] = {30, 100, 250, 400, 600, 800};
    int n_reorder = env_int("TSNE_REORDER", 1) ? 6 : 0;
    const char *reorder_env = getenv("TSNE_REORDER_ITERS");
    if (n_reorder > 0 && reorder_env != nullptr && *reorder_env != '\0') {
        n_reorder = 0;
        for (const char *c = reorder_env; *c != '\0' && n_reorder < 16;) {
            reorder_iters[n_reorder++] = atoi(c);
            while (*c != '\0' && *c != ',') c++;
            if (*c == ',') c++;
        }
    }
    // the shared-column tile form of the 2D attractive pass (TSNE_ATTR_TILES=1; off by default
    // until it measures faster), built at the renumberings from iteration tiles_from on
    const bool tiles_on = env_int("TSNE_ATTR_TILES", 0) != 0 && window_off() && getenv("TSNE_ATTR_PIPE") != nullptr &&
                          env_int("TSNE_ATTR_PIPE", 0) == 0;
    const int tiles_from = env_int("TSNE_ATTR_TILES_FROM", 100);
    const int tile_rows = env_int("TSNE_ATTR_TILE_ROWS", 64), tile_umax = env_int("TSNE_ATTR_TILE_UMAX", 6144);
    const int h2_freq = p.h2_rebuild_freq > 0 ? p.h2_rebuild_freq : 10;
    const bool never_h2 = h2_freq > 100000;
    cudaStream_t st = ws->st;
    const long long launch0 = ws->n_launch;
    ws->n_rebuild = 0;

    // profiling: events per stage, resolved at the end
    const bool prof = ws->prof != nullptr;
    const bool ktime = env_int("TSNE_KERNEL_TIMING", 0) != 0;
    std::vector<cudaEvent_t> kev;
    size_t kused = 0;
    cudaEvent_t run0, run1;
    TSNE_CUDA_CHECK(cudaEventCreate(&run0));
    TSNE_CUDA_CHECK(cudaEventCreate(&run1));
    TSNE_CUDA_CHECK(cudaEventRecord(run0, st));
    std::vector<cudaEvent_t> evpool;
    size_t evused = 0;
    struct StageEv { int iter; int stage; size_t a, b; };
    std::vector<StageEv> stages;

    int ret = 0;
    bool z_checked = false;   // the current Z has passed the collapse check
    for (int iter = it_begin; iter < it_end; iter++) {
        const double t_iter = wall_sec();
        const double mom = iter >= p.momentum_switch_iter ? p.momentum : p.initial_momentum;
        double exag;
        if (sklearn) exag = iter < p.early_exag_iter ? p.early_exag : 1.0;
        else if (iter < p.early_exag_iter) exag = p.early_exag;
        else if (iter < p.early_exag_iter + 100) exag = p.early_exag - (p.early_exag - 1.0) * ((double)(iter - p.early_exag_iter) / 100.0);
        else exag = 1.0;
        double lr = ws->lr;
        if (!sklearn && iter >= p.momentum_switch_iter) lr = ws->lr * pow(0.995, iter - p.momentum_switch_iter);

        int eff = iter < 20 ? 1 : h2_freq;
        if (iter >= 20 && iter < p.early_exag_iter && rep_reuse && p.h2_rebuild_freq_early > eff)
            eff = p.h2_rebuild_freq_early;
        bool rebuilt = (iter == 0);
        bool attr_ready = false;
        const bool want = iter > 0 && iter % eff == 0;
        if (n >= 2000 && want && !never_h2) {
            size_t e0 = evused;
            if (prof) stage_event(ws, evpool, evused);
            if (next_reorder_due(ws, iter, reorder_iters, n_reorder) && ws->h2_valid) {
                while (ws->next_reorder < n_reorder && iter >= reorder_iters[ws->next_reorder]) ws->next_reorder++;
                const double t0 = wall_sec();
                renumber(ws, ws->h2->perm_device());
                if (D == 2 && tiles_on && iter >= tiles_from) {
                    attr_tiles_build(st, n, ws->padded_nnz, ws->rp.p, ws->col.p, tile_rows, tile_umax, ws->tiles);
                    ws->n_launch += 8;
                }
                if (env_int("TSNE_H2_TIMERS", 0)) printf("RENUMBER iter %d %.1f ms\n", iter, 1e3 * (wall_sec() - t0));
            }
            // the attractive sums of this iteration depend on Y only: they run while the host
            // waits for the build's counts
            const std::function<void()> overlap = [&]() {
                ws->attr.exact(ws->vbytes * n);
                if (D == 2 && ws->tiles.valid)
                    launch_attr_tile_grad(st, n, ws->tiles, ws->rp.p, ws->col.p, ws->val.p, ws->Y.p, ws->attr.p);
                else
                    launch_attr_grad<D>(st, n, ws->rp.p, ws->col.p, ws->val.p, ws->Y.p, ws->attr.p);
                attr_ready = true;
                ws->n_launch++;
            };
            if (rebuild_h2(ws, &overlap) != 0) {
                fprintf(stderr, "ERROR: Failed to rebuild H2 matrix at iteration %d\n", iter);
                ret = -1;
                break;
            }
            rebuilt = true;
            ws->n_rebuild++;
            if (prof) { stage_event(ws, evpool, evused); stages.push_back({iter, 1, e0, evused - 1}); }
        }

        // repulsion: reuse, H2 product, or exact sums
        const void *force = nullptr;
        const int *flag = nullptr;
        size_t e1 = evused;
        if (prof) stage_event(ws, evpool, evused);
        const bool reuse = rep_reuse && !rebuilt && ws->rep_valid_host;
        if (reuse) {
            force = ws->rep.p;
            flag = &ws->sc.p->rep_valid;
        } else if (ws->h2_valid && !never_h2) {
            const long long l0 = ws->h2->launches();
            ws->h2->product_force(ws->rep.p, ws->sc.p, ws->zpart.p, rep_reuse ? 1 : 0);
            ws->n_launch += ws->h2->launches() - l0;
            force = ws->rep.p;
            flag = &ws->sc.p->force_ok;
            if (rep_reuse) ws->rep_valid_host = true;
        } else {
            exact_force<D>(ws);
            force = ws->frc.p;
            flag = &ws->sc.p->force_ok;
        }
        if (prof && !reuse) { stage_event(ws, evpool, evused); stages.push_back({iter, 2, e1, evused - 1}); }

        // Z collapse stop (reference tsne_h2pack.c:1853-1861). A reuse iteration's Z is the
        // stored one, which the product iteration that stored it has checked already (a failed
        // product sets Z = 1 and stops there), so only the first check after a new Z reads it
        // back: one host synchronisation per product iteration instead of one per iteration.
        if (!reuse) z_checked = false;
        if (!sklearn && iter > p.momentum_switch_iter) {
            if (reuse) TSNE_CUDA_CHECK(cudaMemcpyAsync(&ws->sc.p->Z, &ws->sc.p->rep_Z, sizeof(double), cudaMemcpyDeviceToDevice, st));
            if (!z_checked) {
                TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->hsc.p, ws->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
                TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
                if (ws->hsc.p->Z < 10.0) {
                    if (verbose) printf("\n*** STOPPING: Z collapsed to %.3e (threshold: 10.0) ***\n", ws->hsc.p->Z);
                    break;
                }
                z_checked = true;
            }
        }
        const bool want_kl = (verbose && iter % 50 == 0) || iter == n_iter - 1;
        if (want_kl) {
            if (reuse) TSNE_CUDA_CHECK(cudaMemcpyAsync(&ws->sc.p->Z, &ws->sc.p->rep_Z, sizeof(double), cudaMemcpyDeviceToDevice, st));
            launch_kl<D>(st, n, ws->rp.p, ws->col.p, ws->val.p, ws->Y.p, exag, ws->sc.p, ws->klpart.p);
            ws->n_launch += 2;
        }

        size_t e2 = evused;
        if (prof) stage_event(ws, evpool, evused);
        if (attr_ready) {
            launch_update<D>(st, n, ws->rp.p, ws->Y.p, ws->Yn.p, ws->uY.p, ws->gains.p, force, flag, ws->attr.p,
                             (float)(4.0 * exag), (float)mom, (float)lr, ws->part.p);
        } else {
            if (ktime) stage_event(ws, kev, kused);
            if (D == 2 && ws->tiles.valid)
                launch_attr_tile_update(st, n, ws->tiles, ws->rp.p, ws->col.p, ws->val.p, ws->Y.p, ws->Yn.p,
                                        ws->uY.p, ws->gains.p, force, flag, (float)(4.0 * exag), (float)mom,
                                        (float)lr, ws->part.p);
            else
                launch_attr_update<D>(st, n, ws->rp.p, ws->col.p, ws->val.p, ws->Y.p, ws->Yn.p, ws->uY.p,
                                      ws->gains.p, force, flag, (float)(4.0 * exag), (float)mom, (float)lr,
                                      ws->part.p);
            if (ktime) stage_event(ws, kev, kused);
        }
        if (prof) { stage_event(ws, evpool, evused); stages.push_back({iter, 0, e2, evused - 1}); }
        size_t e3 = evused;
        if (prof) stage_event(ws, evpool, evused);
        launch_center<D>(st, n, ws->Yn.p, ws->Y.p, ws->part.p, ws->sc.p, nullptr, nullptr);
        ws->n_launch += 2;

        if (p.enable_early_stopping && iter >= p.min_iter - 1) {
            ws->Yconv.exact(ws->vbytes * n);
            ws->convpart.exact(256);
            const int vs = (int)(ws->vbytes / sizeof(float));
            if (iter >= p.min_iter) {
                k_conv_check<<<148, 256, 0, st>>>(n, (const float *)ws->Y.p, (const float *)ws->Yconv.p, ws->d, vs,
                                                  ws->convpart.p);
                double hm[148];
                TSNE_CUDA_CHECK(cudaMemcpyAsync(hm, ws->convpart.p, sizeof(hm), cudaMemcpyDeviceToHost, st));
                TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
                double mx = 0.0;
                for (double x : hm) mx = std::max(mx, x);
                if (mx < p.convergence_tol) {
                    ws->convergence_count++;
                    if (ws->convergence_count >= p.convergence_patience) {
                        ws->converged = 1;
                        if (verbose) printf("\n*** CONVERGED at iteration %d ***\n", iter + 1);
                        TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->Yconv.p, ws->Y.p, ws->vbytes * n, cudaMemcpyDeviceToDevice, st));
                        break;
                    }
                } else {
                    ws->convergence_count = 0;
                }
            }
            TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->Yconv.p, ws->Y.p, ws->vbytes * n, cudaMemcpyDeviceToDevice, st));
        }
        if (prof) { stage_event(ws, evpool, evused); stages.push_back({iter, 3, e3, evused - 1}); }

        if (verbose && (iter % print_freq == 0 || iter == n_iter - 1 || iter % 50 == 0)) {
            TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->hsc.p, ws->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
            TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
            if (iter % print_freq == 0 || iter == n_iter - 1)
                printf("  Iteration %4d/%d: Z=%.3e, time=%.3f sec\n", iter + 1, n_iter,
                       reuse ? ws->hsc.p->rep_Z : ws->hsc.p->Z, wall_sec() - t_iter);
            if (iter % 50 == 0) printf("  [KL iter %4d] KL divergence: %.5f\n", iter, ws->hsc.p->kl);
        }
        if ((size_t)iter < ws->iter_times.size()) ws->iter_times[iter] = wall_sec() - t_iter;
    }
    TSNE_CUDA_CHECK(cudaEventRecord(run1, st));
    TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->hsc.p, ws->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    if (it_end >= n_iter || ret != 0) ws->kl = ws->hsc.p->kl;
    if (ret == 0 && ws->h2 && ws->h2->wait_failed()) {
        fprintf(stderr, "ERROR: an H2 kernel gave up waiting for a tree dependency; the run is not valid\n");
        ret = -1;
    }
    {
        float ms = 0.f;
        TSNE_CUDA_CHECK(cudaEventElapsedTime(&ms, run0, run1));
        ws->last_run_ms = ms;
        cudaEventDestroy(run0);
        cudaEventDestroy(run1);
        ws->attr_ms = 0.0;
        ws->attr_launches = 0;
        for (size_t k = 0; k + 1 < kused; k += 2) {
            TSNE_CUDA_CHECK(cudaEventElapsedTime(&ms, kev[k], kev[k + 1]));
            ws->attr_ms += ms;
            ws->attr_launches++;
        }
        for (cudaEvent_t e : kev) cudaEventDestroy(e);
    }
    if (prof) {
        for (const StageEv &s : stages) {
            float ms = 0.f;
            TSNE_CUDA_CHECK(cudaEventElapsedTime(&ms, evpool[s.a], evpool[s.b]));
            const double sec = ms * 1e-3;
            if (s.iter < 0 || s.iter >= n_iter) continue;
            if (s.stage == 0) ws->prof->p_matvec_time[s.iter] += sec;
            else if (s.stage == 1) ws->prof->h2_rebuild_time[s.iter] += sec;
            else if (s.stage == 2) ws->prof->h2_matvec_s_time[s.iter] += sec;
            else ws->prof->other_time[s.iter] += sec;
        }
        for (cudaEvent_t e : evpool) cudaEventDestroy(e);
    }
    (void)launch0;
    return ret;
}

}  // namespace


// =====================================================================================
// C ABI
// =====================================================================================
extern "C" {

tsne_params_t tsne_create_default_params(void)
{
    tsne_params_t p;
    memset(&p, 0, sizeof(p));
    p.n_iter = 1000;
    p.perplexity = 30.0;
    p.learning_rate = -1.0;
    p.initial_momentum = 0.5;
    p.momentum = 0.8;
    p.momentum_switch_iter = 250;
    p.early_exag = 12.0;
    p.early_exag_iter = 250;
    p.use_vptree = 2;
    p.h2_tol = 1e-3;
    p.h2_rebuild_freq = 10;
    p.h2pack_print_level = 0;
    p.init_method = 0;
    p.init_Y = nullptr;
    p.random_seed = (int)(unsigned int)time(nullptr);
    p.verbose = 1;
    p.print_freq = 50;
    p.enable_early_stopping = 0;
    p.convergence_tol = 1e-5;
    p.convergence_patience = 10;
    p.min_iter = 250;
    p.sklearn_compatible = 1;
    p.enable_profiling = 0;
    p.profiling_output_file = nullptr;
    p.num_threads = 1;
    p.h2_leaf_size = 100;
    p.h2_rebuild_freq_early = 10;
    return p;
}

// Host arrays of a sparse matrix: large ones on 2 MB boundaries with transparent huge pages
// requested, so that filling (first touch) and freeing a matrix of 10^8 entries takes a few
// hundred page faults instead of hundreds of thousands. Freed with free().
static void *host_array(size_t bytes)
{
    constexpr size_t HUGE_PAGE = size_t(2) << 20;
    if (bytes >= HUGE_PAGE) {
        const size_t rounded = (bytes + HUGE_PAGE - 1) / HUGE_PAGE * HUGE_PAGE;
        void *p = nullptr;
        if (posix_memalign(&p, HUGE_PAGE, rounded) == 0) {
            madvise(p, rounded, MADV_HUGEPAGE);
            return p;
        }
    }
    return malloc(bytes > 0 ? bytes : 1);
}

sparse_matrix_t *sparse_matrix_create(int n_rows, int n_cols, int nnz)
{
    if (n_rows < 0 || nnz < 0) return nullptr;
    sparse_matrix_t *m = (sparse_matrix_t *)malloc(sizeof(sparse_matrix_t));
    if (m == nullptr) return nullptr;
    m->n_rows = n_rows;
    m->n_cols = n_cols;
    m->nnz = nnz;
    m->row_ptr = (int *)host_array(sizeof(int) * ((size_t)n_rows + 1));
    m->col_idx = (int *)host_array(sizeof(int) * ((size_t)nnz > 0 ? nnz : 1));
    m->values = (double *)host_array(sizeof(double) * ((size_t)nnz > 0 ? nnz : 1));
    if (!m->row_ptr || !m->col_idx || !m->values) { sparse_matrix_destroy(m); return nullptr; }
    return m;
}

void sparse_matrix_destroy(sparse_matrix_t *mat)
{
    if (mat == nullptr) return;
    free(mat->row_ptr);
    free(mat->col_idx);
    free(mat->values);
    free(mat);
}

void sparse_matvec(const sparse_matrix_t *A, const double *x, double *y)
{
    for (int i = 0; i < A->n_rows; i++) {
        double s = 0.0;
        for (int e = A->row_ptr[i]; e < A->row_ptr[i + 1]; e++) s += A->values[e] * x[A->col_idx[e]];
        y[i] = s;
    }
}

// The C library's rand() sequence after srand(seed), generated without the library's global,
// locked state: the glibc generator is the additive lagged-Fibonacci generator
// r[i] = r[i-3] + r[i-31] (mod 2^32), seeded by the Park-Miller LCG (16807, 2^31 - 1) in
// Schrage's form, with the first 310 outputs discarded; rand() returns r >> 1.
static void libc_rand_sequence(unsigned int seed, size_t count, unsigned int *out)
{
    int32_t r[34];
    int32_t word = (int32_t)seed;
    if (word == 0) word = 1;
    r[0] = word;
    for (int i = 1; i < 31; i++) {
        const long hi = word / 127773, lo = word % 127773;
        long w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        word = (int32_t)w;
        r[i] = word;
    }
    std::vector<uint32_t> ring(34 + 310 + count);
    for (int i = 0; i < 31; i++) ring[i] = (uint32_t)r[i];
    for (int i = 31; i < 34; i++) ring[i] = ring[i - 31];
    for (size_t i = 34; i < ring.size(); i++) ring[i] = ring[i - 31] + ring[i - 3];
    for (size_t k = 0; k < count; k++) out[k] = ring[k + 344] >> 1;
}

void initialize_embedding(double *Y, int n_point, int low_dim, int method, const double *Y0, unsigned int seed)
{
    if (method == 1 && Y0 != nullptr) {
        memcpy(Y, Y0, sizeof(double) * (size_t)n_point * low_dim);
        return;
    }
    if (method == 1) printf("Warning: init_method=1 without init_Y, using random initialization\n");
    // N(0, 1e-4^2) by Box-Muller on the C library's rand() sequence (the reference's generator);
    // the uniforms are drawn in order, the transform runs on several threads
    const size_t total = (size_t)n_point * low_dim;
    const size_t pairs = (total + 1) / 2;
    std::vector<unsigned int> u(2 * pairs);
    libc_rand_sequence(seed, u.size(), u.data());
    const int nth = (int)std::max<size_t>(1, std::min<size_t>({(size_t)8, (size_t)std::max(1u, std::thread::hardware_concurrency()),
                                                             pairs / 65536 + 1}));
    auto work = [&](int k) {
        const size_t b = pairs * k / nth, e = pairs * (k + 1) / nth;
        for (size_t p = b; p < e; p++) {
            double u1 = (double)u[2 * p] / RAND_MAX;
            const double u2 = (double)u[2 * p + 1] / RAND_MAX;
            if (u1 < 1e-10) u1 = 1e-10;
            const double rad = sqrt(-2.0 * log(u1));
            const size_t i = 2 * p;
            Y[i] = 1e-4 * (rad * cos(2.0 * M_PI * u2));
            if (i + 1 < total) Y[i + 1] = 1e-4 * (rad * sin(2.0 * M_PI * u2));
        }
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nth; k++) th.emplace_back(work, k);
    work(0);
    for (auto &t : th) t.join();
}

sparse_matrix_t *compute_P_from_knn_distances(const double *knn_distances, const int *knn_indices,
                                              const int *knn_indptr, int n_samples, int nnz, double perplexity,
                                              int num_threads)
{
    (void)num_threads;
    if (n_samples < 0 || nnz < 0 || perplexity <= 0.0) return nullptr;
    sparse_matrix_t *P = sparse_matrix_create(n_samples, n_samples, nnz);
    if (P == nullptr) return nullptr;
    memcpy(P->row_ptr, knn_indptr, sizeof(int) * ((size_t)n_samples + 1));
    if (nnz > 0) memcpy(P->col_idx, knn_indices, sizeof(int) * nnz);
    P->nnz = nnz;
    P->row_ptr[n_samples] = nnz;
    if (nnz == 0) return P;
    try {
        cudaStream_t st;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        DevBuf<int> ip;
        DevBuf<double> dist, out;
        ip.exact(n_samples + 1);
        dist.exact(nnz);
        out.exact(nnz);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(ip.p, knn_indptr, sizeof(int) * (n_samples + 1), cudaMemcpyHostToDevice, st));
        TSNE_CUDA_CHECK(cudaMemcpyAsync(dist.p, knn_distances, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
        launch_pcal(st, n_samples, ip.p, dist.p, perplexity, out.p);
        TSNE_CUDA_CHECK(cudaGetLastError());
        TSNE_CUDA_CHECK(cudaMemcpyAsync(P->values, out.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost, st));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
    } catch (const CudaError &) {
        sparse_matrix_destroy(P);
        return nullptr;
    }
    return P;
}

}  // extern "C"

namespace {
// Workspace creation once the arguments are checked: device state, P (through load_P, which
// returns false on bad input), the initial embedding and the first H2 build. P (host, may be
// NULL) is owned by the workspace from here on, as tsne_init_with_P specifies.
tsne_workspace *create_workspace(int n_point, int pt_dim, int low_dim, const tsne_params_t *params,
                                 sparse_matrix_t *P, const std::function<bool(tsne_workspace *)> &load_P)
{
    tsne_workspace *ws = nullptr;
    try {
        ws = new tsne_workspace();   // its pinned host scalars need a device
    } catch (const CudaError &) {
        return nullptr;
    }
    try {
        ws->params = *params;
        if (params->profiling_output_file) ws->prof_file = params->profiling_output_file;
        ws->params.profiling_output_file = nullptr;
        ws->n = n_point;
        ws->d = low_dim;
        ws->pt_dim = pt_dim;
        ws->lr = params->learning_rate < 0.0 ? std::max(200.0, n_point / 12.0) : params->learning_rate;
        if (params->learning_rate < 0.0 && params->verbose)
            printf("Using adaptive learning rate: %.1f (N=%d)\n", ws->lr, n_point);
        ws->vbytes = low_dim == 2 ? vec_bytes<2>() : vec_bytes<3>();
        ws->P = P;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&ws->st, cudaStreamNonBlocking));
        AllocStream guard(ws->st);
        const size_t vb = ws->vbytes * n_point;
        ws->Y.exact(vb); ws->Yn.exact(vb); ws->uY.exact(vb); ws->gains.exact(vb); ws->rep.exact(vb);
        TSNE_CUDA_CHECK(cudaMemsetAsync(ws->uY.p, 0, vb, ws->st));
        TSNE_CUDA_CHECK(cudaMemsetAsync(ws->rep.p, 0, vb, ws->st));
        if (low_dim == 2) launch_fill_vec<2>(ws->st, n_point, ws->gains.p, 1.0f);
        else launch_fill_vec<3>(ws->st, n_point, ws->gains.p, 1.0f);
        ws->sc.exact(1);
        TSNE_CUDA_CHECK(cudaMemsetAsync(ws->sc.p, 0, sizeof(DevScalars), ws->st));
        ws->part.exact((size_t)ROW_GRID * 3);
        ws->zpart.exact(148 * 2 * 3);
        ws->klpart.exact(ROW_GRID);
        const bool tm = env_int("TSNE_E2E_TIMERS", 0) != 0;
        double t0 = wall_sec();
        // the initial embedding (host only) is drawn on another thread while P goes up; the
        // guard joins it on every way out of this block
        std::vector<double> Y0((size_t)n_point * low_dim);
        std::thread init_th([&Y0, n_point, low_dim, params] {
            initialize_embedding(Y0.data(), n_point, low_dim, params->init_method, params->init_Y,
                                 (unsigned int)params->random_seed);
        });
        struct Joiner {
            std::thread &t;
            ~Joiner() { if (t.joinable()) t.join(); }
        } joiner{init_th};
        if (!load_P(ws)) {
            init_th.join();
            tsne_destroy(ws);
            return nullptr;
        }
        if (tm) printf("E2E init: P on the device %.1f ms\n", 1e3 * (wall_sec() - t0));
        t0 = wall_sec();
        init_th.join();
        ws->params.init_Y = nullptr;
        upload_soa(ws, Y0.data(), ws->Y.p);
        ws->iter_times.assign(std::max(params->n_iter, 0), 0.0);
        if (params->enable_profiling) {
            const size_t ni = std::max(params->n_iter, 1);
            ws->prof = (profiling_data_t *)calloc(1, sizeof(profiling_data_t));
            ws->prof->knn_time = (double *)calloc(1, sizeof(double));
            ws->prof->p_construction_time = (double *)calloc(1, sizeof(double));
            ws->prof->p_matvec_time = (double *)calloc(ni, sizeof(double));
            ws->prof->h2_rebuild_time = (double *)calloc(ni, sizeof(double));
            ws->prof->h2_matvec_s_time = (double *)calloc(ni, sizeof(double));
            ws->prof->h2_matvec_v_time = (double *)calloc(ni, sizeof(double));
            ws->prof->z_computation_time = (double *)calloc(ni, sizeof(double));
            ws->prof->gradient_time = (double *)calloc(ni, sizeof(double));
            ws->prof->other_time = (double *)calloc(ni, sizeof(double));
        }
        if (params->verbose)
            printf("Initializing t-SNE with pre-computed P matrix (n=%d, pt_dim=%d, low_dim=%d)\n", n_point, pt_dim,
                   low_dim);
        if (tm) printf("E2E init: embedding %.1f ms\n", 1e3 * (wall_sec() - t0));
        t0 = wall_sec();
        const bool never_h2 = (params->h2_rebuild_freq > 0 ? params->h2_rebuild_freq : 10) > 100000;
        if (n_point >= 2000 && !never_h2) {
            if (rebuild_h2(ws) != 0) {
                printf("Error: Failed to build initial H2 matrix\n");
                tsne_destroy(ws);
                return nullptr;
            }
        }
        TSNE_CUDA_CHECK(cudaStreamSynchronize(ws->st));
        if (tm) printf("E2E init: first H2 build %.1f ms\n", 1e3 * (wall_sec() - t0));
    } catch (const CudaError &) {
        tsne_destroy(ws);
        return nullptr;
    } catch (const BadColumn &) {
        printf("Error: Invalid P matrix (a column index is outside [0, %d))\n", n_point);
        ws->P = nullptr;   // P stays with the caller
        tsne_destroy(ws);
        return nullptr;
    }
    return ws;
}
}  // namespace

extern "C" {

tsne_workspace_t *tsne_init_with_P(const double *X, int n_point, int pt_dim, int low_dim,
                                   const tsne_params_t *params, sparse_matrix_t *P)
{
    (void)X;
    if (low_dim != 2 && low_dim != 3) {
        printf("Error: low_dim must be 2 or 3 (got %d)\n", low_dim);
        return nullptr;
    }
    if (P == nullptr || P->n_rows != n_point || P->n_cols != n_point) {
        printf("Error: Invalid P matrix (expected %dx%d, got %dx%d)\n", n_point, n_point, P ? P->n_rows : 0,
               P ? P->n_cols : 0);
        return nullptr;
    }
    if (params == nullptr || n_point < 1) return nullptr;
    if (!csr_rows_valid(P)) {
        printf("Error: Invalid P matrix (row pointers must start at 0 and not decrease)\n");
        return nullptr;
    }
    return create_workspace(n_point, pt_dim, low_dim, params, P, [](tsne_workspace *w) {
        upload_P(w);
        return true;
    });
}

tsne_workspace_t *tsne_init_with_knn_distances(const double *X, int n_point, int pt_dim, int low_dim,
                                               const tsne_params_t *params, const double *knn_distances,
                                               const int *knn_indices, const int *knn_indptr, int nnz)
{
    (void)X;
    if (low_dim != 2 && low_dim != 3) {
        printf("Error: low_dim must be 2 or 3 (got %d)\n", low_dim);
        return nullptr;
    }
    if (params == nullptr || n_point < 1 || knn_indptr == nullptr || nnz < 0 ||
        (nnz > 0 && (knn_distances == nullptr || knn_indices == nullptr)))
        return nullptr;
    const double perplexity = params->perplexity;
    return create_workspace(n_point, pt_dim, low_dim, params, nullptr, [=](tsne_workspace *w) {
        DevCSR d;
        if (joint_P_device(w->st, n_point, knn_distances, knn_indices, knn_indptr, nnz, perplexity, d) != 0)
            return false;
        pad_P<double>(w, d.rp.p, d.col.p, d.val.p);
        return true;
    });
}

int tsne_run_range(tsne_workspace_t *ws, int iter_begin, int iter_end)
{
    if (ws == nullptr) return -1;
    AllocStream guard(ws->st);
    try {
        const long long l0 = ws->n_launch;
        const int rc = ws->d == 2 ? run_range_impl<2>(ws, iter_begin, iter_end) : run_range_impl<3>(ws, iter_begin, iter_end);
        (void)l0;
        return rc;
    } catch (const CudaError &) {
        return -1;
    }
}

int tsne_run(tsne_workspace_t *ws)
{
    if (ws == nullptr) return -1;
    if (ws->params.verbose) printf("\nStarting t-SNE optimization (%d iterations)\n", ws->params.n_iter);
    const long long l0 = ws->n_launch;
    const int rc = tsne_run_range(ws, 0, ws->params.n_iter);
    ws->n_launch = ws->n_launch - l0;
    if (ws->params.verbose) printf("\nOptimization complete\n");
    if (env_int("TSNE_H2_TIMERS", 0) && ws->h2) {
        printf("H2REBUILDS %d\n", ws->n_rebuild);
        try { ws->h2->flush_timers(); } catch (const CudaError &) {}
    }
    if (rc == 0 && ws->prof && !ws->prof_file.empty()) tsne_write_profiling_data(ws, ws->prof_file.c_str());
    return rc;
}

void tsne_get_embedding(tsne_workspace_t *ws, double *Y_out)
{
    if (ws == nullptr || Y_out == nullptr) return;
    AllocStream guard(ws->st);
    try {
        download_soa(ws, ws->Y.p, Y_out);
    } catch (const CudaError &) {
    }
}

double compute_kl_divergence(tsne_workspace_t *ws)
{
    if (ws == nullptr) return 0.0;
    return ws->kl;
}

void tsne_destroy(tsne_workspace_t *ws)
{
    if (ws == nullptr) return;
    const bool tm = env_int("TSNE_E2E_TIMERS", 0) != 0;
    double t0 = wall_sec();
    if (ws->st) cudaStreamSynchronize(ws->st);
    AllocStream guard(ws->st);
    double t1 = wall_sec();
    ws->h2.reset();
    double t2 = wall_sec();
    if (ws->P) sparse_matrix_destroy(ws->P);
    double t3 = wall_sec();
    if (tm) printf("E2E destroy: sync %.1f ms, h2 %.1f ms, host P %.1f ms\n", 1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (t3 - t2));
    if (ws->prof) {
        free(ws->prof->knn_time); free(ws->prof->p_construction_time); free(ws->prof->p_matvec_time);
        free(ws->prof->h2_rebuild_time); free(ws->prof->h2_matvec_s_time); free(ws->prof->h2_matvec_v_time);
        free(ws->prof->z_computation_time); free(ws->prof->gradient_time); free(ws->prof->other_time);
        free(ws->prof);
    }
    cudaStream_t st = ws->st;
    t0 = wall_sec();
    delete ws;   // device buffers are released here
    if (st) cudaStreamDestroy(st);
    if (tm) printf("E2E destroy: workspace buffers %.1f ms\n", 1e3 * (wall_sec() - t0));
}

int tsne_fit_transform_with_P(const double *X, int n_point, int pt_dim, int low_dim, const tsne_params_t *params,
                              sparse_matrix_t *P, double *Y_out)
{
    tsne_workspace_t *ws = tsne_init_with_P(X, n_point, pt_dim, low_dim, params, P);
    if (ws == nullptr) return -1;
    const int rc = tsne_run(ws);
    if (rc != 0) { tsne_destroy(ws); return rc; }
    tsne_get_embedding(ws, Y_out);
    tsne_destroy(ws);
    return 0;
}

void tsne_write_profiling_data(tsne_workspace_t *ws, const char *filename)
{
    if (ws == nullptr || ws->prof == nullptr || filename == nullptr) return;
    FILE *fp = fopen(filename, "w");
    if (!fp) { fprintf(stderr, "Error: Cannot write profiling data to %s\n", filename); return; }
    profiling_data_t *pr = ws->prof;
    const int n_iter = ws->params.n_iter;
    fprintf(fp, "iteration,p_matvec,h2_rebuild,h2_matvec_s,h2_matvec_v,z_computation,gradient,other,total\n");
    double tp = 0, tr = 0, tm = 0, tg = 0, tt = 0;
    for (int i = 0; i < n_iter; i++) {
        const double tot = pr->p_matvec_time[i] + pr->h2_rebuild_time[i] + pr->h2_matvec_s_time[i] +
                           pr->h2_matvec_v_time[i] + pr->z_computation_time[i] + pr->gradient_time[i] + pr->other_time[i];
        fprintf(fp, "%d,%.6f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6f\n", i, pr->p_matvec_time[i], pr->h2_rebuild_time[i],
                pr->h2_matvec_s_time[i], pr->h2_matvec_v_time[i], pr->z_computation_time[i], pr->gradient_time[i],
                pr->other_time[i], tot);
        tp += pr->p_matvec_time[i];
        tr += pr->h2_rebuild_time[i];
        tm += pr->h2_matvec_s_time[i] + pr->h2_matvec_v_time[i];
        tg += pr->gradient_time[i];
        tt += tot;
    }
    const double tdiv = tt > 0 ? tt : 1.0;
    fprintf(fp, "\n# Summary Statistics\n");
    fprintf(fp, "# k-NN time: %.3f seconds\n", pr->knn_time[0]);
    fprintf(fp, "# P construction: %.3f seconds\n", pr->p_construction_time[0]);
    fprintf(fp, "# Total P-matvec: %.3f seconds (%.1f%%)\n", tp, 100.0 * tp / tdiv);
    fprintf(fp, "# Total H²-rebuild: %.3f seconds (%.1f%%)\n", tr, 100.0 * tr / tdiv);
    fprintf(fp, "# Total H²-matvec: %.3f seconds (%.1f%%)\n", tm, 100.0 * tm / tdiv);
    fprintf(fp, "# Total gradient: %.3f seconds (%.1f%%)\n", tg, 100.0 * tg / tdiv);
    fprintf(fp, "# Total optimization time: %.3f seconds\n", tt);
    fclose(fp);
    if (ws->params.verbose) printf("\nProfiling data written to: %s\n", filename);
}

void tsne_set_init_profiling_times(tsne_workspace_t *ws, double knn_time, double p_construction_time)
{
    if (ws == nullptr || ws->prof == nullptr) return;
    ws->prof->knn_time[0] = knn_time;
    ws->prof->p_construction_time[0] = p_construction_time;
}

void compute_attractive_forces(const sparse_matrix_t *P, const double *Y, int low_dim, int n_point,
                               double early_exag, double *grad, int num_threads)
{
    (void)num_threads;
    if (P == nullptr || Y == nullptr || grad == nullptr || (low_dim != 2 && low_dim != 3)) return;
    if (P->n_rows != n_point || P->n_cols != n_point || !csr_rows_valid(P)) return;
    sparse_matrix_t *Pc = sparse_matrix_create(P->n_rows, P->n_cols, P->row_ptr[P->n_rows]);
    if (Pc == nullptr) return;
    memcpy(Pc->row_ptr, P->row_ptr, sizeof(int) * (P->n_rows + 1));
    memcpy(Pc->col_idx, P->col_idx, sizeof(int) * Pc->nnz);
    memcpy(Pc->values, P->values, sizeof(double) * Pc->nnz);
    tsne_workspace ws;
    try {
        ws.n = n_point; ws.d = low_dim; ws.P = Pc;
        ws.vbytes = low_dim == 2 ? vec_bytes<2>() : vec_bytes<3>();
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&ws.st, cudaStreamNonBlocking));
        upload_P(&ws);
        ws.Y.exact(ws.vbytes * n_point);
        upload_soa(&ws, Y, ws.Y.p);
        DevBuf<double> g;
        g.exact((size_t)n_point * low_dim);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(g.p, grad, sizeof(double) * n_point * low_dim, cudaMemcpyHostToDevice, ws.st));
        if (low_dim == 2) launch_attr_only<2>(ws.st, n_point, ws.rp.p, ws.col.p, ws.val.p, ws.Y.p, 4.0 * early_exag, g.p);
        else launch_attr_only<3>(ws.st, n_point, ws.rp.p, ws.col.p, ws.val.p, ws.Y.p, 4.0 * early_exag, g.p);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(grad, g.p, sizeof(double) * n_point * low_dim, cudaMemcpyDeviceToHost, ws.st));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(ws.st));
    } catch (const CudaError &) {
    } catch (const BadColumn &) {   // grad is left unchanged
    }
    sparse_matrix_destroy(Pc);
    ws.P = nullptr;
    if (ws.st) cudaStreamDestroy(ws.st);
    ws.st = nullptr;
}

H2Pack_p tsne_get_h2_matrix(tsne_workspace_t *ws)
{
    if (ws == nullptr || !ws->h2_valid) return nullptr;
    static thread_local tsne_h2_matrix handle;
    handle.ws = ws;
    return &handle;
}

double compute_repulsive_forces_h2pack(H2Pack_p h2pack_W, const double *Y, int low_dim, int n_point,
                                       tsne_workspace_t *ws, double *grad, int iter)
{
    (void)iter;
    if (ws == nullptr || Y == nullptr || grad == nullptr || low_dim != ws->d || n_point != ws->n) return 1.0;
    AllocStream guard(ws->st);
    try {
        std::vector<double> F((size_t)n_point * low_dim);
        double Z = 1.0;
        if (h2pack_W != nullptr && ws->h2_valid) {
            // the H2 matrix applies to the embedding it was built from (the workspace's)
            ws->h2->product_force(ws->frc.exact(ws->vbytes * n_point), ws->sc.p, ws->zpart.p, 0);
        } else {
            DevBuf<unsigned char> saveY;
            saveY.exact(ws->vbytes * n_point);
            TSNE_CUDA_CHECK(cudaMemcpyAsync(saveY.p, ws->Y.p, ws->vbytes * n_point, cudaMemcpyDeviceToDevice, ws->st));
            upload_soa(ws, Y, ws->Y.p);
            if (ws->has_order) {
                // Y is given in the caller's order; the workspace works in its own numbering
                TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->Y.p, saveY.p, ws->vbytes * n_point, cudaMemcpyDeviceToDevice, ws->st));
                return 1.0;
            }
            if (low_dim == 2) exact_force<2>(ws); else exact_force<3>(ws);
            TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->Y.p, saveY.p, ws->vbytes * n_point, cudaMemcpyDeviceToDevice, ws->st));
        }
        download_soa(ws, ws->frc.p, F.data());
        TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->hsc.p, ws->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, ws->st));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(ws->st));
        Z = ws->hsc.p->Z;
        if (ws->hsc.p->force_ok)
            for (size_t i = 0; i < F.size(); i++) grad[i] -= F[i];
        return Z;
    } catch (const CudaError &) {
        return 1.0;
    }
}

int update_h2_matrix(tsne_workspace_t *ws, int force_rebuild)
{
    (void)force_rebuild;
    if (ws == nullptr) return -1;
    AllocStream guard(ws->st);
    try {
        return rebuild_h2(ws);
    } catch (const CudaError &) {
        return -1;
    }
}

int tsne_h2_matmul(H2Pack_p h2, const int nv, const double *const *X, double *const *Y, void **wsp)
{
    (void)wsp;
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2_valid || nv < 1 || nv > 4) return -1;
    tsne_workspace *ws = h2->ws;
    if (ws->has_order) return -1;
    try {
        const int n = ws->n;
        std::vector<int> perm(n);
        double corner[3], radius;
        ws->h2->copy_tree(perm.data(), corner, &radius);
        std::vector<float> xt((size_t)n * 4, 0.f), yt;
        for (int k = 0; k < n; k++)
            for (int c = 0; c < nv; c++) xt[(size_t)k * 4 + c] = (float)X[c][perm[k]];
        ws->h2->product_columns(xt, yt);
        for (int k = 0; k < n; k++)
            for (int c = 0; c < nv; c++) Y[c][perm[k]] = (double)yt[(size_t)k * 4 + c] + X[c][perm[k]];
        return 0;
    } catch (const CudaError &) {
        return -1;
    }
}

void tsne_h2_matmul_free(void **wsp)
{
    if (wsp) *wsp = nullptr;
}

int tsne_renumber_points(tsne_workspace_t *ws, const int *ord, int num_threads)
{
    (void)num_threads;
    if (ws == nullptr || ord == nullptr) return -1;
    try {
        DevBuf<int> d;
        d.exact(ws->n);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(d.p, ord, sizeof(int) * ws->n, cudaMemcpyHostToDevice, ws->st));
        renumber(ws, d.p);
        ws->h2_valid = false;   // the tree refers to the old numbering
        return 0;
    } catch (const CudaError &) {
        return -1;
    }
}

int tsne_h2_info(H2Pack_p h2, int *n_node, int *max_level, int *n_far, int *n_near)
{
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2) return -1;
    const H2Stats &s = h2->ws->h2->stats();
    if (n_node) *n_node = s.n_node;
    if (max_level) *max_level = s.max_level;
    if (n_far) *n_far = s.n_far;
    if (n_near) *n_near = s.n_near;
    return 0;
}

int tsne_h2_get_tree(H2Pack_p h2, int *perm, double *corner, double *radius)
{
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2) return -1;
    try { h2->ws->h2->copy_tree(perm, corner, radius); } catch (const CudaError &) { return -1; }
    return 0;
}

int tsne_h2_get_nodes(H2Pack_p h2, int *start, int *end, int *level, int *parent, int *first_child, int *n_child,
                      int *is_leaf)
{
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2) return -1;
    try { h2->ws->h2->copy_nodes(start, end, level, parent, first_child, n_child, is_leaf); } catch (const CudaError &) { return -1; }
    return 0;
}

int tsne_h2_get_lists(H2Pack_p h2, int *far_ptr, int *far_idx, int *near_ptr, int *near_idx)
{
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2) return -1;
    try { h2->ws->h2->copy_lists(far_ptr, far_idx, near_ptr, near_idx); } catch (const CudaError &) { return -1; }
    return 0;
}

int tsne_h2_get_ranks(H2Pack_p h2, int *rank)
{
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2) return -1;
    try { h2->ws->h2->copy_ranks(rank); } catch (const CudaError &) { return -1; }
    return 0;
}

int tsne_h2_get_bases(H2Pack_p h2, int *n_rows, int *max_rank, long long *row_off, float *U, float *skel)
{
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2 || n_rows == nullptr || max_rank == nullptr) return -1;
    if (U != nullptr && (row_off == nullptr || skel == nullptr)) return -1;
    try { return h2->ws->h2->copy_bases(n_rows, max_rank, row_off, U, skel); } catch (const CudaError &) { return -1; }
}

int tsne_h2_probe_dependency_timeout(H2Pack_p h2, int max_polls)
{
    if (h2 == nullptr || h2->ws == nullptr || !h2->ws->h2 || max_polls < 1 || max_polls > (1 << 22)) return -1;
    try { return h2->ws->h2->probe_dependency_timeout(max_polls); } catch (const CudaError &) { return -1; }
}

int tsne_get_state(tsne_workspace_t *ws, double *Y_out, double *rep_out, double *rep_Z)
{
    if (ws == nullptr) return -1;
    try {
        if (Y_out) download_soa(ws, ws->Y.p, Y_out);
        if (rep_out) download_soa(ws, ws->rep.p, rep_out);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(ws->hsc.p, ws->sc.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, ws->st));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(ws->st));
        if (rep_Z) *rep_Z = ws->hsc.p->rep_Z;
    } catch (const CudaError &) {
        return -1;
    }
    return 0;
}

int tsne_set_embedding(tsne_workspace_t *ws, const double *Y_in)
{
    if (ws == nullptr || Y_in == nullptr) return -1;
    try {
        std::vector<double> Yc((size_t)ws->n * ws->d);
        if (ws->has_order) {
            std::vector<int> ord(ws->n);
            TSNE_CUDA_CHECK(cudaStreamSynchronize(ws->st));
            TSNE_CUDA_CHECK(cudaMemcpy(ord.data(), ws->order.p, sizeof(int) * ws->n, cudaMemcpyDeviceToHost));
            for (int k = 0; k < ws->d; k++)
                for (int j = 0; j < ws->n; j++) Yc[(size_t)k * ws->n + j] = Y_in[(size_t)k * ws->n + ord[j]];
        } else {
            memcpy(Yc.data(), Y_in, sizeof(double) * Yc.size());
        }
        upload_soa(ws, Yc.data(), ws->Y.p);
        const size_t vb = ws->vbytes * ws->n;
        TSNE_CUDA_CHECK(cudaMemsetAsync(ws->uY.p, 0, vb, ws->st));
        if (ws->d == 2) launch_fill_vec<2>(ws->st, ws->n, ws->gains.p, 1.0f);
        else launch_fill_vec<3>(ws->st, ws->n, ws->gains.p, 1.0f);
        TSNE_CUDA_CHECK(cudaStreamSynchronize(ws->st));
    } catch (const CudaError &) {
        return -1;
    }
    return 0;
}

int tsne_get_timing(tsne_workspace_t *ws, double *run_ms, double *attr_ms, int *attr_launches)
{
    if (ws == nullptr) return -1;
    if (run_ms) *run_ms = ws->last_run_ms;
    if (attr_ms) *attr_ms = ws->attr_ms;
    if (attr_launches) *attr_launches = ws->attr_launches;
    return 0;
}

int tsne_get_run_stats(tsne_workspace_t *ws, int *n_rebuild, long long *n_launch)
{
    if (ws == nullptr) return -1;
    if (n_rebuild) *n_rebuild = ws->n_rebuild;
    if (n_launch) *n_launch = ws->n_launch;
    return 0;
}

}  // extern "C"
