// Batched and served embedding jobs: many independent t-SNE optimisations on one GPU.
//
// A server owns a pool of worker threads. Jobs (P, dimensions, parameters) are submitted at
// any time and queue in arrival order; a worker starts the job at the head of the queue when
// fewer than `max_concurrent` jobs run and the device memory the job needs (an upper estimate
// from N and nnz(P)) fits under the HBM budget next to the running jobs' - or when nothing
// runs, so that a job larger than the budget still runs, alone. Every job is a workspace of
// its own with its own CUDA stream, so the kernels of the running jobs overlap on the device,
// and a job that arrives while others run starts as soon as a slot and memory free up
// (continuous batching). A job's computation does not depend on what else runs: its result is
// bit for bit the one it gets alone. There is no counterpart in the reference, which runs one
// embedding per call.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tsne_h2pack.h"

namespace {

double now_sec()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum JobState { QUEUED = 0, RUNNING = 1, DONE = 2, FAILED = 3 };

struct Job {
    int id = 0;
    int n = 0, d = 2;
    tsne_params_t params{};
    std::vector<double> init_Y;     // copy of params.init_Y (the caller's array may go away)
    std::string prof_file;
    sparse_matrix_t *P = nullptr;   // owned until the workspace takes it
    size_t bytes = 0;               // admission estimate
    int state = QUEUED;
    bool collected = false;         // the result was handed out and released
    std::vector<double> Y;          // result, low_dim x n
    double kl = 0.0;
    double t_submit = 0.0, t_start = 0.0, t_end = 0.0, run_s = 0.0;
};

}  // namespace

struct tsne_server {
    std::mutex mu;
    std::condition_variable cv_work;   // workers: a job may be admissible
    std::condition_variable cv_done;   // waiters: a job finished
    std::deque<int> queue;             // queued job ids, arrival order
    std::vector<std::unique_ptr<Job>> jobs;
    std::vector<std::thread> workers;
    int max_concurrent = 1;
    size_t budget = 0;
    size_t running_bytes = 0;
    int running = 0;
    bool stop = false;
    int device = 0;
};

namespace {

// device bytes a job may hold at its peak: P (padded copy, the renumbering copy and the
// upload's temporaries), the per-point vectors, the H2 tree, lists and bases
size_t job_bytes(int n, long long nnz)
{
    return (size_t)(32 * nnz) + (size_t)n * 2048 + (size_t(64) << 20);
}

bool run_job(Job *job)
{
    tsne_params_t prm = job->params;
    prm.init_Y = job->init_Y.empty() ? nullptr : job->init_Y.data();
    prm.profiling_output_file = job->prof_file.empty() ? nullptr : const_cast<char *>(job->prof_file.c_str());
    sparse_matrix_t *P = job->P;
    job->P = nullptr;
    const double t0 = now_sec();
    tsne_workspace_t *ws = tsne_init_with_P(nullptr, job->n, 0, job->d, &prm, P);
    bool ok = ws != nullptr;
    if (ok) ok = tsne_run(ws) == 0;
    if (ok) {
        job->Y.assign((size_t)job->n * job->d, 0.0);
        tsne_get_embedding(ws, job->Y.data());
        job->kl = compute_kl_divergence(ws);
    }
    if (ws != nullptr) tsne_destroy(ws);
    job->run_s = now_sec() - t0;
    return ok;
}

void worker_loop(tsne_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        Job *job = nullptr;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_work.wait(lock, [&] {
                if (s->stop) return true;
                if (s->queue.empty() || s->running >= s->max_concurrent) return false;
                const Job *head = s->jobs[s->queue.front()].get();
                return s->running == 0 || s->running_bytes + head->bytes <= s->budget;
            });
            if (s->stop) return;
            job = s->jobs[s->queue.front()].get();
            s->queue.pop_front();
            s->running++;
            s->running_bytes += job->bytes;
            job->state = RUNNING;
            job->t_start = now_sec();
        }
        const bool ok = run_job(job);
        {
            std::lock_guard<std::mutex> lock(s->mu);
            job->state = ok ? DONE : FAILED;
            job->t_end = now_sec();
            s->running--;
            s->running_bytes -= job->bytes;
        }
        s->cv_work.notify_all();
        s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

tsne_server_t *tsne_server_create(int max_concurrent, double hbm_budget_gb)
{
    if (max_concurrent < 1 || !(hbm_budget_gb > 0.0)) return nullptr;
    tsne_server *s = new tsne_server();
    s->max_concurrent = max_concurrent;
    s->budget = (size_t)(hbm_budget_gb * 1e9);
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        delete s;
        return nullptr;
    }
    for (int i = 0; i < max_concurrent; i++) s->workers.emplace_back(worker_loop, s);
    return s;
}

int tsne_server_submit(tsne_server_t *s, int n_point, int low_dim, const tsne_params_t *params, sparse_matrix_t *P)
{
    if (s == nullptr || params == nullptr || P == nullptr || n_point < 1 || (low_dim != 2 && low_dim != 3) ||
        P->n_rows != n_point || P->n_cols != n_point)
        return -1;
    std::unique_ptr<Job> job(new Job());
    job->n = n_point;
    job->d = low_dim;
    job->params = *params;
    if (params->init_Y != nullptr && params->init_method == 1)
        job->init_Y.assign(params->init_Y, params->init_Y + (size_t)n_point * low_dim);
    job->params.init_Y = nullptr;
    if (params->enable_profiling && params->profiling_output_file) job->prof_file = params->profiling_output_file;
    job->params.profiling_output_file = nullptr;
    job->P = P;
    job->bytes = job_bytes(n_point, P->row_ptr[n_point]);
    job->t_submit = now_sec();
    int id;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        id = (int)s->jobs.size();
        job->id = id;
        s->jobs.push_back(std::move(job));
        s->queue.push_back(id);
    }
    s->cv_work.notify_all();
    return id;
}

int tsne_server_wait(tsne_server_t *s, int job_id, double *Y_out, tsne_job_info_t *info)
{
    if (s == nullptr) return -1;
    Job *job;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        if (job_id < 0 || job_id >= (int)s->jobs.size()) return -1;
        job = s->jobs[job_id].get();
        s->cv_done.wait(lock, [&] { return job->state >= DONE; });
    }
    if (info != nullptr) {
        info->job = job->id;
        info->status = job->state == DONE ? 0 : -1;
        info->n_point = job->n;
        info->low_dim = job->d;
        info->latency_s = job->t_end - job->t_submit;
        info->queue_s = job->t_start - job->t_submit;
        info->run_s = job->run_s;
        info->kl = job->kl;
        info->start_s = job->t_start;
        info->end_s = job->t_end;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (job->state != DONE || job->collected) return -1;
    if (Y_out != nullptr) memcpy(Y_out, job->Y.data(), sizeof(double) * job->Y.size());
    job->collected = true;
    std::vector<double>().swap(job->Y);   // a long-running server keeps no finished embeddings
    return 0;
}

int tsne_server_pending(tsne_server_t *s)
{
    if (s == nullptr) return -1;
    std::lock_guard<std::mutex> lock(s->mu);
    return (int)s->queue.size() + s->running;
}

void tsne_server_destroy(tsne_server_t *s)
{
    if (s == nullptr) return;
    {
        // jobs that have not started are cancelled; running ones finish
        std::lock_guard<std::mutex> lock(s->mu);
        for (int id : s->queue) {
            s->jobs[id]->state = FAILED;
            s->jobs[id]->t_end = now_sec();
        }
        s->queue.clear();
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (auto &t : s->workers) t.join();
    for (auto &j : s->jobs)
        if (j->P) sparse_matrix_destroy(j->P);
    delete s;
}

}  // extern "C"
