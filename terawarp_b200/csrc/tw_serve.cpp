// tw_serve.cpp -- continuous-batching warp server.
//
// Jobs (affine or TPS, uint8 or uint16, any size) are submitted from any
// thread.  One worker thread owns a private context and loops:
//   1. admission: FIFO, while the HBM reservation of the next job fits the
//      budget and fewer than max_inflight jobs are on the device -- its
//      landmarks are solved (FP64), its node grid evaluated and its source
//      volume copied to HBM on a stream of its own;
//   2. batching: every job whose inputs are resident joins the next resample
//      round; jobs sharing (dtype, kind, g, interp) run in one persistent
//      launch over all their bricks, so work of jobs that arrived at
//      different times overlaps on the device;
//   3. completion: each job's result is copied back on its own stream while
//      later rounds compute, and its latency (submit -> result in host
//      memory) is recorded.
// Every job gives the same voxels alone or batched: the kernels' arithmetic
// depends only on the job, never on the launch it shares.  A job whose source
// or destination is device memory is warped in place (no copy for it), so
// volumes that already live in HBM are served without PCIe traffic.  The
// worker never waits on the host for queued GPU work: landmark uploads go
// through pinned chunks the server owns, job descriptors through the
// context's slot ring.
// The reference has no serving mode.
#include "tw_host.h"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

using namespace tw;

namespace {

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t esize(int dtype) { return dtype == TW_U8 ? 1 : 2; }

enum JobState { kQueued = 0, kPrepared = 1, kComputing = 2, kDone = 3 };

// Landmark staging per in-flight TPS job: centres (3n) and values (4n
// doubles, homogeneous) for up to kLandMax pairs, in pinned memory owned by
// the server, so a solve's uploads never wait on the host.
constexpr int kLandMax = 4096;
constexpr size_t kLandChunk = 7 * (size_t)kLandMax;  // doubles

struct JobRec {
    uint64_t id = 0;
    tw_job spec;
    std::vector<tw_marker> ctr, val;
    double t_submit = 0, t_admit = 0, t_done = 0;
    tw_status status = TW_ERR_NOT_READY;
    int state = kQueued;
    size_t reserve = 0;
    void *d_src = nullptr, *d_dst = nullptr, *d_nodes = nullptr;
    bool own_src = true, own_dst = true;   // false: the caller's device buffer is used in place
    size_t src_b = 0, dst_b = 0, nodes_b = 0;
    tw_tps *tps = nullptr;
    int land = -1;                          // landmark staging chunk
    cudaStream_t st = nullptr;
    // stage timing: admission (job stream), solve done (solve stream), node
    // grid done, inputs resident, resample round start / end (batch
    // stream), result in place
    enum { kT0, kSolve, kGrid, kReady, kRs0, kRs1, kDone, kEv };
    cudaEvent_t ev[kEv] = {};
    double times[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
};

}  // namespace

struct tw_server {
    tw_ctx *ctx = nullptr;  // private context of the worker
    size_t budget = 0, used = 0;
    int max_inflight = 8;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<JobRec *> queued;
    std::map<uint64_t, std::unique_ptr<JobRec>> jobs;
    std::vector<JobRec *> active;
    std::vector<cudaStream_t> streams;
    cudaStream_t batch = nullptr;
    // all solves run on this one stream, one after another: each is a
    // cooperative kernel that wants every SM, and they are short
    cudaStream_t solve_st = nullptr;
    double *land_h = nullptr;               // pinned, max_inflight x kLandChunk doubles
    std::vector<int> land_free;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread worker;
};

namespace {

size_t job_reserve(const JobRec &j)
{
    const tw_job &s = j.spec;
    const size_t es = esize(s.dtype);
    size_t b = (j.own_src ? es * (size_t)(s.src_sz[0] * s.src_sz[1] * s.src_sz[2]) : 0) +
               (j.own_dst ? es * (size_t)(s.dst_sz[0] * s.dst_sz[1] * s.dst_sz[2]) : 0);
    if (s.kind == 1) {
        b += sizeof(float4) * (size_t)(grid_size(s.dst_sz[0], s.g) * grid_size(s.dst_sz[1], s.g) *
                                       grid_size(s.dst_sz[2], s.g));
        const size_t m = s.n > 4 ? (size_t)(s.n - 4) : 0;
        b += sizeof(double) * (m * m + 48 * (size_t)s.n + 64);  // solve workspace
    }
    return b;
}

// Seconds from event a to event b, or -1 when either was not recorded.
double span_s(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    if (!a || !b || cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return -1.0;
    }
    return 1e-3 * ms;
}

void release(tw_server *s, JobRec *j, bool completed)
{
    if (completed) {
        // stage times relative to admission (the job's stream has finished,
        // so every event recorded for it has completed)
        for (int k = JobRec::kSolve; k <= JobRec::kDone; ++k) j->times[k] = span_s(j->ev[JobRec::kT0], j->ev[k]);
    } else if (j->land >= 0) {
        // a job that failed while its uploads may still be queued: the
        // staging chunk is reused only once they have run
        cudaStreamSynchronize(s->solve_st);
    }
    if (j->st) {
        if (j->d_src && j->own_src) cudaFreeAsync(j->d_src, j->st);
        if (j->d_dst && j->own_dst) cudaFreeAsync(j->d_dst, j->st);
        if (j->d_nodes) cudaFreeAsync(j->d_nodes, j->st);
    }
    j->d_src = j->d_dst = j->d_nodes = nullptr;
    if (j->tps) {
        destroy_tps(j->tps);
        j->tps = nullptr;
    }
    if (j->land >= 0) s->land_free.push_back(j->land);
    j->land = -1;
    for (auto &e : j->ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    if (j->st) s->streams.push_back(j->st);
    j->st = nullptr;
    std::vector<tw_marker>().swap(j->ctr);
    std::vector<tw_marker>().swap(j->val);
}

// Puts a job's inputs on the device: FP64 solve + node grid (TPS) and the
// source volume, all on the job's own stream.
tw_status prepare(tw_server *s, JobRec *j)
{
    tw_ctx *ctx = s->ctx;
    const tw_job &sp = j->spec;
    const size_t es = esize(sp.dtype);
    if (s->streams.empty()) {
        cudaStream_t st;
        TW_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        s->streams.push_back(st);
    }
    j->st = s->streams.back();
    s->streams.pop_back();
    j->t_admit = now_s();
    for (auto &e : j->ev) TW_CUDA_TRY(cudaEventCreate(&e));
    TW_CUDA_TRY(cudaEventRecord(j->ev[JobRec::kT0], j->st));
    if (sp.kind == 1) {
        // the solve (on the solve stream, its landmarks staged in the
        // server's pinned chunk), the node grid and the upload (on the job's
        // stream) are queued without a host wait; the solve's status is read
        // at completion
        double *stage = nullptr;
        if (sp.n <= kLandMax && !s->land_free.empty()) {
            j->land = s->land_free.back();
            s->land_free.pop_back();
            stage = s->land_h + (size_t)j->land * kLandChunk;
        }
        TW_CUDA_TRY(cudaStreamWaitEvent(s->solve_st, j->ev[JobRec::kT0], 0));
        TW_TRY(make_tps(ctx, j->ctr.data(), j->val.data(), sp.n, sp.lambda > 0 ? sp.lambda : 0.2, 1.0, s->solve_st,
                        &j->tps, /*wait=*/false, stage));
        TW_CUDA_TRY(cudaEventRecord(j->ev[JobRec::kSolve], s->solve_st));
        TW_CUDA_TRY(cudaStreamWaitEvent(j->st, j->ev[JobRec::kSolve], 0));
        const int64_t gsz[3] = {grid_size(sp.dst_sz[0], sp.g), grid_size(sp.dst_sz[1], sp.g),
                                grid_size(sp.dst_sz[2], sp.g)};
        j->nodes_b = sizeof(float4) * (size_t)(gsz[0] * gsz[1] * gsz[2]);
        TW_CUDA_TRY(cudaMallocFromPoolAsync(&j->d_nodes, j->nodes_b, ctx->pool, j->st));
        const int64_t off[3] = {0, 0, 0};
        TW_TRY(eval_grid(ctx, j->tps, gsz, sp.g, off, static_cast<float4 *>(j->d_nodes), j->st));
        TW_CUDA_TRY(cudaEventRecord(j->ev[JobRec::kGrid], j->st));
    }
    j->src_b = es * (size_t)(sp.src_sz[0] * sp.src_sz[1] * sp.src_sz[2]);
    j->dst_b = es * (size_t)(sp.dst_sz[0] * sp.dst_sz[1] * sp.dst_sz[2]);
    if (j->own_src) {
        TW_CUDA_TRY(cudaMallocFromPoolAsync(&j->d_src, j->src_b, ctx->pool, j->st));
        TW_CUDA_TRY(cudaMemcpyAsync(j->d_src, sp.src, j->src_b, cudaMemcpyHostToDevice, j->st));
    } else {
        j->d_src = const_cast<void *>(sp.src);
    }
    if (j->own_dst) TW_CUDA_TRY(cudaMallocFromPoolAsync(&j->d_dst, j->dst_b, ctx->pool, j->st));
    else j->d_dst = sp.dst;
    TW_CUDA_TRY(cudaEventRecord(j->ev[JobRec::kReady], j->st));
    return TW_OK;
}

// One resample round over every prepared job whose inputs are resident.
tw_status batch_round(tw_server *s, std::vector<JobRec *> &ready)
{
    tw_ctx *ctx = s->ctx;
    std::map<std::tuple<int, int, int, int>, std::vector<JobRec *>> groups;
    for (JobRec *j : ready) groups[{j->spec.dtype, j->spec.kind, j->spec.g, j->spec.interp}].push_back(j);
    for (auto &kv : groups) {
        std::vector<RJob> rj;
        for (JobRec *j : kv.second) {
            TW_CUDA_TRY(cudaStreamWaitEvent(s->batch, j->ev[JobRec::kReady], 0));
            TW_CUDA_TRY(cudaEventRecord(j->ev[JobRec::kRs0], s->batch));
            const tw_job &sp = j->spec;
            if (sp.kind == 1)
                rj.push_back(tps_job(j->d_src, sp.src_sz, j->d_dst, sp.dst_sz, static_cast<const float4 *>(j->d_nodes),
                                     sp.g, sp.dtype, sp.interp));
            else
                rj.push_back(affine_job(j->d_src, sp.src_sz, j->d_dst, sp.dst_sz, sp.M, sp.dtype, sp.interp));
        }
        TW_TRY(run_jobs(ctx, rj.data(), (int)rj.size(), s->batch));
        // each job's stream continues after its own resample-end event, so a
        // job's completion is never stamped before the end of its resample
        for (JobRec *j : kv.second) TW_CUDA_TRY(cudaEventRecord(j->ev[JobRec::kRs1], s->batch));
        for (JobRec *j : kv.second) {
            TW_CUDA_TRY(cudaStreamWaitEvent(j->st, j->ev[JobRec::kRs1], 0));
            if (j->own_dst)
                TW_CUDA_TRY(cudaMemcpyAsync(j->spec.dst, j->d_dst, j->dst_b, cudaMemcpyDeviceToHost, j->st));
            TW_CUDA_TRY(cudaEventRecord(j->ev[JobRec::kDone], j->st));
            j->state = kComputing;
        }
    }
    return TW_OK;
}

void finish(tw_server *s, JobRec *j, tw_status st, bool completed)
{
    release(s, j, completed);
    std::lock_guard<std::mutex> lk(s->mu);
    j->status = st;
    j->t_done = now_s();
    j->times[0] = j->t_admit > 0 ? j->t_admit - j->t_submit : -1.0;
    j->times[7] = j->t_done - j->t_submit;
    j->state = kDone;
    s->used -= j->reserve;
    s->cv_done.notify_all();
}

void worker_main(tw_server *s)
{
    cudaSetDevice(s->ctx->device);
    for (;;) {
        bool progressed = false;
        // 1. admission (FIFO, budget and in-flight bound)
        for (;;) {
            JobRec *j = nullptr;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                if (s->queued.empty() || (int)s->active.size() >= s->max_inflight) break;
                JobRec *h = s->queued.front();
                if (s->used + h->reserve > s->budget && !s->active.empty()) break;  // wait for memory
                s->queued.pop_front();
                s->used += h->reserve;
                j = h;
            }
            progressed = true;
            if (j->reserve > s->budget) {
                finish(s, j, TW_ERR_OOM, false);
                continue;
            }
            tw_status st = prepare(s, j);
            if (st != TW_OK) {
                finish(s, j, st, false);
                continue;
            }
            j->state = kPrepared;
            s->active.push_back(j);
        }
        // 2. batch every prepared job whose inputs are on the device
        std::vector<JobRec *> ready;
        for (JobRec *j : s->active)
            if (j->state == kPrepared && cudaEventQuery(j->ev[JobRec::kReady]) == cudaSuccess) ready.push_back(j);
        if (!ready.empty()) {
            progressed = true;
            tw_status st = batch_round(s, ready);
            if (st != TW_OK)
                for (JobRec *j : ready) j->status = st;
        }
        // 3. completion
        for (size_t i = 0; i < s->active.size();) {
            JobRec *j = s->active[i];
            bool done = false, completed = false;
            tw_status st = TW_OK;
            if (j->state == kComputing) {
                cudaError_t e = cudaEventQuery(j->ev[JobRec::kDone]);
                if (e == cudaSuccess) {
                    done = completed = true;
                    if (j->tps) st = solve_status(s->ctx, j->tps->d_status, j->st);  // stream is idle: no wait
                } else if (e != cudaErrorNotReady) {
                    done = true;
                    st = TW_ERR_CUDA;
                }
            } else if (j->state == kPrepared && j->status != TW_ERR_NOT_READY) {
                done = true;
                st = j->status;
            }
            if (done) {
                progressed = true;
                finish(s, j, st, completed);
                s->active.erase(s->active.begin() + i);
            } else {
                ++i;
            }
        }
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->stop && s->queued.empty() && s->active.empty()) break;
        if (!progressed) s->cv_work.wait_for(lk, std::chrono::microseconds(100));
    }
}

}  // namespace

extern "C" {

tw_status tw_server_create(tw_ctx *ctx, size_t hbm_budget_bytes, int max_inflight, tw_server **out)
{
    if (!ctx || !out) return TW_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<tw_server> s(new tw_server);
    TW_TRY(tw_ctx_create(ctx->device, 0, &s->ctx));
    s->budget = hbm_budget_bytes ? hbm_budget_bytes : s->ctx->budget / 2;
    s->max_inflight = max_inflight > 0 ? max_inflight : 16;
    if (cudaStreamCreateWithFlags(&s->batch, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->solve_st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaHostAlloc((void **)&s->land_h, sizeof(double) * kLandChunk * (size_t)s->max_inflight,
                      cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        if (s->batch) cudaStreamDestroy(s->batch);
        if (s->solve_st) cudaStreamDestroy(s->solve_st);
        tw_ctx_destroy(s->ctx);
        return TW_ERR_CUDA;
    }
    for (int i = s->max_inflight - 1; i >= 0; --i) s->land_free.push_back(i);
    s->worker = std::thread(worker_main, s.get());
    *out = s.release();
    return TW_OK;
}

tw_status tw_server_submit(tw_server *s, const tw_job *job, uint64_t *job_id)
{
    if (!s || !job || !job_id) return TW_ERR_ARG;
    const tw_job &sp = *job;
    if ((sp.dtype != TW_U8 && sp.dtype != TW_U16) || (sp.interp != 0 && sp.interp != 1) || !sp.src || !sp.dst)
        return TW_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (sp.src_sz[a] < 1 || sp.dst_sz[a] < 1) return TW_ERR_ARG;
    if (sp.kind == 1) {
        if (!g_supported(sp.g) || !sp.centres || !sp.values || sp.n < 4) return TW_ERR_ARG;
    } else if (sp.kind != 0) {
        return TW_ERR_ARG;
    }
    std::unique_ptr<JobRec> j(new JobRec);
    j->spec = sp;
    j->own_src = !is_device_ptr(sp.src);  // device buffers are used in place: no copy either way
    j->own_dst = !is_device_ptr(sp.dst);
    if (sp.kind == 1) {
        j->ctr.assign(sp.centres, sp.centres + sp.n);
        j->val.assign(sp.values, sp.values + sp.n);
        j->spec.centres = j->ctr.data();
        j->spec.values = j->val.data();
    }
    j->reserve = job_reserve(*j);
    j->t_submit = now_s();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return TW_ERR_ARG;
    j->id = s->next_id++;
    *job_id = j->id;
    s->queued.push_back(j.get());
    s->jobs[j->id] = std::move(j);
    s->cv_work.notify_one();
    return TW_OK;
}

tw_status tw_server_poll(tw_server *s, uint64_t job_id, double *latency_s)
{
    if (!s) return TW_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return TW_ERR_ARG;
    JobRec *j = it->second.get();
    if (j->state != kDone) return TW_ERR_NOT_READY;
    if (latency_s) *latency_s = j->t_done - j->t_submit;
    return j->status;
}

tw_status tw_server_wait(tw_server *s, uint64_t job_id, double timeout_s, double *latency_s)
{
    if (!s) return TW_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return TW_ERR_ARG;
    JobRec *j = it->second.get();
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (j->state != kDone) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && j->state != kDone)
            return TW_ERR_TIMEOUT;
    }
    if (latency_s) *latency_s = j->t_done - j->t_submit;
    return j->status;
}

tw_status tw_server_destroy(tw_server *s)
{
    if (!s) return TW_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->batch);
    cudaStreamSynchronize(s->solve_st);
    for (cudaStream_t st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    cudaStreamDestroy(s->batch);
    cudaStreamDestroy(s->solve_st);
    if (s->land_h) cudaFreeHost(s->land_h);
    tw_ctx_destroy(s->ctx);
    delete s;
    return TW_OK;
}

tw_status tw_server_job_times(tw_server *s, uint64_t job_id, double times[8])
{
    if (!s || !times) return TW_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return TW_ERR_ARG;
    const JobRec *j = it->second.get();
    if (j->state != kDone) return TW_ERR_NOT_READY;
    for (int k = 0; k < 8; ++k) times[k] = j->times[k];
    return TW_OK;
}

}  // extern "C"
