// tw_api.cpp -- host side of the C ABI: context, solve / evaluate / warp entry
// points, the reference's operator-level functions and the TeraWarp command's
// parameter surface.
#include "tw_internal.h"
#include "tw_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

using namespace tw;

namespace tw {

tw_status fail(const tw_ctx *ctx, tw_status code, const std::string &msg)
{
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->err_mu);
        const_cast<tw_ctx *>(ctx)->last_error = msg;
    }
    return code;
}

tw_status dmalloc(tw_ctx *ctx, void **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) return TW_OK;
    size_t prev = ctx->used.fetch_add(bytes);
    if (prev + bytes > ctx->budget) {
        ctx->used.fetch_sub(bytes);
        return fail(ctx, TW_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes exceeds the HBM budget");
    }
    // stream-ordered allocation from the context's pool on its compute
    // stream, made visible to every stream of the context before returning
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        ctx->used.fetch_sub(bytes);
        *p = nullptr;
        cudaGetLastError();
        return fail(ctx, TW_ERR_OOM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    return TW_OK;
}

// Returns a block to the pool once all work queued so far on the context's
// streams is done (callers free only after their last use was enqueued).
void dfree(tw_ctx *ctx, void *p, size_t bytes)
{
    if (!p) return;
    cudaStreamSynchronize(ctx->h2d);
    cudaStreamSynchronize(ctx->d2h);
    cudaFreeAsync(p, ctx->stream);
    ctx->used.fetch_sub(bytes);
}

tw_status dmalloc_on(tw_ctx *ctx, void **p, size_t bytes, cudaStream_t st)
{
    *p = nullptr;
    if (bytes == 0) return TW_OK;
    size_t prev = ctx->used.fetch_add(bytes);
    if (prev + bytes > ctx->budget) {
        ctx->used.fetch_sub(bytes);
        return fail(ctx, TW_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes exceeds the HBM budget");
    }
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, st);
    if (e != cudaSuccess) {
        ctx->used.fetch_sub(bytes);
        *p = nullptr;
        cudaGetLastError();
        return fail(ctx, TW_ERR_OOM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    return TW_OK;
}

void dfree_on(tw_ctx *ctx, void *p, size_t bytes, cudaStream_t st)
{
    if (!p) return;
    cudaFreeAsync(p, st);
    ctx->used.fetch_sub(bytes);
}

tw_status upload(tw_ctx *ctx, void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) return TW_OK;
    if (bytes > tw_ctx::kStageBytes || !ctx->stage_h) {
        TW_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        return TW_OK;
    }
    std::lock_guard<std::mutex> lk(ctx->stage_mu);
    const int s = ctx->stage_next;
    ctx->stage_next = (s + 1) % tw_ctx::kStageSlots;
    TW_CUDA_TRY(cudaEventSynchronize(ctx->stage_ev[s]));  // the slot's previous copy has finished
    unsigned char *h = ctx->stage_h + (size_t)s * tw_ctx::kStageBytes;
    std::memcpy(h, src, bytes);
    TW_CUDA_TRY(cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, st));
    TW_CUDA_TRY(cudaEventRecord(ctx->stage_ev[s], st));
    return TW_OK;
}

tw_status check_kernel_errors(tw_ctx *ctx)
{
    if (!ctx->d_err) return TW_OK;
    int h = 0;
    TW_CUDA_TRY(cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h == 0) return TW_OK;
    TW_CUDA_TRY(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return fail(ctx, TW_ERR_TIMEOUT, "a resample kernel gave up waiting for a staged source plane");
}

int64_t grid_size(int64_t sz, int g) { return (int64_t)std::ceil((double)sz / (double)g) + 3; }

bool is_device_ptr(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool is_pinned_ptr(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Device aux block of a TPS: d (16 doubles) then the status word.
static constexpr size_t kTpsAuxBytes = sizeof(double) * 16 + 16;

// Device-resident TPS field of one job: coefficients + node grid.
tw_status make_tps(tw_ctx *ctx, const tw_marker *centres, const tw_marker *values, int n, double lambda,
                   double scale, cudaStream_t st, tw_tps **out, bool wait, double *h_stage)
{
    *out = nullptr;
    if (!centres || !values || n < 4) return fail(ctx, TW_ERR_ARG, "TPS needs n >= 4 landmark pairs");
    std::unique_ptr<tw_tps> t(new tw_tps);
    t->ctx = ctx;
    t->n = n;
    std::vector<double> hc(3 * (size_t)n), hv(3 * (size_t)n);
    double o[3] = {0, 0, 0};
    for (int i = 0; i < n; ++i) {
        // landmarks go through float (Coord3D_JBA) before the FP64 solve,
        // as in the reference (q_imgwarp_tps_quicksmallmemory.cpp:2039-2046)
        float cx = (float)(scale * centres[i].x), cy = (float)(scale * centres[i].y), cz = (float)(scale * centres[i].z);
        float vx = (float)(scale * values[i].x), vy = (float)(scale * values[i].y), vz = (float)(scale * values[i].z);
        hc[3 * i] = cx; hc[3 * i + 1] = cy; hc[3 * i + 2] = cz;
        hv[3 * i] = vx; hv[3 * i + 1] = vy; hv[3 * i + 2] = vz;
        o[0] += cx; o[1] += cy; o[2] += cz;
    }
    for (int a = 0; a < 3; ++a) o[a] = std::floor(o[a] / n + 0.5);
    // coefficients and the FP32 evaluation arrays (centres relative to o,
    // negated coefficients) are all written on `st` by the solve, which waits
    // for `st` once at its end; after that every stream may use them
    const size_t cbytes = sizeof(double) * 4 * (size_t)n;
    const size_t fbytes = sizeof(float4) * (size_t)n;
    tw_status s = dmalloc_on(ctx, (void **)&t->d_c, cbytes, st);
    if (s == TW_OK) s = dmalloc_on(ctx, (void **)&t->d_ctr32, fbytes, st);
    if (s == TW_OK) s = dmalloc_on(ctx, (void **)&t->d_coef32, fbytes, st);
    if (s == TW_OK) s = dmalloc_on(ctx, (void **)&t->d_d, kTpsAuxBytes, st);
    if (s == TW_OK) {
        t->d_status = reinterpret_cast<int *>(t->d_d + 16);
        s = solve_tps_device(ctx, hc.data(), hv.data(), n, lambda, t->d_c, t->d_d, t->d_status,
                             wait ? t->h_d : nullptr, o, t->d_ctr32, t->d_coef32, st, h_stage);
    }
    if (s != TW_OK) {
        dfree_on(ctx, t->d_c, cbytes, st);
        dfree_on(ctx, t->d_ctr32, fbytes, st);
        dfree_on(ctx, t->d_coef32, fbytes, st);
        dfree_on(ctx, t->d_d, kTpsAuxBytes, st);
        return s;
    }
    for (int a = 0; a < 3; ++a) t->o32[a] = o[a];
    t->h_ctr = new double[3 * (size_t)n];
    std::memcpy(t->h_ctr, hc.data(), sizeof(double) * 3 * n);
    *out = t.release();
    return TW_OK;
}

void destroy_tps(tw_tps *t)
{
    if (!t) return;
    tw_ctx *ctx = t->ctx;
    dfree(ctx, t->d_c, sizeof(double) * 4 * (size_t)t->n);
    dfree(ctx, t->d_ctr32, sizeof(float4) * (size_t)t->n);
    dfree(ctx, t->d_coef32, sizeof(float4) * (size_t)t->n);
    dfree(ctx, t->d_d, kTpsAuxBytes);
    delete[] t->h_ctr;
    delete t;
}

tw_status eval_grid(tw_ctx *ctx, const tw_tps *t, const int64_t gsz[3], int g, const int64_t off[3], float4 *out,
                    cudaStream_t st)
{
    EvalParams p;
    p.ctr = t->d_ctr32;
    p.coef = t->d_coef32;
    p.n = t->n;
    // the affine part stays on the device (the kernel folds it with o), so an
    // evaluation can follow an unwaited solve on the same stream
    p.aff = t->d_d;
    for (int a = 0; a < 3; ++a) p.o[a] = t->o32[a];
    for (int a = 0; a < 3; ++a) {
        p.gsz[a] = gsz[a];
        p.node_o[a] = (int64_t)(-g + off[a] - (int64_t)t->o32[a]);
    }
    p.g = g;
    p.out = out;
    TW_CUDA_TRY(launch_tps_eval(p, st, ctx->sm_count));
    count_launch(ctx);
    return TW_OK;
}

}  // namespace tw

// ===================================================================== ABI

extern "C" {

const char *tw_status_string(tw_status s)
{
    switch (s) {
    case TW_OK: return "ok";
    case TW_ERR_ARG: return "invalid argument";
    case TW_ERR_SINGULAR: return "singular or degenerate landmark system";
    case TW_ERR_OOM: return "out of memory / over HBM budget";
    case TW_ERR_CUDA: return "CUDA error";
    case TW_ERR_TIMEOUT: return "timeout";
    case TW_ERR_IO: return "tile source/sink callback failed";
    case TW_ERR_UNSUPPORTED: return "unsupported";
    case TW_ERR_NOT_READY: return "not ready";
    }
    return "unknown status";
}

int tw_abi_version(void) { return TW_ABI_VERSION; }

static tw_status destroy_partial(tw_ctx *c)
{
    cudaGetLastError();
    tw_ctx_destroy(c);
    return TW_ERR_CUDA;
}

tw_status tw_ctx_create(int device, size_t hbm_budget_bytes, tw_ctx **out)
{
    if (!out) return TW_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return TW_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return TW_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return TW_ERR_CUDA;
    std::unique_ptr<tw_ctx> c(new tw_ctx);
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TW_ERR_CUDA;
    c->sm_count = prop.multiProcessorCount;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return TW_ERR_CUDA;
    c->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(0.9 * (double)fr);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return TW_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking) != cudaSuccess) return TW_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking) != cudaSuccess) return TW_ERR_CUDA;
    // a private pool (not the device's default pool) that caches freed blocks
    // for the context's lifetime, so per-call workspaces cost no cudaMalloc
    cudaMemPoolProps pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &pp) != cudaSuccess) return TW_ERR_CUDA;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    const size_t ring = sizeof(tw::RJob) * tw_ctx::kJobSlots * tw_ctx::kJobsPerSlot;
    if (cudaMallocHost((void **)&c->job_h, ring) != cudaSuccess) return destroy_partial(c.release());
    if (cudaMalloc((void **)&c->job_d, ring) != cudaSuccess) return destroy_partial(c.release());
    for (int s = 0; s < tw_ctx::kJobSlots; ++s)
        if (cudaEventCreateWithFlags(&c->job_ev[s], cudaEventDisableTiming) != cudaSuccess)
            return destroy_partial(c.release());
    if (cudaMallocHost((void **)&c->stage_h, tw_ctx::kStageBytes * tw_ctx::kStageSlots) != cudaSuccess)
        return destroy_partial(c.release());
    if (cudaMalloc((void **)&c->d_err, 256) != cudaSuccess || cudaMemset(c->d_err, 0, 256) != cudaSuccess)
        return destroy_partial(c.release());
    for (int s = 0; s < tw_ctx::kStageSlots; ++s)
        if (cudaEventCreateWithFlags(&c->stage_ev[s], cudaEventDisableTiming) != cudaSuccess)
            return destroy_partial(c.release());
    *out = c.release();
    return TW_OK;
}

tw_status tw_ctx_destroy(tw_ctx *ctx)
{
    if (!ctx) return TW_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->h2d) cudaStreamSynchronize(ctx->h2d);
    if (ctx->d2h) cudaStreamSynchronize(ctx->d2h);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->h2d) cudaStreamDestroy(ctx->h2d);
    if (ctx->d2h) cudaStreamDestroy(ctx->d2h);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    for (int s = 0; s < tw_ctx::kJobSlots; ++s)
        if (ctx->job_ev[s]) cudaEventDestroy(ctx->job_ev[s]);
    if (ctx->job_d) cudaFree(ctx->job_d);
    if (ctx->job_h) cudaFreeHost(ctx->job_h);
    for (int s = 0; s < tw_ctx::kStageSlots; ++s)
        if (ctx->stage_ev[s]) cudaEventDestroy(ctx->stage_ev[s]);
    if (ctx->stage_h) cudaFreeHost(ctx->stage_h);
    if (ctx->d_err) cudaFree(ctx->d_err);
    delete ctx;
    return TW_OK;
}

const char *tw_ctx_last_error(const tw_ctx *ctx)
{
    if (!ctx) return "";
    std::lock_guard<std::mutex> lk(ctx->err_mu);
    return ctx->last_error.c_str();
}

uint64_t tw_ctx_kernel_launches(const tw_ctx *ctx) { return ctx ? ctx->launches.load() : 0; }

void tw_ctx_transfer_bytes(const tw_ctx *ctx, uint64_t *h2d, uint64_t *d2h)
{
    if (h2d) *h2d = ctx ? ctx->h2d_bytes.load() : 0;
    if (d2h) *d2h = ctx ? ctx->d2h_bytes.load() : 0;
}

tw_status tw_ctx_synchronize(tw_ctx *ctx)
{
    if (!ctx) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->h2d));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->d2h));
    return check_kernel_errors(ctx);
}

// Test hook, not part of the public header: sets how long the solve's CTAs
// wait at a grid barrier on this context (0 restores the 30 s default) and
// returns the previous value.  A test shortens it to make the bounded wait
// give up and checks that the solve reports TW_ERR_TIMEOUT and the context
// keeps working.
unsigned long long tw_internal_set_solve_barrier_ns(tw_ctx *ctx, unsigned long long ns)
{
    if (!ctx) return 0;
    return ctx->solve_barrier_ns.exchange(ns ? ns : 30000000000ull);
}

// Test hook, not part of the public header: turns the shared-memory staging
// of TPS resample units on (1) or off (0) for this context and returns the
// previous setting; off, every unit gathers its taps from global memory.
int tw_internal_set_resample_staging(tw_ctx *ctx, int on)
{
    if (!ctx) return 0;
    return ctx->resample_staging.exchange(on ? 1 : 0);
}

int64_t tw_grid_size(int64_t sz, int g) { return g > 0 && sz > 0 ? grid_size(sz, g) : -1; }

tw_status tw_tps_solve(tw_ctx *ctx, const tw_marker *centres, const tw_marker *values, int n, double lambda,
                       tw_tps **out)
{
    if (!ctx || !out) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    return make_tps(ctx, centres, values, n, lambda, 1.0, ctx->stream, out);
}

tw_status tw_tps_destroy(tw_tps *tps)
{
    if (tps) {
        cudaSetDevice(tps->ctx->device);
        destroy_tps(tps);
    }
    return TW_OK;
}

int tw_tps_count(const tw_tps *tps) { return tps ? tps->n : 0; }

tw_status tw_tps_get_coeffs(const tw_tps *tps, double *c, double *d)
{
    if (!tps) return TW_ERR_ARG;
    tw_ctx *ctx = tps->ctx;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    if (c) {
        TW_CUDA_TRY(cudaMemcpyAsync(c, tps->d_c, sizeof(double) * 4 * (size_t)tps->n, cudaMemcpyDeviceToHost,
                                    ctx->stream));
        TW_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    if (d) std::memcpy(d, tps->h_d, sizeof(double) * 16);
    return TW_OK;
}

tw_status tw_tps_eval_grid(tw_ctx *ctx, const tw_tps *tps, int64_t gsz0, int64_t gsz1, int64_t gsz2, int g,
                           int64_t ox, int64_t oy, int64_t oz, void *dev_nodes, void *stream)
{
    if (!ctx || !tps || !dev_nodes || g < 1 || gsz0 < 1 || gsz1 < 1 || gsz2 < 1) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const int64_t gsz[3] = {gsz0, gsz1, gsz2}, off[3] = {ox, oy, oz};
    TW_TRY(eval_grid(ctx, tps, gsz, g, off, static_cast<float4 *>(dev_nodes), st));
    if (!stream) TW_CUDA_TRY(cudaStreamSynchronize(st));
    return TW_OK;
}

tw_status tw_warp_tps_device(tw_ctx *ctx, const void *dev_nodes, int g, int dtype, int interp, const void *dev_src,
                             void *dev_dst, const int64_t sz[3], void *stream)
{
    if (!ctx || !dev_nodes || !dev_src || !dev_dst || !sz) return TW_ERR_ARG;
    if (!g_supported(g)) return fail(ctx, TW_ERR_UNSUPPORTED, "grid spacing must be 4, 8, 16, 32 or 64");
    if ((dtype != TW_U8 && dtype != TW_U16) || (interp != 0 && interp != 1)) return TW_ERR_ARG;
    if (sz[0] < 1 || sz[1] < 1 || sz[2] < 1) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    RJob j = tps_job(dev_src, sz, dev_dst, sz, static_cast<const float4 *>(dev_nodes), g, dtype, interp);
    TW_TRY(run_jobs(ctx, &j, 1, st));
    if (!stream) {
        TW_CUDA_TRY(cudaStreamSynchronize(st));
        return check_kernel_errors(ctx);
    }
    return TW_OK;
}

tw_status tw_warp_affine_device(tw_ctx *ctx, const double M[16], int dtype, int interp, const void *dev_src,
                                const int64_t src_sz[3], void *dev_dst, const int64_t dst_sz[3], void *stream)
{
    if (!ctx || !M || !dev_src || !dev_dst || !src_sz || !dst_sz) return TW_ERR_ARG;
    if ((dtype != TW_U8 && dtype != TW_U16) || (interp != 0 && interp != 1)) return TW_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (src_sz[a] < 1 || dst_sz[a] < 1) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    RJob j = affine_job(dev_src, src_sz, dev_dst, dst_sz, M, dtype, interp);
    TW_TRY(run_jobs(ctx, &j, 1, st));
    if (!stream) TW_CUDA_TRY(cudaStreamSynchronize(st));
    return TW_OK;
}

tw_status tw_fit_affine(tw_ctx *ctx, const tw_marker *tar, const tw_marker *sub, int n, double M[16])
{
    if (!ctx || !tar || !sub || !M) return TW_ERR_ARG;
    if (n < 4) return fail(ctx, TW_ERR_ARG, "affine fit needs n >= 4 landmark pairs");
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    std::vector<double> a(3 * (size_t)n), b(3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        a[3 * i] = tar[i].x; a[3 * i + 1] = tar[i].y; a[3 * i + 2] = tar[i].z;
        b[3 * i] = sub[i].x; b[3 * i + 1] = sub[i].y; b[3 * i + 2] = sub[i].z;
    }
    return fit_affine_device(ctx, a.data(), b.data(), n, M, ctx->stream);
}

tw_status tw_make_affine(int warp_mode, int deformation_mode, const double para[3], const int64_t in_sz[3],
                         const int64_t out_sz[3], double M[16])
{
    if (!para || !M || !in_sz || !out_sz) return TW_ERR_ARG;
    return make_param_affine(warp_mode, deformation_mode, para, in_sz, out_sz, M);
}

}  // extern "C"
