// tw_internal.h -- shared internals of libterawarp_b200 (not installed).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/terawarp_b200.h"

namespace tw {

// ----------------------------------------------------------------- status

struct Error {
    tw_status code;
    std::string msg;
};

#define TW_CUDA_TRY(expr)                                                              \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return ::tw::fail(ctx, TW_ERR_CUDA, std::string(#expr) + ": " +            \
                                                    cudaGetErrorString(e_));          \
    } while (0)

#define TW_TRY(expr)                                                                   \
    do {                                                                               \
        tw_status s_ = (expr);                                                         \
        if (s_ != TW_OK) return s_;                                                    \
    } while (0)

// ------------------------------------------------------------- resample job

// One warp job as the resample kernel sees it.  All coordinates are voxels;
// "global" means the full subject / output volume of the job.  128-byte
// aligned because the TMA descriptor of the source buffer sits at its start
// (64-byte alignment is the descriptor's own requirement).
struct alignas(128) RJob {
    CUtensorMap tmap;      // 3-D tensor map of the source buffer (x, y, z), one-row boxes (TPS staging)
    const void *src;       // source buffer, first element = global voxel src_o
    void *dst;             // output buffer, first element = global output voxel out_o
    const float4 *nodes;   // TPS node grid (DF, float4), node i at (i-1)g; null for affine
    int64_t src_py, src_pz;   // source buffer pitches (elements)
    int64_t dst_py, dst_pz;   // output buffer pitches (elements)
    int64_t src_o[3];      // global coords of the source buffer's first voxel
    int64_t src_n[3];      // source buffer dims
    int64_t glob[3];       // subject volume dims (OOB rule q in [0, glob-1])
    int64_t out_o[3];      // global output coords of this job's region (multiple of g for TPS)
    int64_t out_n[3];      // region dims
    int64_t gsz[3];        // node grid dims
    double M[12];          // affine rows (kind 0)
    int64_t bricks[3];     // brick counts along x, y, z
    int64_t brick_begin;   // first flattened brick index of this job in its launch
    int g;                 // grid spacing (TPS)
    int zs;                // output planes per TPS work unit (divides g or is a multiple of it; set by run_jobs)
    int tma_ok;            // tmap is valid: TPS units may stage their source footprint in shared memory
    int dtype;             // 1 u8, 2 u16
    int kind;              // 0 affine, 1 TPS
    int interp;            // 0 trilinear, 1 nearest
};

// Launch one resample pass over `njobs` jobs that share (dtype, kind, g).
// jobs_dev is device memory holding the RJob array; total_bricks is the sum
// of all jobs' bricks.  Returns a cudaError_t from the launch.
// err: device word the kernel ORs a failure code into (a bounded wait that
// gave up); may be null.  stage_ws: for trilinear TPS, device memory of
// tps_stage_ws_bytes(total_bricks) whose first 8 bytes are zero: the units
// are planned, staged units run the TMA-staged kernel and the rest the
// gather kernel; null: the gather kernel takes every unit.
cudaError_t launch_resample(const RJob *jobs_dev, int njobs, int64_t total_bricks, int dtype,
                            int kind, int g, int interp, cudaStream_t st, int sm_count, int *err,
                            void *stage_ws);
size_t tps_stage_ws_bytes(int64_t total_bricks);
// Brick extents for a (kind, g) pair: x, y and the z extent a unit's frame
// is anchored to (a control cell layer for TPS).
void brick_dims(int kind, int g, int64_t out[3]);
// Fills j.tmap / j.tma_ok for a TPS job (false when the source buffer's
// address or pitches do not meet the TMA rules; the job then gathers).
bool encode_source_map(RJob &j);
// Device error word bits set by the resample kernels.
constexpr int kKernErrTimeout = 1;
// The TMA box of the staged TPS path: source elements per staged row and rows
// per staged plane (the staged box of a unit is at most this large).  A row
// of 128 elements keeps the row pitch in shared memory a multiple of 32
// banks, so a warp whose taps straddle two rows reads them without bank
// conflicts.
constexpr int kStageBoxW = 128;
constexpr int kStageBoxH = 32;

// ---------------------------------------------------------------- TPS eval

struct EvalParams {
    const float4 *ctr;     // n centres, relative to the job origin `o`
    const float4 *coef;    // n coefficients (-c_x, -c_y, -c_z, 0)
    int n;
    const double *aff;     // device 4 x 4 FP64 affine part d of the TPS (row-major)
    double o[3];           // the origin: a0 / alin are folded from aff and o on the device
    int64_t gsz[3];
    int g;
    int64_t node_o[3];     // position of node (0,0,0) relative to the origin
    float4 *out;
};
cudaError_t launch_tps_eval(const EvalParams &p, cudaStream_t st, int sm_count);

// ------------------------------------------------------------------- solve

struct SolveWork;   // device workspace of one solve
// Solves on `st`: c into d_c_out (n x 4), d into d_d_out (4 x 4) and the
// status bits into d_status_out, all device memory that outlives the call.
// With h_d_out it waits for `st` once, at the end, copies d to the host and
// turns the status into the return value; without it nothing waits and the
// caller reads the status later (solve_status).  When ctr32_out and
// coef32_out are given it also writes the FP32 evaluation arrays: centres
// relative to `o` and the negated non-affine coefficients (-c_x, -c_y, -c_z).
// h_stage: optional pinned host memory of at least 7n doubles that stays
// untouched until the solve's copies have run (the caller owns it); the
// landmark uploads then go through it instead of the context's staging ring,
// so the host never waits for earlier work queued on `st`.
tw_status solve_tps_device(tw_ctx *ctx, const double *h_ctr, const double *h_val, int n, double lambda,
                           double *d_c_out, double *d_d_out, int *d_status_out, double *h_d_out,
                           const double o[3], float4 *ctr32_out, float4 *coef32_out, cudaStream_t st,
                           double *h_stage = nullptr);
// The status word of a solve as a tw_status (waits for `st`).
tw_status solve_status(tw_ctx *ctx, const int *d_status, cudaStream_t st);
tw_status fit_affine_device(tw_ctx *ctx, const double *h_tar, const double *h_sub, int n, double M[16],
                            cudaStream_t st);
// The affine fit kernel alone on caller-provided device buffers (d_status
// must hold 0 when it starts; the kernel only sets failure bits).
cudaError_t launch_affine_fit(const double *d_tar, const double *d_sub, int n, double *d_out, int *d_status,
                              cudaStream_t st);

// --------------------------------------------------------------- helpers

int64_t grid_size(int64_t sz, int g);
bool g_supported(int g);

}  // namespace tw

// ------------------------------------------------------------- the context

struct tw_ctx {
    int device = 0;
    int sm_count = 148;
    size_t budget = 0;
    std::atomic<size_t> used{0};
    cudaStream_t stream = nullptr;      // compute
    cudaStream_t h2d = nullptr;         // host -> device copies
    cudaStream_t d2h = nullptr;         // device -> host copies
    cudaMemPool_t pool = nullptr;       // stream-ordered pool that keeps freed blocks
    // Job descriptors of resample launches: a ring of slots, each a pinned
    // host staging area with its device copy.  A slot is reused once the
    // launch that last read it has completed (its event), so a launch of up
    // to kJobsPerSlot jobs needs no allocation and no host wait.
    static constexpr int kJobSlots = 32;
    static constexpr int kJobsPerSlot = 64;
    std::mutex job_mu;
    tw::RJob *job_h = nullptr;          // pinned, kJobSlots x kJobsPerSlot
    tw::RJob *job_d = nullptr;          // device, same shape
    cudaEvent_t job_ev[kJobSlots] = {};
    int job_next = 0;
    // pinned staging ring for small host -> device uploads (landmarks, ...)
    static constexpr int kStageSlots = 8;
    static constexpr size_t kStageBytes = (size_t)1 << 20;
    std::mutex stage_mu;
    unsigned char *stage_h = nullptr;   // pinned, kStageSlots x kStageBytes
    cudaEvent_t stage_ev[kStageSlots] = {};
    int stage_next = 0;
    std::atomic<uint64_t> launches{0};
    std::atomic<uint64_t> h2d_bytes{0}, d2h_bytes{0};  // streamed by the slab and tile paths
    int *d_err = nullptr;               // device word: kernels OR failure bits into it (kKernErrTimeout)
    // how long a CTA of the cooperative solve waits at a grid barrier before
    // it gives up (TW_ERR_TIMEOUT); tests shorten it through
    // tw_internal_set_solve_barrier_ns
    std::atomic<unsigned long long> solve_barrier_ns{30000000000ull};
    // TPS resample units may stage their source footprint in shared memory
    // (TMA); tests turn it off through tw_internal_set_resample_staging to
    // compare the staged output with the gathered one
    std::atomic<int> resample_staging{1};
    mutable std::mutex err_mu;
    std::string last_error;
};

struct tw_tps {
    tw_ctx *ctx = nullptr;
    int n = 0;
    double *d_c = nullptr;     // device n x 4 (FP64)
    double h_d[16] = {0};      // host 4 x 4 (FP64), valid once the solve was waited for
    double *d_d = nullptr;     // device 4 x 4 (FP64)
    int *d_status = nullptr;   // device solve status bits
    float4 *d_ctr32 = nullptr; // centres, FP32, relative to origin o32
    float4 *d_coef32 = nullptr;
    double o32[3] = {0, 0, 0};
    double *h_ctr = nullptr;   // host copy of centres (FP64 from float input)
};

namespace tw {
tw_status fail(const tw_ctx *ctx, tw_status code, const std::string &msg);
// Budgeted device allocation.
tw_status dmalloc(tw_ctx *ctx, void **p, size_t bytes);
void dfree(tw_ctx *ctx, void *p, size_t bytes);
// Budgeted stream-ordered allocation on `st`, without a host wait: valid for
// work queued on `st` after it, and for other streams only once the host has
// waited for `st`.  dfree_on returns the block on `st`.
tw_status dmalloc_on(tw_ctx *ctx, void **p, size_t bytes, cudaStream_t st);
void dfree_on(tw_ctx *ctx, void *p, size_t bytes, cudaStream_t st);
// Host -> device copy on `st` through the context's pinned staging ring, so
// the host does not wait for earlier work on `st` (a pageable copy would);
// copies larger than a staging slot fall back to a pageable copy.
tw_status upload(tw_ctx *ctx, void *dst, const void *src, size_t bytes, cudaStream_t st);
inline void count_launch(tw_ctx *ctx, uint64_t k = 1) { if (ctx) ctx->launches += k; }
// Reads and clears the context's device error word (call after the work that
// may have set it has completed); TW_ERR_TIMEOUT when a kernel gave up on a
// bounded wait.
tw_status check_kernel_errors(tw_ctx *ctx);
}  // namespace tw
