// tw_noalloc.cu -- tw_fit_affine_noalloc: the affine landmark fit with its
// scratch in one fixed device array instead of the context's memory pool.
//
// The fit itself is the same kernel tw_fit_affine launches (3-D DLT with
// Hartley normalisation, FP64), so the two return the same matrix.  What
// differs is only where the landmark copies, the result and the status word
// live: in g_fit_scratch below, whose address is looked up once per device
// context (again if that context was destroyed and created anew).

#include <cuda.h>

#include <mutex>

#include "tw_internal.h"

namespace tw {
namespace {

constexpr int kMaxN = TW_FIT_AFFINE_NOALLOC_MAX;
constexpr int kMaxDevices = 64;

// Layout, in doubles, for n <= kMaxN landmark pairs:
//   [0, 3N)        target coordinates, FP64 (x, y, z per pair)
//   [3N, 6N)       subject coordinates, FP64
//   [6N, 9N)       the tw_marker arrays as copied from the host: 3N floats of
//                  target, then 3N floats of subject
//   [9N, 9N + 16)  the fitted 4x4 matrix
//   [9N + 16]      status word (int); must be 0 when the fit kernel starts,
//                  k_stage_markers clears it on every call
constexpr size_t kScratchDoubles = 9 * (size_t)kMaxN + 17;
static __device__ __align__(256) double g_fit_scratch[kScratchDoubles];

// g_fit_scratch's device address on each device, and the id of the device
// context it was looked up in (0 = unknown).  A context that was destroyed
// (cudaDeviceReset) and created again has a new id, so the lookup is redone
// instead of handing the kernel an address from the old context.
struct ScratchAddr {
    double *ptr = nullptr;
    unsigned long long ctx_id = 0;
};
std::mutex g_mu[kMaxDevices];              // one caller at a time per device
ScratchAddr g_addr[kMaxDevices];

static_assert(sizeof(tw_marker) == 3 * sizeof(float), "tw_marker must be three packed floats");

__global__ void k_stage_markers(const float *t32, const float *s32, int m, double *t, double *s, int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *status = 0;
    for (int k = i; k < m; k += gridDim.x * blockDim.x) {
        t[k] = t32[k];
        s[k] = s32[k];
    }
}

// Id of the calling thread's current device context through the driver API
// (looked up through the runtime, so the library needs no -lcuda); 0 when the
// driver offers no such query.
unsigned long long current_ctx_id()
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Puts the caller's current device back when the call returns.
struct DeviceRestore {
    int dev = -1;
    DeviceRestore() { if (cudaGetDevice(&dev) != cudaSuccess) { dev = -1; cudaGetLastError(); } }
    ~DeviceRestore() { if (dev >= 0) cudaSetDevice(dev); }
};

// Waits for the context's stream before the per-device lock is released, on
// every return path: work already queued on the scratch array (copies, the
// fit kernel) must finish before another call may touch it.
struct StreamDrain {
    cudaStream_t st;
    ~StreamDrain()
    {
        if (st && cudaStreamSynchronize(st) != cudaSuccess) cudaGetLastError();
    }
};

}  // namespace
}  // namespace tw

using namespace tw;

tw_status tw_fit_affine_noalloc(tw_ctx *ctx, const tw_marker *tar, const tw_marker *sub, int n, double M[16])
{
    if (!ctx || !tar || !sub || !M) return TW_ERR_ARG;
    if (n < 4) return fail(ctx, TW_ERR_ARG, "affine fit needs n >= 4 landmark pairs");
    if (n > kMaxN)
        return fail(ctx, TW_ERR_ARG,
                    "tw_fit_affine_noalloc takes at most TW_FIT_AFFINE_NOALLOC_MAX (4096) landmark pairs; "
                    "use tw_fit_affine for more");
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return fail(ctx, TW_ERR_ARG, "tw_fit_affine_noalloc supports device indices 0..63");
    DeviceRestore restore;
    std::lock_guard<std::mutex> lock(g_mu[ctx->device]);
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    StreamDrain drain{ctx->stream};  // declared after the lock: runs before it is released
    ScratchAddr &sa = g_addr[ctx->device];
    const unsigned long long id = current_ctx_id();
    if (!sa.ptr || (id != 0 && id != sa.ctx_id)) {
        // set-up, once per device context, with that device current
        double *p = nullptr;
        TW_CUDA_TRY(cudaGetSymbolAddress((void **)&p, g_fit_scratch));
        sa.ptr = p;
        sa.ctx_id = id;
    }
    double *base = sa.ptr;
    double *t64 = base;
    double *s64 = base + 3 * (size_t)kMaxN;
    float *t32 = reinterpret_cast<float *>(base + 6 * (size_t)kMaxN);
    float *s32 = t32 + 3 * (size_t)kMaxN;
    double *out = base + 9 * (size_t)kMaxN;
    int *status = reinterpret_cast<int *>(out + 16);

    cudaStream_t st = ctx->stream;
    const int m = 3 * n;
    TW_CUDA_TRY(cudaMemcpyAsync(t32, tar, sizeof(tw_marker) * (size_t)n, cudaMemcpyHostToDevice, st));
    TW_CUDA_TRY(cudaMemcpyAsync(s32, sub, sizeof(tw_marker) * (size_t)n, cudaMemcpyHostToDevice, st));
    k_stage_markers<<<(m + 255) / 256, 256, 0, st>>>(t32, s32, m, t64, s64, status);
    TW_CUDA_TRY(cudaGetLastError());
    TW_CUDA_TRY(launch_affine_fit(t64, s64, n, out, status, st));
    count_launch(ctx, 2);
    int h_status = 0;
    TW_CUDA_TRY(cudaMemcpyAsync(M, out, sizeof(double) * 16, cudaMemcpyDeviceToHost, st));
    TW_CUDA_TRY(cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    TW_CUDA_TRY(cudaStreamSynchronize(st));
    if (h_status) return fail(ctx, TW_ERR_SINGULAR, "affine DLT is degenerate (h13 = 0)");
    return TW_OK;
}
