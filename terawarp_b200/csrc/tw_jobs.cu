// tw_jobs.cu -- resample job construction and launch, sample-hull kernels for
// footprint planning, the parameter-surface matrices, and the slab pipeline
// that streams host volumes through HBM with H2D / compute / D2H overlapped.
#include "tw_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>

namespace tw {

RJob tps_job(const void *src, const int64_t src_sz[3], void *dst, const int64_t dst_sz[3], const float4 *nodes, int g,
             int dtype, int interp)
{
    RJob j;
    std::memset(&j, 0, sizeof(j));
    j.src = src;
    j.dst = dst;
    j.nodes = nodes;
    j.src_py = src_sz[0];
    j.src_pz = src_sz[0] * src_sz[1];
    j.dst_py = dst_sz[0];
    j.dst_pz = dst_sz[0] * dst_sz[1];
    for (int a = 0; a < 3; ++a) {
        j.src_o[a] = 0;
        j.src_n[a] = src_sz[a];
        j.glob[a] = src_sz[a];
        j.out_o[a] = 0;
        j.out_n[a] = dst_sz[a];
        j.gsz[a] = grid_size(dst_sz[a], g);
    }
    j.g = g;
    j.dtype = dtype;
    j.kind = 1;
    j.interp = interp;
    return j;
}

RJob affine_job(const void *src, const int64_t src_sz[3], void *dst, const int64_t dst_sz[3], const double M[16],
                int dtype, int interp)
{
    RJob j;
    std::memset(&j, 0, sizeof(j));
    j.src = src;
    j.dst = dst;
    j.src_py = src_sz[0];
    j.src_pz = src_sz[0] * src_sz[1];
    j.dst_py = dst_sz[0];
    j.dst_pz = dst_sz[0] * dst_sz[1];
    for (int a = 0; a < 3; ++a) {
        j.src_o[a] = 0;
        j.src_n[a] = src_sz[a];
        j.glob[a] = src_sz[a];
        j.out_o[a] = 0;
        j.out_n[a] = dst_sz[a];
    }
    for (int i = 0; i < 12; ++i) j.M[i] = M[i];
    j.g = 0;
    j.dtype = dtype;
    j.kind = 0;
    j.interp = interp;
    return j;
}

namespace {

// A stream-ordered pool block returned on its stream when the scope ends.
struct StreamBlock {
    tw_ctx *ctx = nullptr;
    cudaStream_t st = nullptr;
    void *p = nullptr;
    size_t bytes = 0;
    ~StreamBlock() { if (p) dfree_on(ctx, p, bytes, st); }
};

}  // namespace

tw_status run_jobs(tw_ctx *ctx, RJob *jobs, int njobs, cudaStream_t st)
{
    if (njobs <= 0) return TW_OK;
    int64_t total = 0;
    auto count = [&](int zs) {
        total = 0;
        for (int i = 0; i < njobs; ++i) {
            int64_t bd[3];
            brick_dims(jobs[i].kind, jobs[i].g, bd);
            if (jobs[i].kind == 1) bd[2] = zs;
            jobs[i].zs = zs;
            for (int a = 0; a < 3; ++a) jobs[i].bricks[a] = (jobs[i].out_n[a] + bd[a] - 1) / bd[a];
            jobs[i].brick_begin = total;
            total += jobs[i].bricks[0] * jobs[i].bricks[1] * jobs[i].bricks[2];
        }
    };
    // TPS units walk 64 output planes (several cell layers: the staged source
    // window is loaded once per walk); when a launch has too few units to
    // fill every SM a few times, they get shorter, down to parts of a layer
    int zs = jobs[0].kind == 1 ? std::max(64, jobs[0].g) : 8;
    count(zs);
    while (jobs[0].kind == 1 && zs > 1 && total < 8 * (int64_t)ctx->sm_count) {
        zs /= 2;
        count(zs);
    }
    if (total == 0) return TW_OK;
    bool staged = false;  // some job's source can be staged by TMA
    if (jobs[0].kind == 1 && jobs[0].interp == 0)
        for (int i = 0; i < njobs; ++i) {
            if (ctx->resample_staging.load()) encode_source_map(jobs[i]);
            else jobs[i].tma_ok = 0;
            staged = staged || jobs[i].tma_ok;
        }
    // the units' staging plans and the list of units left to the gather kernel
    StreamBlock fb{ctx, st};
    if (staged) {
        fb.bytes = tps_stage_ws_bytes(total);
        TW_TRY(dmalloc_on(ctx, &fb.p, fb.bytes, st));
        TW_CUDA_TRY(cudaMemsetAsync(fb.p, 0, sizeof(int64_t), st));
    }
    void *d_fb = fb.p;
    // plan, walk lists, staged (interior walks), staged (other walks), gather
    const uint64_t launches = staged ? 5 : 1;
    const size_t bytes = sizeof(RJob) * (size_t)njobs;
    if (njobs <= tw_ctx::kJobsPerSlot && ctx->job_d) {
        // descriptors through the context's slot ring: an asynchronous copy
        // from pinned memory, so the host never waits for earlier work here
        std::lock_guard<std::mutex> lk(ctx->job_mu);
        const int s = ctx->job_next;
        ctx->job_next = (s + 1) % tw_ctx::kJobSlots;
        TW_CUDA_TRY(cudaEventSynchronize(ctx->job_ev[s]));  // the slot's previous launch has finished
        RJob *h = ctx->job_h + (size_t)s * tw_ctx::kJobsPerSlot;
        RJob *d = ctx->job_d + (size_t)s * tw_ctx::kJobsPerSlot;
        std::memcpy(h, jobs, bytes);
        TW_CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
        cudaError_t e = launch_resample(d, njobs, total, jobs[0].dtype, jobs[0].kind, jobs[0].g, jobs[0].interp, st,
                                        ctx->sm_count, ctx->d_err, d_fb);
        if (e != cudaSuccess) return fail(ctx, TW_ERR_CUDA, std::string("resample launch: ") + cudaGetErrorString(e));
        TW_CUDA_TRY(cudaEventRecord(ctx->job_ev[s], st));
        count_launch(ctx, launches);
        return TW_OK;
    }
    RJob *d_jobs = nullptr;
    TW_CUDA_TRY(cudaMallocAsync((void **)&d_jobs, bytes, st));
    TW_CUDA_TRY(cudaMemcpyAsync(d_jobs, jobs, bytes, cudaMemcpyHostToDevice, st));
    cudaError_t e = launch_resample(d_jobs, njobs, total, jobs[0].dtype, jobs[0].kind, jobs[0].g, jobs[0].interp, st,
                                    ctx->sm_count, ctx->d_err, d_fb);
    cudaFreeAsync(d_jobs, st);
    if (e != cudaSuccess) return fail(ctx, TW_ERR_CUDA, std::string("resample launch: ") + cudaGetErrorString(e));
    count_launch(ctx, launches);
    return TW_OK;
}

// ------------------------------------------------------- TMA descriptors

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link the driver API); null when the driver lacks it.
EncodeTiled encode_fn()
{
    static EncodeTiled fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiled) nullptr;
        }
        return reinterpret_cast<EncodeTiled>(f);
    }();
    return fn;
}

}  // namespace

bool encode_source_map(RJob &j)
{
    j.tma_ok = 0;
    const EncodeTiled fn = encode_fn();
    if (!fn || !j.src) return false;
    const uint64_t es = j.dtype == TW_U8 ? 1 : 2;
    // TMA rules: 16-byte aligned base and row / plane pitches; a box (one
    // staged plane: kStageBoxW x kStageBoxH elements) no larger than the tensor
    if (reinterpret_cast<uintptr_t>(j.src) % 16 != 0) return false;
    if ((j.src_py * es) % 16 != 0 || (j.src_pz * es) % 16 != 0) return false;
    if (j.src_n[0] < kStageBoxW || j.src_n[1] < kStageBoxH || j.src_n[2] < 1) return false;
    if (j.src_n[0] > 0xffffffffLL || j.src_n[1] > 0xffffffffLL || j.src_n[2] > 0xffffffffLL) return false;
    if ((uint64_t)j.src_pz * es >= (1ull << 40)) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)j.src_n[0], (cuuint64_t)j.src_n[1], (cuuint64_t)j.src_n[2]};
    const cuuint64_t strides[2] = {(cuuint64_t)j.src_py * es, (cuuint64_t)j.src_pz * es};
    const cuuint32_t box[3] = {(cuuint32_t)kStageBoxW, (cuuint32_t)kStageBoxH, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(&j.tmap, es == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 3,
                          const_cast<void *>(j.src), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    j.tma_ok = 1;
    return true;
}

// ------------------------------------------------------------ sample hulls

namespace {

__device__ __forceinline__ void warp_minmax(float &mn, float &mx)
{
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
}

// One CTA per output cell-layer cz: min/max of q_z = DF_z + (k-1)g over node
// planes k = cz..cz+3 (convex-hull bound of the cubic B-spline).
__global__ void k_layer_zhull(const float4 *nodes, int64_t gx, int64_t gy, int g, float *zmin, float *zmax)
{
    __shared__ float smn[32], smx[32];
    const int cz = blockIdx.x;
    float mn = 3.4e38f, mx = -3.4e38f;
    const int64_t plane = gx * gy;
    for (int k = 0; k < 4; ++k) {
        const float zpos = (float)((int64_t)(cz + k - 1) * g);
        const float4 *p = nodes + (int64_t)(cz + k) * plane;
        for (int64_t i = threadIdx.x; i < plane; i += blockDim.x) {
            float q = p[i].z + zpos;
            mn = fminf(mn, q);
            mx = fmaxf(mx, q);
        }
    }
    warp_minmax(mn, mx);
    if ((threadIdx.x & 31) == 0) { smn[threadIdx.x >> 5] = mn; smx[threadIdx.x >> 5] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { mn = fminf(mn, smn[w]); mx = fmaxf(mx, smx[w]); }
        zmin[cz] = fminf(mn, smn[0]);
        zmax[cz] = fmaxf(mx, smx[0]);
    }
}

// One CTA per box: min/max of q = DF + node position over nodes
// [c0, c1 + 3) on each axis (clamped to the grid).
__global__ void k_box_hull(const float4 *nodes, int64_t gx, int64_t gy, int64_t gz, int g, const int64_t *boxes,
                           float *lo, float *hi)
{
    __shared__ float sm[6][32];
    const int64_t *b = boxes + 6 * blockIdx.x;
    int64_t n0[3], n1[3];
    const int64_t gs[3] = {gx, gy, gz};
    for (int a = 0; a < 3; ++a) {
        n0[a] = b[a];
        n1[a] = b[3 + a] + 3;
        if (n1[a] > gs[a]) n1[a] = gs[a];
    }
    const int64_t ex = n1[0] - n0[0], ey = n1[1] - n0[1], ez = n1[2] - n0[2];
    const int64_t tot = ex * ey * ez;
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int64_t i = threadIdx.x; i < tot; i += blockDim.x) {
        int64_t x = n0[0] + i % ex, t = i / ex;
        int64_t y = n0[1] + t % ey, z = n0[2] + t / ey;
        float4 d = nodes[(z * gy + y) * gx + x];
        float q[3] = {d.x + (float)((x - 1) * g), d.y + (float)((y - 1) * g), d.z + (float)((z - 1) * g)};
        for (int a = 0; a < 3; ++a) { mn[a] = fminf(mn[a], q[a]); mx[a] = fmaxf(mx[a], q[a]); }
    }
    for (int a = 0; a < 3; ++a) warp_minmax(mn[a], mx[a]);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) { sm[a][w] = mn[a]; sm[3 + a][w] = mx[a]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) {
            float m0 = sm[a][0], m1 = sm[3 + a][0];
            for (int k = 1; k < (int)(blockDim.x >> 5); ++k) { m0 = fminf(m0, sm[a][k]); m1 = fmaxf(m1, sm[3 + a][k]); }
            lo[3 * blockIdx.x + a] = m0;
            hi[3 * blockIdx.x + a] = m1;
        }
    }
}

}  // namespace

tw_status tps_layer_zhull(tw_ctx *ctx, const float4 *nodes, const int64_t gsz[3], int g, cudaStream_t st,
                          std::vector<float> &zmin, std::vector<float> &zmax)
{
    const int64_t layers = gsz[2] - 3;
    zmin.assign(layers, 0.f);
    zmax.assign(layers, 0.f);
    if (layers <= 0) return TW_OK;
    float *d = nullptr;
    TW_CUDA_TRY(cudaMallocAsync((void **)&d, sizeof(float) * 2 * layers, st));
    k_layer_zhull<<<(unsigned)layers, 256, 0, st>>>(nodes, gsz[0], gsz[1], g, d, d + layers);
    TW_CUDA_TRY(cudaGetLastError());
    count_launch(ctx);
    TW_CUDA_TRY(cudaMemcpyAsync(zmin.data(), d, sizeof(float) * layers, cudaMemcpyDeviceToHost, st));
    TW_CUDA_TRY(cudaMemcpyAsync(zmax.data(), d + layers, sizeof(float) * layers, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(d, st);
    TW_CUDA_TRY(cudaStreamSynchronize(st));
    return TW_OK;
}

tw_status tps_box_hull(tw_ctx *ctx, const float4 *nodes, const int64_t gsz[3], int g,
                       const std::vector<CellBox> &boxes, cudaStream_t st, std::vector<float> &lo,
                       std::vector<float> &hi)
{
    const size_t nb = boxes.size();
    lo.assign(3 * nb, 0.f);
    hi.assign(3 * nb, 0.f);
    if (nb == 0) return TW_OK;
    std::vector<int64_t> hb(6 * nb);
    for (size_t i = 0; i < nb; ++i)
        for (int a = 0; a < 3; ++a) {
            hb[6 * i + a] = boxes[i].c0[a];
            hb[6 * i + 3 + a] = boxes[i].c1[a];
        }
    int64_t *db = nullptr;
    float *dh = nullptr;
    TW_CUDA_TRY(cudaMallocAsync((void **)&db, sizeof(int64_t) * 6 * nb, st));
    TW_CUDA_TRY(cudaMallocAsync((void **)&dh, sizeof(float) * 6 * nb, st));
    TW_CUDA_TRY(cudaMemcpyAsync(db, hb.data(), sizeof(int64_t) * 6 * nb, cudaMemcpyHostToDevice, st));
    k_box_hull<<<(unsigned)nb, 256, 0, st>>>(nodes, gsz[0], gsz[1], gsz[2], g, db, dh, dh + 3 * nb);
    TW_CUDA_TRY(cudaGetLastError());
    count_launch(ctx);
    TW_CUDA_TRY(cudaMemcpyAsync(lo.data(), dh, sizeof(float) * 3 * nb, cudaMemcpyDeviceToHost, st));
    TW_CUDA_TRY(cudaMemcpyAsync(hi.data(), dh + 3 * nb, sizeof(float) * 3 * nb, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(db, st);
    cudaFreeAsync(dh, st);
    TW_CUDA_TRY(cudaStreamSynchronize(st));
    return TW_OK;
}

// ------------------------------------------------------- parameter surface

namespace {
void mat_mul4(const double *a, const double *b, double *c)
{
    double t[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += a[i * 4 + k] * b[k * 4 + j];
            t[i * 4 + j] = s;
        }
    std::memcpy(c, t, sizeof(t));
}
void ident4(double *m)
{
    for (int i = 0; i < 16; ++i) m[i] = (i % 5 == 0) ? 1.0 : 0.0;
}
}  // namespace

tw_status make_param_affine(int warp_mode, int deformation_mode, const double para[3], const int64_t in_sz[3],
                            const int64_t out_sz[3], double M[16])
{
    ident4(M);
    if (warp_mode == 0 && deformation_mode == 2) {
        // scaling about the origin voxel: out(p) = in(p / s)
        for (int a = 0; a < 3; ++a) {
            if (!(para[a] > 0.0)) return TW_ERR_ARG;
            M[a * 5] = 1.0 / para[a];
        }
        return TW_OK;
    }
    if (warp_mode == 1 && deformation_mode == 1) {
        // translation: out(p) = in(p - t)
        for (int a = 0; a < 3; ++a) M[a * 4 + 3] = -para[a];
        return TW_OK;
    }
    if (warp_mode == 1 && deformation_mode == 0) {
        // rotation by angles (degrees) about x, then y, then z, about the
        // input centre, which lands on the output centre:
        //   forward  p_out = c_out + Rz Ry Rx (p_in - c_in)
        //   pull-back p_in = c_in + (Rz Ry Rx)^T (p_out - c_out)
        const double d2r = std::acos(-1.0) / 180.0;
        const double ax = para[0] * d2r, ay = para[1] * d2r, az = para[2] * d2r;
        double Rx[16], Ry[16], Rz[16], R[16];
        ident4(Rx); ident4(Ry); ident4(Rz);
        Rx[5] = std::cos(ax); Rx[6] = -std::sin(ax); Rx[9] = std::sin(ax); Rx[10] = std::cos(ax);
        Ry[0] = std::cos(ay); Ry[2] = std::sin(ay); Ry[8] = -std::sin(ay); Ry[10] = std::cos(ay);
        Rz[0] = std::cos(az); Rz[1] = -std::sin(az); Rz[4] = std::sin(az); Rz[5] = std::cos(az);
        mat_mul4(Ry, Rx, R);
        mat_mul4(Rz, R, R);
        double ci[3], co[3];
        for (int a = 0; a < 3; ++a) {
            ci[a] = 0.5 * (double)(in_sz[a] - 1);
            co[a] = 0.5 * (double)(out_sz[a] - 1);
        }
        for (int r = 0; r < 3; ++r) {
            double t = ci[r];
            for (int c = 0; c < 3; ++c) {
                M[r * 4 + c] = R[c * 4 + r];  // transpose
                t -= R[c * 4 + r] * co[c];
            }
            M[r * 4 + 3] = t;
        }
        return TW_OK;
    }
    return TW_ERR_ARG;
}

// ---------------------------------------------------------- slab pipeline

namespace {

struct Pinned {
    void *p = nullptr;
    size_t bytes = 0;
    ~Pinned() { if (p) cudaFreeHost(p); }
};

struct Events {
    std::vector<cudaEvent_t> ev;
    ~Events() { for (auto e : ev) cudaEventDestroy(e); }
    cudaError_t make(size_t n)
    {
        ev.resize(n, nullptr);
        for (auto &e : ev) {
            cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    }
};

}  // namespace

tw_status stream_slabs(tw_ctx *ctx, const SlabIO &io,
                       const std::function<void(int64_t, int64_t, int64_t &, int64_t &)> &need,
                       const std::function<tw_status(int64_t, int64_t, const void *, void *, cudaStream_t)> &compute)
{
    const bool src_dev = is_device_ptr(io.src), dst_dev = is_device_ptr(io.dst);
    const bool src_pin = !src_dev && is_pinned_ptr(io.src), dst_pin = !dst_dev && is_pinned_ptr(io.dst);
    const size_t src_bytes = io.src_plane_bytes * (size_t)io.src_planes;
    const size_t dst_bytes = io.dst_plane_bytes * (size_t)io.dst_planes;
    void *d_src = src_dev ? const_cast<void *>(io.src) : nullptr;
    void *d_dst = dst_dev ? io.dst : nullptr;
    struct Guard {
        tw_ctx *c; void *p; size_t b;
        ~Guard() { if (p) dfree(c, p, b); }
    } gs{ctx, nullptr, 0}, gd{ctx, nullptr, 0};
    if (!src_dev) {
        TW_TRY(dmalloc(ctx, &d_src, src_bytes));
        gs.p = d_src; gs.b = src_bytes;
    }
    if (!dst_dev) {
        TW_TRY(dmalloc(ctx, &d_dst, dst_bytes));
        gd.p = d_dst; gd.b = dst_bytes;
    }
    // source chunks of ~64 MiB (whole planes)
    int64_t chunk = std::max<int64_t>(1, (int64_t)((64ull << 20) / std::max<size_t>(io.src_plane_bytes, 1)));
    chunk = std::min(chunk, io.src_planes);
    const int64_t nchunks = (io.src_planes + chunk - 1) / chunk;
    const int64_t nslabs = (io.dst_planes + io.slab - 1) / io.slab;
    Events ev_up, ev_comp, ev_down;
    TW_CUDA_TRY(ev_up.make(nchunks));
    TW_CUDA_TRY(ev_comp.make(nslabs));
    TW_CUDA_TRY(ev_down.make(nslabs));
    // pageable host memory goes through pinned staging rings
    const int kRing = 3;
    Pinned up_ring[kRing], down_ring[kRing];
    const size_t up_slot = io.src_plane_bytes * (size_t)chunk;
    const size_t down_slot = io.dst_plane_bytes * (size_t)io.slab;
    if (!src_dev && !src_pin)
        for (auto &r : up_ring) {
            TW_CUDA_TRY(cudaHostAlloc(&r.p, up_slot, cudaHostAllocDefault));
            r.bytes = up_slot;
        }
    if (!dst_dev && !dst_pin)
        for (auto &r : down_ring) {
            TW_CUDA_TRY(cudaHostAlloc(&r.p, down_slot, cudaHostAllocDefault));
            r.bytes = down_slot;
        }
    std::vector<int64_t> up_slot_owner(kRing, -1), down_slot_owner(kRing, -1);
    int64_t uploaded = 0;  // chunks issued
    std::deque<int64_t> pending_down;  // slabs whose D2H into a staging slot must be copied out

    auto drain_one = [&](void) -> tw_status {
        const int64_t s = pending_down.front();
        pending_down.pop_front();
        TW_CUDA_TRY(cudaEventSynchronize(ev_down.ev[s]));
        const int64_t z0 = s * io.slab, z1 = std::min(io.dst_planes, z0 + io.slab);
        std::memcpy(static_cast<char *>(io.dst) + (size_t)z0 * io.dst_plane_bytes, down_ring[s % kRing].p,
                    (size_t)(z1 - z0) * io.dst_plane_bytes);
        return TW_OK;
    };

    auto upload_until = [&](int64_t zhi) -> tw_status {
        const int64_t need_chunk = src_dev ? -1 : std::min(nchunks - 1, zhi / chunk);
        while (uploaded <= need_chunk) {
            const int64_t k = uploaded;
            const int64_t z0 = k * chunk, z1 = std::min(io.src_planes, z0 + chunk);
            const size_t bytes = (size_t)(z1 - z0) * io.src_plane_bytes;
            char *dptr = static_cast<char *>(d_src) + (size_t)z0 * io.src_plane_bytes;
            const char *hptr = static_cast<const char *>(io.src) + (size_t)z0 * io.src_plane_bytes;
            if (src_pin) {
                TW_CUDA_TRY(cudaMemcpyAsync(dptr, hptr, bytes, cudaMemcpyHostToDevice, ctx->h2d));
            } else {
                const int slot = (int)(k % kRing);
                if (up_slot_owner[slot] >= 0) TW_CUDA_TRY(cudaEventSynchronize(ev_up.ev[up_slot_owner[slot]]));
                std::memcpy(up_ring[slot].p, hptr, bytes);
                TW_CUDA_TRY(cudaMemcpyAsync(dptr, up_ring[slot].p, bytes, cudaMemcpyHostToDevice, ctx->h2d));
                up_slot_owner[slot] = k;
            }
            TW_CUDA_TRY(cudaEventRecord(ev_up.ev[k], ctx->h2d));
            ctx->h2d_bytes += bytes;
            ++uploaded;
        }
        if (need_chunk >= 0) TW_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ev_up.ev[need_chunk], 0));
        return TW_OK;
    };

    for (int64_t s = 0; s < nslabs; ++s) {
        const int64_t z0 = s * io.slab, z1 = std::min(io.dst_planes, z0 + io.slab);
        int64_t lo = 0, hi = io.src_planes - 1;
        need(z0, z1, lo, hi);
        hi = std::max<int64_t>(0, std::min(hi, io.src_planes - 1));
        TW_TRY(upload_until(hi));
        TW_TRY(compute(z0, z1, d_src, d_dst, ctx->stream));
        TW_CUDA_TRY(cudaEventRecord(ev_comp.ev[s], ctx->stream));
        if (!dst_dev) {
            TW_CUDA_TRY(cudaStreamWaitEvent(ctx->d2h, ev_comp.ev[s], 0));
            const size_t bytes = (size_t)(z1 - z0) * io.dst_plane_bytes;
            const char *dptr = static_cast<const char *>(d_dst) + (size_t)z0 * io.dst_plane_bytes;
            if (dst_pin) {
                TW_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(io.dst) + (size_t)z0 * io.dst_plane_bytes, dptr, bytes,
                                            cudaMemcpyDeviceToHost, ctx->d2h));
            } else {
                const int slot = (int)(s % kRing);
                while (!pending_down.empty() && pending_down.front() <= s - kRing) TW_TRY(drain_one());
                TW_CUDA_TRY(cudaMemcpyAsync(down_ring[slot].p, dptr, bytes, cudaMemcpyDeviceToHost, ctx->d2h));
                pending_down.push_back(s);
            }
            TW_CUDA_TRY(cudaEventRecord(ev_down.ev[s], ctx->d2h));
            ctx->d2h_bytes += (size_t)(z1 - z0) * io.dst_plane_bytes;
        }
    }
    while (!pending_down.empty()) TW_TRY(drain_one());
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->d2h));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->h2d));
    return check_kernel_errors(ctx);
}

}  // namespace tw
