// tw_eval.cu -- TPS evaluation at the coarse control-grid nodes (FP32,
// compensated landmark sums) on sm_100a.
//
// Reference: get_cd (weiyijisuan.cu:91-114) keeps a float xmxn_K1[20000]
// per thread (80 KB of local memory) and launches once per z plane; the CPU
// loops are q_imgwarp_tps_quicksmallmemory.cpp:620-648 and :1117-1146.
//
// Here one launch covers the whole grid.  Landmarks (centres and negated
// coefficients) are staged through shared memory in tiles and read as
// warp-wide broadcasts; each thread evaluates kNPT nodes so every shared
// load feeds kNPT node-landmark pairs.  Per pair: 3 FADD, 1 FMUL, 2 FFMA,
// 1 sqrt, 3 FFMA.  Sums are two-level: plain FP32 FMA chains over 32
// landmarks, then Kahan-compensated accumulation of those partials.
//
// Coordinates are taken relative to an origin o near the landmarks so the
// FP32 magnitudes stay small; the affine part is pre-folded on the host in
// FP64 into a0 + alin * p' with the identity already subtracted, so the
// kernel writes the displacement f(p) - p directly without cancelling two
// large numbers.

#include "tw_internal.h"

namespace tw {

namespace {

constexpr int kEvalThreads = 256;
constexpr int kNPT = 4;      // nodes per thread
constexpr int kTile = 256;   // landmarks staged per shared-memory tile
constexpr int kSub = 32;     // landmarks per plain FP32 partial sum

__device__ __forceinline__ float fast_sqrt(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float x)
{
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

__global__ void __launch_bounds__(kEvalThreads) k_tps_eval(EvalParams p)
{
    __shared__ float4 s_ctr[kTile];
    __shared__ float4 s_coef[kTile];
    const int64_t nnodes = p.gsz[0] * p.gsz[1] * p.gsz[2];
    const int64_t base = (int64_t)blockIdx.x * (kEvalThreads * kNPT) + threadIdx.x;

    float px[kNPT], py[kNPT], pz[kNPT];
    float sx[kNPT], sy[kNPT], sz[kNPT], cx[kNPT], cy[kNPT], cz[kNPT];
#pragma unroll
    for (int j = 0; j < kNPT; ++j) {
        int64_t L = base + (int64_t)j * kEvalThreads;
        if (L >= nnodes) L = nnodes - 1;  // duplicate work, store is skipped below
        int64_t i = L % p.gsz[0];
        int64_t t = L / p.gsz[0];
        int64_t jj = t % p.gsz[1];
        int64_t k = t / p.gsz[1];
        px[j] = (float)(p.node_o[0] + i * p.g);
        py[j] = (float)(p.node_o[1] + jj * p.g);
        pz[j] = (float)(p.node_o[2] + k * p.g);
        sx[j] = sy[j] = sz[j] = 0.f;
        cx[j] = cy[j] = cz[j] = 0.f;
    }

    for (int t0 = 0; t0 < p.n; t0 += kTile) {
        const int cnt = min(kTile, p.n - t0);
        __syncthreads();
        for (int l = threadIdx.x; l < kTile; l += kEvalThreads) {
            if (l < cnt) {
                s_ctr[l] = p.ctr[t0 + l];
                s_coef[l] = p.coef[t0 + l];
            } else {
                s_ctr[l] = make_float4(0.f, 0.f, 0.f, 0.f);
                s_coef[l] = make_float4(0.f, 0.f, 0.f, 0.f);  // zero weight pads the tile
            }
        }
        __syncthreads();
        const int nsub = (cnt + kSub - 1) / kSub;
        for (int sb = 0; sb < nsub; ++sb) {
            float ax[kNPT], ay[kNPT], az[kNPT];
#pragma unroll
            for (int j = 0; j < kNPT; ++j) ax[j] = ay[j] = az[j] = 0.f;
#pragma unroll 4
            for (int l = sb * kSub; l < sb * kSub + kSub; ++l) {
                const float4 c = s_ctr[l];
                const float4 w = s_coef[l];
#pragma unroll
                for (int j = 0; j < kNPT; ++j) {
                    float dx = px[j] - c.x, dy = py[j] - c.y, dz = pz[j] - c.z;
                    float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                    float r = fast_sqrt(r2);
                    ax[j] = fmaf(r, w.x, ax[j]);
                    ay[j] = fmaf(r, w.y, ay[j]);
                    az[j] = fmaf(r, w.z, az[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < kNPT; ++j) {
                kahan_add(sx[j], cx[j], ax[j]);
                kahan_add(sy[j], cy[j], ay[j]);
                kahan_add(sz[j], cz[j], az[j]);
            }
        }
    }

    // affine part: f_c(q) = d[0][c] + sum_r q_r d[r+1][c]; with q = o + p:
    // DF_c = (d[0][c] + o.d[1:4][c] - o_c) + sum_r p_r (d[r+1][c] - delta),
    // folded in FP64 without contraction, then rounded once to float
    float a0[3], alin[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double s = __ldg(&p.aff[c + 1]);
#pragma unroll
        for (int r = 0; r < 3; ++r) s = __dadd_rn(s, __dmul_rn(p.o[r], __ldg(&p.aff[(r + 1) * 4 + c + 1])));
        a0[c] = (float)__dsub_rn(s, p.o[c]);
#pragma unroll
        for (int r = 0; r < 3; ++r) alin[r][c] = (float)__dsub_rn(__ldg(&p.aff[(r + 1) * 4 + c + 1]), r == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int j = 0; j < kNPT; ++j) {
        const int64_t L = base + (int64_t)j * kEvalThreads;
        if (L >= nnodes) continue;
        float dfx = a0[0] + alin[0][0] * px[j] + alin[1][0] * py[j] + alin[2][0] * pz[j];
        float dfy = a0[1] + alin[0][1] * px[j] + alin[1][1] * py[j] + alin[2][1] * pz[j];
        float dfz = a0[2] + alin[0][2] * px[j] + alin[1][2] * py[j] + alin[2][2] * pz[j];
        // the running compensation holds minus the lost low-order part
        dfx += sx[j] - cx[j];
        dfy += sy[j] - cy[j];
        dfz += sz[j] - cz[j];
        p.out[L] = make_float4(dfx, dfy, dfz, 0.f);
    }
}

}  // namespace

cudaError_t launch_tps_eval(const EvalParams &p, cudaStream_t st, int sm_count)
{
    (void)sm_count;
    const int64_t nnodes = p.gsz[0] * p.gsz[1] * p.gsz[2];
    if (nnodes <= 0) return cudaSuccess;
    const int64_t per_block = (int64_t)kEvalThreads * kNPT;
    const int64_t grid = (nnodes + per_block - 1) / per_block;
    if (grid > 0x7fffffff) return cudaErrorInvalidValue;
    k_tps_eval<<<(unsigned)grid, kEvalThreads, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace tw
