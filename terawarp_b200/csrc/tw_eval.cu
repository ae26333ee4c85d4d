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
// 1 sqrt, 3 FFMA, issued as Blackwell FP32x2 instructions over two nodes at a
// time (the landmark is staged with each component duplicated, negated
// centre), so a pair costs ~5.5 issue slots.  Sums are two-level: plain FP32
// FMA chains over 32 landmarks, then Kahan-compensated accumulation of those
// partials.
//
// Coordinates are taken relative to an origin o near the landmarks so the
// FP32 magnitudes stay small; the affine part is folded (in FP64, on the
// device) into a0 + alin * p' with the identity already subtracted, so the
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
    // per landmark: (-cx, -cx, -cy, -cy), (-cz, -cz, wx, wx), (wy, wy, wz, wz)
    __shared__ float4 s_lm[kTile][3];
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

    float2 px2[kNPT / 2], py2[kNPT / 2], pz2[kNPT / 2];
#pragma unroll
    for (int k = 0; k < kNPT / 2; ++k) {
        px2[k] = make_float2(px[2 * k], px[2 * k + 1]);
        py2[k] = make_float2(py[2 * k], py[2 * k + 1]);
        pz2[k] = make_float2(pz[2 * k], pz[2 * k + 1]);
    }

    for (int t0 = 0; t0 < p.n; t0 += kTile) {
        const int cnt = min(kTile, p.n - t0);
        __syncthreads();
        for (int l = threadIdx.x; l < kTile; l += kEvalThreads) {
            float4 c = make_float4(0.f, 0.f, 0.f, 0.f), w = c;  // zero weight pads the tile
            if (l < cnt) {
                c = p.ctr[t0 + l];
                w = p.coef[t0 + l];
            }
            s_lm[l][0] = make_float4(-c.x, -c.x, -c.y, -c.y);
            s_lm[l][1] = make_float4(-c.z, -c.z, w.x, w.x);
            s_lm[l][2] = make_float4(w.y, w.y, w.z, w.z);
        }
        __syncthreads();
        const int nsub = (cnt + kSub - 1) / kSub;
        for (int sb = 0; sb < nsub; ++sb) {
            // node pairs (2k, 2k+1); the same operations, in the same order,
            // as one FP32 instruction per node and landmark
            float2 ax[kNPT / 2], ay[kNPT / 2], az[kNPT / 2];
#pragma unroll
            for (int k = 0; k < kNPT / 2; ++k) ax[k] = ay[k] = az[k] = make_float2(0.f, 0.f);
#pragma unroll 4
            for (int l = sb * kSub; l < sb * kSub + kSub; ++l) {
                const float4 A = s_lm[l][0], B = s_lm[l][1], Cw = s_lm[l][2];
                const float2 ncx = make_float2(A.x, A.y), ncy = make_float2(A.z, A.w);
                const float2 ncz = make_float2(B.x, B.y), wx = make_float2(B.z, B.w);
                const float2 wy = make_float2(Cw.x, Cw.y), wz = make_float2(Cw.z, Cw.w);
#pragma unroll
                for (int k = 0; k < kNPT / 2; ++k) {
                    const float2 dx = __fadd2_rn(px2[k], ncx), dy = __fadd2_rn(py2[k], ncy);
                    const float2 dz = __fadd2_rn(pz2[k], ncz);
                    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                    const float2 r = make_float2(fast_sqrt(r2.x), fast_sqrt(r2.y));
                    ax[k] = __ffma2_rn(r, wx, ax[k]);
                    ay[k] = __ffma2_rn(r, wy, ay[k]);
                    az[k] = __ffma2_rn(r, wz, az[k]);
                }
            }
#pragma unroll
            for (int j = 0; j < kNPT; ++j) {
                const float axj = (j & 1) ? ax[j >> 1].y : ax[j >> 1].x;
                const float ayj = (j & 1) ? ay[j >> 1].y : ay[j >> 1].x;
                const float azj = (j & 1) ? az[j >> 1].y : az[j >> 1].x;
                kahan_add(sx[j], cx[j], axj);
                kahan_add(sy[j], cy[j], ayj);
                kahan_add(sz[j], cz[j], azj);
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
