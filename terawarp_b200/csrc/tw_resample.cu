// tw_resample.cu -- fused cubic B-spline expansion + trilinear/NN resampling
// of uint8/uint16 volumes on sm_100a, for TPS (node-grid) and affine warps.
//
// Work unit: a "brick" of output voxels, 256 wide in x.  One CTA of 256
// threads (8 warps) owns a brick; warp w takes rows w, w+8, ..., and lane l
// the voxel pairs (2l + 64k, 2l + 64k + 1), so a warp's gathers for one tap
// touch 64 consecutive voxels and each pair is written with one 2-element
// store, coalesced across the warp.  A launch covers the
// bricks of one or more jobs that share (dtype, kind, g): the flattened brick
// index is mapped to its job by a binary search over the jobs' prefix sums,
// so uneven edge tiles and many small jobs run in one persistent launch.
//
// TPS bricks (reference: q_dfblcokinterp_bspline + q_imgblockwarp,
// q_imgwarp_tps_quicksmallmemory.cpp:85-203, and chazhi.cu:226-338, which
// does a dense 64x64x3 matvec per 4^3 cell): the cubic B-spline is evaluated
// separably.  Per brick the 4 x (CY+3) x (CX+3) nodes are staged in shared
// memory as node' = DF + node position - brick origin (the B-spline
// reproduces linear functions, so the spline of node' is the sample position
// q itself, relative to the brick origin).  They are contracted along y once
// per brick (R), along z once per output slice (Q), and along x per voxel
// (12 FMA), i.e. ~14 FMA per voxel instead of 192.
//
// Sampling follows the reference exactly: a sample with any q_i < 0 or
// q_i > sz_i - 1 writes 0; weights come from floor(q); TPS rounds with +0.5
// and truncates, affine truncates (q_warp_affine_tps.cpp:1433).  A brick whose
// whole sample hull (convex-hull property of the B-spline: weights are >= 0
// and sum to 1) lies strictly inside the source takes a fast path with no
// per-voxel bounds tests.

#include "tw_internal.h"

#include <cstdint>

namespace tw {

namespace {

constexpr int kThreads = 256;
constexpr int kTX = 32;
constexpr int kTY = 8;
constexpr int kV = 8;                 // voxels per lane per brick row (4 pairs)
constexpr int kBX = kTX * kV;         // 256 voxels per brick along x
constexpr float kMagic = 12582912.0f; // 1.5 * 2^23: add.rm(q, kMagic) = kMagic + floor(q)
constexpr int kMagicBits = 0x4B400000;

template <int G>
struct Geom {
    static constexpr int BX = kBX;
    static constexpr int BY = G < 8 ? 8 : G;

    static constexpr int CX = BX / G;
    static constexpr int CY = BY / G;
    static constexpr int NX = CX + 3;
    static constexpr int NY = CY + 3;

    static constexpr int ROWS = BY / kTY;
    static constexpr int ND = 4 * NY * NX;       // staged nodes
    static constexpr int NR = BY * 4 * NX;       // y-contracted
    static constexpr int NQ = 2 * BY * NX;       // z-contracted, double-buffered
    static constexpr int UNION = ND > NQ ? ND : NQ;
    static constexpr size_t smem_bytes = sizeof(float4) * (size_t)(UNION + NR + G) + 64;
};

// Uniform cubic B-spline blending weights at t = i/g (rows of T*B/6,
// q_imgwarp_tps_quicksmallmemory.cpp:671-689), evaluated in double and
// rounded once to float.
__device__ __forceinline__ float4 bspline_w(int i, int g)
{
    double t = (double)i / (double)g;
    double t2 = t * t, t3 = t2 * t;
    double w0 = (-t3 + 3.0 * t2 - 3.0 * t + 1.0) / 6.0;
    double w1 = (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0;
    double w2 = (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
    double w3 = t3 / 6.0;
    return make_float4((float)w0, (float)w1, (float)w2, (float)w3);
}

// Loads one voxel and converts it to float without the conversion pipe:
// 2^23 + v has v in its low mantissa bits, so OR-ing the integer into the
// exponent pattern of 2^23 and subtracting 2^23 is exact (v < 2^23).
template <typename T>
__device__ __forceinline__ float ldv(const T *p)
{
    const uint32_t v = (uint32_t)__ldg(p);
    return __int_as_float(0x4B000000 | (int)v) - 8388608.0f;
}

__device__ __forceinline__ float floor_magic(float q, int &i)
{
    float m = __fadd_rd(q, kMagic);
    i = __float_as_int(m) - kMagicBits;
    return m - kMagic;
}

// Output conversion: TPS rounds (+0.5) then truncates; affine truncates.
template <typename T, bool ROUND>
__device__ __forceinline__ uint32_t to_out(float v)
{
    float r = ROUND ? v + 0.5f : v;
    r = fmaxf(r, 0.0f);
    uint32_t u = (uint32_t)(__float_as_int(__fadd_rd(r, 8388608.0f)) - 0x4B000000);
    const uint32_t mx = sizeof(T) == 1 ? 255u : 65535u;
    return u > mx ? mx : u;
}

// Trilinear sample at brick-relative position (qx,qy,qz) from `base`
// (the source element at the brick origin), no bounds tests.
template <typename T>
__device__ __forceinline__ float tri_fast(const T *__restrict__ base, int py, int pz, float qx, float qy,
                                          float qz)
{
    int ix, iy, iz;
    float fx = qx - floor_magic(qx, ix);
    float fy = qy - floor_magic(qy, iy);
    float fz = qz - floor_magic(qz, iz);
    const T *p = base + (iz * pz + iy * py + ix);
    float v000 = ldv(p), v100 = ldv(p + 1);
    float v010 = ldv(p + py), v110 = ldv(p + py + 1);
    float v001 = ldv(p + pz), v101 = ldv(p + pz + 1);
    float v011 = ldv(p + pz + py), v111 = ldv(p + pz + py + 1);
    float a0 = fmaf(fx, v100 - v000, v000);
    float a1 = fmaf(fx, v110 - v010, v010);
    float a2 = fmaf(fx, v101 - v001, v001);
    float a3 = fmaf(fx, v111 - v011, v011);
    float b0 = fmaf(fy, a1 - a0, a0);
    float b1 = fmaf(fy, a3 - a2, a2);
    return fmaf(fz, b1 - b0, b0);
}

// Bounds of a brick's frame for the checked sampler: with positions q taken
// relative to the brick origin O, the reference's rule 0 <= O+q <= glob-1
// becomes lo <= q <= hi (exact in float: integers below 2^24), and every
// index is clamped to the source buffer's extent [bl, bh] in the same frame.
struct Frame {
    float lo[3], hi[3];
    int bl[3], bh[3];
};

__device__ __forceinline__ Frame make_frame(const RJob &J, const int64_t O[3])
{
    Frame f;
    // |q| stays below 2^22 so that the magic-number floor is exact
    const float lim = 4194304.0f;
    for (int a = 0; a < 3; ++a) {
        f.lo[a] = fmaxf((float)(-O[a]), -lim);
        f.hi[a] = fminf((float)(J.glob[a] - 1 - O[a]), lim);
        int64_t bl = J.src_o[a] - O[a], bh = J.src_o[a] + J.src_n[a] - 1 - O[a];
        f.bl[a] = (int)max((int64_t)-0x3fffffff, bl);
        f.bh[a] = (int)min((int64_t)0x3fffffff, bh);
    }
    return f;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Checked sample at brick-relative q: returns false when the reference would
// write 0 (any axis outside [0, sz-1], or a NaN position).  `base` points at
// the source element of the brick origin (it may lie outside the buffer; the
// clamped indices never do).  x_b = ceil(q) equals floor(q)+1 except when q
// is integral, where its weight is 0, so clamping it changes no value.
template <typename T, int INTERP>
__device__ __forceinline__ bool sample_checked(const T *__restrict__ base, int64_t py, int64_t pz, const Frame &f,
                                               float qx, float qy, float qz, float &out)
{
    if (!(qx >= f.lo[0] && qx <= f.hi[0] && qy >= f.lo[1] && qy <= f.hi[1] && qz >= f.lo[2] && qz <= f.hi[2]))
        return false;
    if (INTERP == 1) {
        // (long)(q + 0.5) clamped to sz - 1 (q_imgwarp_tps_quicksmallmemory.cpp:119-129)
        int ix, iy, iz;
        floor_magic(qx + 0.5f, ix);
        floor_magic(qy + 0.5f, iy);
        floor_magic(qz + 0.5f, iz);
        ix = clampi(min(ix, (int)f.hi[0]), f.bl[0], f.bh[0]);
        iy = clampi(min(iy, (int)f.hi[1]), f.bl[1], f.bh[1]);
        iz = clampi(min(iz, (int)f.hi[2]), f.bl[2], f.bh[2]);
        out = ldv(base + ((int64_t)iz * pz + (int64_t)iy * py + ix));
        return true;
    }
    int ix, iy, iz;
    const float fx = qx - floor_magic(qx, ix);
    const float fy = qy - floor_magic(qy, iy);
    const float fz = qz - floor_magic(qz, iz);
    const int x0 = clampi(ix, f.bl[0], f.bh[0]), x1 = clampi(ix + 1, f.bl[0], f.bh[0]);
    const int y0 = clampi(iy, f.bl[1], f.bh[1]), y1 = clampi(iy + 1, f.bl[1], f.bh[1]);
    const int z0 = clampi(iz, f.bl[2], f.bh[2]), z1 = clampi(iz + 1, f.bl[2], f.bh[2]);
    const T *r00 = base + ((int64_t)z0 * pz + (int64_t)y0 * py);
    const T *r10 = base + ((int64_t)z0 * pz + (int64_t)y1 * py);
    const T *r01 = base + ((int64_t)z1 * pz + (int64_t)y0 * py);
    const T *r11 = base + ((int64_t)z1 * pz + (int64_t)y1 * py);
    float v000 = ldv(r00 + x0), v100 = ldv(r00 + x1);
    float v010 = ldv(r10 + x0), v110 = ldv(r10 + x1);
    float v001 = ldv(r01 + x0), v101 = ldv(r01 + x1);
    float v011 = ldv(r11 + x0), v111 = ldv(r11 + x1);
    float a0 = fmaf(fx, v100 - v000, v000);
    float a1 = fmaf(fx, v110 - v010, v010);
    float a2 = fmaf(fx, v101 - v001, v001);
    float a3 = fmaf(fx, v111 - v011, v011);
    float b0 = fmaf(fy, a1 - a0, a0);
    float b1 = fmaf(fy, a3 - a2, a2);
    out = fmaf(fz, b1 - b0, b0);
    return true;
}

template <typename T, int INTERP>
__device__ __forceinline__ float sample_fast(const T *__restrict__ base, int py, int pz, float qx, float qy,
                                             float qz)
{
    if (INTERP == 1) {
        int ix, iy, iz;
        floor_magic(qx + 0.5f, ix);
        floor_magic(qy + 0.5f, iy);
        floor_magic(qz + 0.5f, iz);
        return ldv(base + (iz * pz + iy * py + ix));
    }
    return tri_fast<T>(base, py, pz, qx, qy, qz);
}

__device__ __forceinline__ int find_job(const RJob *jobs, int njobs, int64_t b)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].brick_begin <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Block-wide min/max reduction of 3 components (6 floats), result broadcast.
__device__ __forceinline__ void block_minmax(float (&mn)[3], float (&mx)[3], float *red)
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            red[warp * 6 + a] = mn[a];
            red[warp * 6 + 3 + a] = mx[a];
        }
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float m0 = red[a], m1 = red[3 + a];
        for (int w = 1; w < kThreads / 32; ++w) {
            m0 = fminf(m0, red[w * 6 + a]);
            m1 = fmaxf(m1, red[w * 6 + 3 + a]);
        }
        mn[a] = m0;
        mx[a] = m1;
    }
}

// Is every brick-relative sample position in [lo, hi] strictly inside both
// the subject volume and the source buffer, and are all byte offsets
// representable in 32 bits?
__device__ __forceinline__ bool hull_inside(const RJob &J, const int64_t O[3], const float (&lo)[3],
                                            const float (&hi)[3])
{
    const float margin = 1.0f / 64.0f;
    int64_t span = 0;
    const int64_t pitch[3] = {1, J.src_py, J.src_pz};
    for (int a = 0; a < 3; ++a) {
        // subject volume: 0 <= O + q and O + q < glob - 1 (so floor+1 is in range)
        double glo = (double)O[a] + (double)lo[a] - margin;
        double ghi = (double)O[a] + (double)hi[a] + margin;
        if (!(glo >= 0.0) || !(ghi < (double)(J.glob[a] - 1))) return false;
        // source buffer covers [src_o, src_o + src_n - 1]
        if (!(glo >= (double)J.src_o[a]) || !(ghi < (double)(J.src_o[a] + J.src_n[a] - 1))) return false;
        double ext = fmax(fabs((double)lo[a]), fabs((double)hi[a])) + 2.0;
        span += (int64_t)ext * pitch[a];
    }
    return span < (int64_t)0x7fffffff / 2;
}

// Do all offsets between the brick origin and any tap within the hull fit
// in 32 bits (so the unchecked path can use int offsets)?
__device__ __forceinline__ bool offsets_fit_32(const RJob &J, const float (&lo)[3], const float (&hi)[3])
{
    const double pitch[3] = {1.0, (double)J.src_py, (double)J.src_pz};
    double span = 0.0;
    for (int a = 0; a < 3; ++a) {
        const double ext = fmax(fabs((double)lo[a]), fabs((double)hi[a])) + 2.0;
        if (!(ext < 1e9)) return false;
        span += ext * pitch[a];
    }
    return span < 1.0e9;
}

// ------------------------------------------------------------------ TPS

// Writes a lane's pair of voxels (x, x+1): one 2-element store when the
// address is aligned for it, else element by element within the row.
template <typename T>
__device__ __forceinline__ void store_pair(T *p, uint32_t v0, uint32_t v1, bool pair_ok, int nvalid)
{
    if (pair_ok && nvalid >= 2) {
        if (sizeof(T) == 2) *reinterpret_cast<uint32_t *>(p) = v0 | (v1 << 16);
        else *reinterpret_cast<uint16_t *>(p) = (uint16_t)(v0 | (v1 << 8));
    } else {
        if (nvalid >= 1) p[0] = (T)v0;
        if (nvalid >= 2) p[1] = (T)v1;
    }
}

// One output slice of a brick.  Lane l of warp w owns voxel pairs
// (x, x+1), x = 2l + 64k (k = 0..3), of rows y = w + 8r: a warp's gathers
// then cover 64 consecutive voxels (about one 128-byte line per tap) instead
// of 256.  The pair shares one cell (G >= 2), its 4 node taps come from Q
// (z/y-contracted nodes), and the x expansion is 12 FMA per voxel.
template <typename T, int G, int INTERP>
__device__ __forceinline__ void tps_pair(const float4 *Q, const float4 (&wx)[2], int y, int x, bool fast, int xe,
                                         const T *base, int py32, int pz32, int64_t py, int64_t pz,
                                         const Frame &frame, T *drow, bool pair_ok)
{
    using Gm = Geom<G>;
    const float4 *qn = Q + y * Gm::NX + x / G;
    const float4 n0 = qn[0], n1 = qn[1], n2 = qn[2], n3 = qn[3];
    uint32_t outv[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const float4 w = wx[j];
        const float qx = fmaf(w.x, n0.x, fmaf(w.y, n1.x, fmaf(w.z, n2.x, w.w * n3.x)));
        const float qy = fmaf(w.x, n0.y, fmaf(w.y, n1.y, fmaf(w.z, n2.y, w.w * n3.y)));
        const float qz = fmaf(w.x, n0.z, fmaf(w.y, n1.z, fmaf(w.z, n2.z, w.w * n3.z)));
        float v;
        if (fast) {
            v = sample_fast<T, INTERP>(base, py32, pz32, qx, qy, qz);
            outv[j] = INTERP == 1 ? (uint32_t)v : to_out<T, true>(v);
        } else {
            const bool ok = (x + j) < xe && sample_checked<T, INTERP>(base, py, pz, frame, qx, qy, qz, v);
            outv[j] = ok ? (INTERP == 1 ? (uint32_t)v : to_out<T, true>(v)) : 0u;
        }
    }
    store_pair<T>(drow + x, outv[0], outv[1], pair_ok, fast ? 2 : xe - x);
}

// ALL_FAST: the whole brick is inside; else segf[y*4 + k] says whether the
// warp-row segment (row y, voxels 64k..64k+63) may skip the bounds checks.
template <typename T, int G, int INTERP, bool ALL_FAST>
__device__ __forceinline__ void tps_rows(const float4 *Q, const float4 (&wx)[2], int lane, int ty, int ye, int xe,
                                         const T *base, int py32, int pz32, int64_t py, int64_t pz,
                                         const Frame &frame, T *dslice, int64_t dpy, bool pair_ok,
                                         const unsigned char *segf)
{
    using Gm = Geom<G>;
#pragma unroll 1
    for (int r = 0; r < Gm::ROWS; ++r) {
        const int y = ty + kTY * r;
        if (y >= ye) continue;
        T *drow = dslice + (int64_t)y * dpy;
#pragma unroll
        for (int k = 0; k < Gm::BX / 64; ++k) {
            const int x = 2 * lane + 64 * k;
            if (ALL_FAST) {
                tps_pair<T, G, INTERP>(Q, wx, y, x, true, xe, base, py32, pz32, py, pz, frame, drow, pair_ok);
            } else if (segf[y * 4 + k]) {  // warp-uniform
                tps_pair<T, G, INTERP>(Q, wx, y, x, true, xe, base, py32, pz32, py, pz, frame, drow, pair_ok);
            } else if (x < xe) {
                tps_pair<T, G, INTERP>(Q, wx, y, x, false, xe, base, py32, pz32, py, pz, frame, drow, pair_ok);
            }
        }
    }
}

template <typename T, int G, int INTERP>
__device__ void tps_brick(const RJob &J, int64_t bx, int64_t by, int64_t bz, float4 *sm, float *red,
                          unsigned char *segf)
{
    using Gm = Geom<G>;
    float4 *Nd = sm;                       // [4][NY][NX]   (aliases Q)
    float4 *Qb = sm;                       // [2][BY][NX]
    float4 *R = sm + Gm::UNION;            // [BY][4][NX]
    const float4 *W = sm + Gm::UNION + Gm::NR;  // [G] weights
    const int tid = threadIdx.x;
    const int tx = tid & 31, ty = tid >> 5;

    // a brick spans zs output planes of one cell layer (zs divides G; small
    // jobs split the layer over several CTAs to fill the machine)
    // The frame origin O is the brick's corner with z at the start of its cell
    // layer, so sample positions (and their FP32 rounding) do not depend on
    // how a launch splits layers: a job gives the same voxels alone or batched.
    const int zs = J.zs;
    const int64_t zfirst = J.out_o[2] + bz * zs;          // first output plane of this brick
    const int64_t O[3] = {J.out_o[0] + bx * Gm::BX, J.out_o[1] + by * Gm::BY, (zfirst / G) * G};
    const int64_t c0[3] = {O[0] / G, O[1] / G, O[2] / G};  // first cell (= first node index)
    const int zoff = (int)(zfirst - O[2]);                 // first plane within the cell layer

    // 1. stage node' = DF + node position - O, and its hull (a non-finite
    // node forces the checked path)
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = tid; i < Gm::ND; i += kThreads) {
        int nx = i % Gm::NX, t = i / Gm::NX;
        int ny = t % Gm::NY, nz = t / Gm::NY;
        int64_t gx = c0[0] + nx, gy = c0[1] + ny, gz = c0[2] + nz;
        gx = gx < J.gsz[0] ? gx : J.gsz[0] - 1;
        gy = gy < J.gsz[1] ? gy : J.gsz[1] - 1;
        gz = gz < J.gsz[2] ? gz : J.gsz[2] - 1;
        float4 d = J.nodes[(gz * J.gsz[1] + gy) * J.gsz[0] + gx];
        // node gx sits at (gx-1)*G; relative to O that is (gx-1)*G - O (exact in float)
        float4 v;
        v.x = d.x + (float)((gx - 1) * G - O[0]);
        v.y = d.y + (float)((gy - 1) * G - O[1]);
        v.z = d.z + (float)((gz - 1) * G - O[2]);
        v.w = 0.f;
        Nd[i] = v;
        if (isfinite(v.x) && isfinite(v.y) && isfinite(v.z)) {
            mn[0] = fminf(mn[0], v.x); mn[1] = fminf(mn[1], v.y); mn[2] = fminf(mn[2], v.z);
            mx[0] = fmaxf(mx[0], v.x); mx[1] = fmaxf(mx[1], v.y); mx[2] = fmaxf(mx[2], v.z);
        } else {
            mn[0] = mn[1] = mn[2] = -3.4e38f;
            mx[0] = mx[1] = mx[2] = 3.4e38f;
        }
    }
    block_minmax(mn, mx, red);  // contains __syncthreads (Nd visible after it)

    const bool inside_out = (O[0] + Gm::BX <= J.out_o[0] + J.out_n[0]) &&
                            (O[1] + Gm::BY <= J.out_o[1] + J.out_n[1]) &&
                            (zfirst + zs <= J.out_o[2] + J.out_n[2]);
    const bool fast = inside_out && hull_inside(J, O, mn, mx);
    const Frame frame = make_frame(J, O);
    const bool span_ok = offsets_fit_32(J, mn, mx);

    // 2. R[y][c][nx] = sum_b wy_b(y) Nd[c][y/G + b][nx]
    for (int i = tid; i < Gm::NR; i += kThreads) {
        int nx = i % Gm::NX, t = i / Gm::NX;
        int c = t & 3, y = t >> 2;
        float4 w = W[y % G];
        int cy = y / G;
        const float4 *n0 = Nd + (c * Gm::NY + cy) * Gm::NX + nx;
        float4 a = n0[0], b = n0[Gm::NX], e = n0[2 * Gm::NX], f = n0[3 * Gm::NX];
        float4 r;
        r.x = fmaf(w.x, a.x, fmaf(w.y, b.x, fmaf(w.z, e.x, w.w * f.x)));
        r.y = fmaf(w.x, a.y, fmaf(w.y, b.y, fmaf(w.z, e.y, w.w * f.y)));
        r.z = fmaf(w.x, a.z, fmaf(w.y, b.z, fmaf(w.z, e.z, w.w * f.z)));
        r.w = 0.f;
        R[i] = r;
    }
    __syncthreads();

    // per row segment (row y, 64 voxels 64k..64k+63): does the hull of the
    // y-contracted nodes it uses (all four z layers, weights >= 0) keep every
    // tap inside the volume and the buffer?  Then that warp-row segment takes
    // the unchecked path even in a border brick.
    const int64_t xe = J.out_o[0] + J.out_n[0] - O[0];  // valid x extent in this brick
    if (!fast && tid < Gm::BY * 4) {
        const int y = tid >> 2, k = tid & 3;
        const int t0 = (64 * k) / G, t1 = (64 * k + 63) / G + 3;
        float lo3[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi3[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
        bool finite = true;
        for (int c = 0; c < 4; ++c)
            for (int nx = t0; nx <= t1; ++nx) {
                const float4 r = R[(y * 4 + c) * Gm::NX + nx];
                finite = finite && isfinite(r.x) && isfinite(r.y) && isfinite(r.z);
                lo3[0] = fminf(lo3[0], r.x); lo3[1] = fminf(lo3[1], r.y); lo3[2] = fminf(lo3[2], r.z);
                hi3[0] = fmaxf(hi3[0], r.x); hi3[1] = fmaxf(hi3[1], r.y); hi3[2] = fmaxf(hi3[2], r.z);
            }
        bool ok = finite && span_ok && (64 * k + 64 <= xe);
        for (int a = 0; a < 3; ++a) {
            const float lb = fmaxf(frame.lo[a], (float)frame.bl[a]) + 1.0f / 64.0f;
            const float hb = fminf(frame.hi[a], (float)frame.bh[a]) - 1.0f / 64.0f;
            ok = ok && lo3[a] >= lb && hi3[a] < hb;
        }
        segf[tid] = ok ? 1 : 0;
    }
    __syncthreads();

    // x weights of the lane's voxel pair (2l, 2l+1) + 64k: the brick origin is
    // a multiple of G and G divides 64, so they do not depend on k
    float4 wx[2];
    wx[0] = W[(2 * tx) % G];
    wx[1] = W[(2 * tx + 1) % G];

    const T *src = static_cast<const T *>(J.src);
    T *dst = static_cast<T *>(J.dst);
    const int64_t sbase = (O[2] - J.src_o[2]) * J.src_pz + (O[1] - J.src_o[1]) * J.src_py + (O[0] - J.src_o[0]);
    const T *base = src + sbase;
    const int py32 = (int)J.src_py, pz32 = (int)J.src_pz;
    // output plane z of the loop below is zfirst + z
    const int64_t dbase0 = (zfirst - J.out_o[2]) * J.dst_pz + (O[1] - J.out_o[1]) * J.dst_py + (O[0] - J.out_o[0]);
    // a voxel pair (even x) can be written as one 2-element store
    const bool pair_ok = ((((uintptr_t)(dst + dbase0)) % (2 * sizeof(T))) == 0) && (J.dst_py % 2 == 0) &&
                         (J.dst_pz % 2 == 0);
    const int64_t ye = J.out_o[1] + J.out_n[1] - O[1];
    const int64_t ze = J.out_o[2] + J.out_n[2] - zfirst;

    for (int z = 0; z < zs; ++z) {
        float4 *Q = Qb + (z & 1) * (Gm::BY * Gm::NX);
        const float4 wz = W[zoff + z];
        for (int i = tid; i < Gm::BY * Gm::NX; i += kThreads) {
            int nx = i % Gm::NX, y = i / Gm::NX;
            const float4 *r = R + (y * 4) * Gm::NX + nx;
            float4 a = r[0], b = r[Gm::NX], e = r[2 * Gm::NX], f = r[3 * Gm::NX];
            float4 q;
            q.x = fmaf(wz.x, a.x, fmaf(wz.y, b.x, fmaf(wz.z, e.x, wz.w * f.x)));
            q.y = fmaf(wz.x, a.y, fmaf(wz.y, b.y, fmaf(wz.z, e.y, wz.w * f.y)));
            q.z = fmaf(wz.x, a.z, fmaf(wz.y, b.z, fmaf(wz.z, e.z, wz.w * f.z)));
            q.w = 0.f;
            Q[i] = q;
        }
        __syncthreads();
        if (z >= ze) continue;  // uniform: whole slice outside the region
        // fast bricks skip the per-segment flags; otherwise each warp-row
        // segment picks its path (uniform across the warp)
        if (fast) {
            tps_rows<T, G, INTERP, true>(Q, wx, tx, ty, (int)ye, (int)xe, base, py32, pz32, J.src_py, J.src_pz, frame,
                                          dst + dbase0 + (int64_t)z * J.dst_pz, J.dst_py, pair_ok, segf);
        } else {
            tps_rows<T, G, INTERP, false>(Q, wx, tx, ty, (int)ye, (int)xe, base, py32, pz32, J.src_py, J.src_pz,
                                           frame, dst + dbase0 + (int64_t)z * J.dst_pz, J.dst_py, pair_ok, segf);
        }
    }
    __syncthreads();  // smem reuse by the next brick
}

// ---------------------------------------------------------------- affine

constexpr int kABY = 8, kABZ = 8;

// Rows of an affine brick with the same lane-pair layout as the TPS path:
// lane l owns voxels (x, x+1), x = 2l + 64k; q = fo + M_lin l in FP32.
template <typename T, int INTERP, bool FAST>
__device__ __forceinline__ void affine_rows(const float (&m)[3][3], const float (&fo)[3], int lane, int ty, int ye,
                                            int ze, int xe, const T *base, int py32, int pz32, int64_t py, int64_t pz,
                                            const Frame &frame, T *dbrick, int64_t dpy, int64_t dpz, bool pair_ok)
{
#pragma unroll 1
    for (int z = 0; z < kABZ; ++z) {
        if (z >= ze) break;
        const int y = ty;
        if (y >= ye) continue;
        const float bx0 = fo[0] + m[0][1] * (float)y + m[0][2] * (float)z;
        const float by0 = fo[1] + m[1][1] * (float)y + m[1][2] * (float)z;
        const float bz0 = fo[2] + m[2][1] * (float)y + m[2][2] * (float)z;
        T *drow = dbrick + (int64_t)z * dpz + (int64_t)y * dpy;
#pragma unroll
        for (int k = 0; k < kBX / 64; ++k) {
            const int x = 2 * lane + 64 * k;
            if (!FAST && x >= xe) continue;
            uint32_t outv[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const float lx = (float)(x + j);
                const float qx = fmaf(m[0][0], lx, bx0), qy = fmaf(m[1][0], lx, by0), qz = fmaf(m[2][0], lx, bz0);
                float v;
                if (FAST) {
                    v = sample_fast<T, INTERP>(base, py32, pz32, qx, qy, qz);
                    outv[j] = INTERP == 1 ? (uint32_t)v : to_out<T, false>(v);
                } else {
                    const bool ok = (x + j) < xe && sample_checked<T, INTERP>(base, py, pz, frame, qx, qy, qz, v);
                    outv[j] = ok ? (INTERP == 1 ? (uint32_t)v : to_out<T, false>(v)) : 0u;
                }
            }
            store_pair<T>(drow + x, outv[0], outv[1], pair_ok, FAST ? 2 : xe - x);
        }
    }
}

template <typename T, int INTERP>
__device__ void affine_brick(const RJob &J, int64_t bx, int64_t by, int64_t bz, float *red)
{
    const int tid = threadIdx.x;
    const int tx = tid & 31, ty = tid >> 5;
    const int64_t O[3] = {J.out_o[0] + bx * kBX, J.out_o[1] + by * kABY, J.out_o[2] + bz * kABZ};
    // q(O + l) = M (O + l) = qO + Mlin l  (FP64 at the origin, FP32 increments)
    double qO[3];
    for (int r = 0; r < 3; ++r)
        qO[r] = J.M[r * 4 + 0] * (double)O[0] + J.M[r * 4 + 1] * (double)O[1] + J.M[r * 4 + 2] * (double)O[2] +
                J.M[r * 4 + 3];
    // hull over the brick corners, relative to floor(qO)
    int64_t qf[3];
    float fo[3];
    float lo[3], hi[3];
    for (int r = 0; r < 3; ++r) {
        if (!(fabs(qO[r]) < 1e15)) {  // non-finite or absurd matrix: every sample is out of range
            qf[r] = 0;
            fo[r] = __int_as_float(0x7fc00000);
            lo[r] = hi[r] = fo[r];
            continue;
        }
        double f = floor(qO[r]);
        qf[r] = (int64_t)f;
        fo[r] = (float)(qO[r] - f);
        double l = 0, h = 0;
        const double ext[3] = {kBX - 1.0, kABY - 1.0, kABZ - 1.0};
        for (int a = 0; a < 3; ++a) {
            double v = J.M[r * 4 + a] * ext[a];
            if (v < 0) l += v; else h += v;
        }
        lo[r] = (float)(fo[r] + l);
        hi[r] = (float)(fo[r] + h);
    }
    (void)red;
    const bool inside_out = (O[0] + kBX <= J.out_o[0] + J.out_n[0]) && (O[1] + kABY <= J.out_o[1] + J.out_n[1]) &&
                            (O[2] + kABZ <= J.out_o[2] + J.out_n[2]);
    const bool fast = inside_out && hull_inside(J, qf, lo, hi);
    const float m[3][3] = {{(float)J.M[0], (float)J.M[1], (float)J.M[2]},
                           {(float)J.M[4], (float)J.M[5], (float)J.M[6]},
                           {(float)J.M[8], (float)J.M[9], (float)J.M[10]}};
    const T *src = static_cast<const T *>(J.src);
    T *dst = static_cast<T *>(J.dst);
    const int64_t sbase = (qf[2] - J.src_o[2]) * J.src_pz + (qf[1] - J.src_o[1]) * J.src_py + (qf[0] - J.src_o[0]);
    const T *base = src + sbase;
    const Frame frame = make_frame(J, qf);
    const int py32 = (int)J.src_py, pz32 = (int)J.src_pz;
    const int64_t dbase0 = (O[2] - J.out_o[2]) * J.dst_pz + (O[1] - J.out_o[1]) * J.dst_py + (O[0] - J.out_o[0]);
    const bool pair_ok = ((((uintptr_t)(dst + dbase0)) % (2 * sizeof(T))) == 0) && (J.dst_py % 2 == 0) &&
                         (J.dst_pz % 2 == 0);
    const int64_t xe = J.out_o[0] + J.out_n[0] - O[0];
    const int64_t ye = J.out_o[1] + J.out_n[1] - O[1];
    const int64_t ze = J.out_o[2] + J.out_n[2] - O[2];
    if (fast)
        affine_rows<T, INTERP, true>(m, fo, tx, ty, (int)ye, (int)ze, (int)xe, base, py32, pz32, J.src_py, J.src_pz,
                                     frame, dst + dbase0, J.dst_py, J.dst_pz, pair_ok);
    else
        affine_rows<T, INTERP, false>(m, fo, tx, ty, (int)ye, (int)ze, (int)xe, base, py32, pz32, J.src_py, J.src_pz,
                                      frame, dst + dbase0, J.dst_py, J.dst_pz, pair_ok);
}

// ---------------------------------------------------------------- kernels

template <typename T, int G, int INTERP>
__global__ void __launch_bounds__(kThreads, 3) k_resample_tps(const RJob *__restrict__ jobs, int njobs,
                                                            int64_t total_bricks)
{
    extern __shared__ float4 smem[];
    __shared__ float red[6 * (kThreads / 32)];
    __shared__ unsigned char segf[256];
    using Gm = Geom<G>;
    float4 *W = smem + Gm::UNION + Gm::NR;
    if (threadIdx.x < G) W[threadIdx.x] = bspline_w(threadIdx.x, G);
    __syncthreads();
    for (int64_t b = blockIdx.x; b < total_bricks; b += gridDim.x) {
        const int j = find_job(jobs, njobs, b);
        const RJob &J = jobs[j];
        int64_t lb = b - J.brick_begin;
        int64_t bx = lb % J.bricks[0];
        int64_t t = lb / J.bricks[0];
        int64_t by = t % J.bricks[1];
        int64_t bz = t / J.bricks[1];
        tps_brick<T, G, INTERP>(J, bx, by, bz, smem, red, segf);
    }
}

template <typename T, int INTERP>
__global__ void __launch_bounds__(kThreads) k_resample_affine(const RJob *__restrict__ jobs, int njobs,
                                                               int64_t total_bricks)
{
    __shared__ float red[6 * (kThreads / 32)];
    for (int64_t b = blockIdx.x; b < total_bricks; b += gridDim.x) {
        const int j = find_job(jobs, njobs, b);
        const RJob &J = jobs[j];
        int64_t lb = b - J.brick_begin;
        int64_t bx = lb % J.bricks[0];
        int64_t t = lb / J.bricks[0];
        int64_t by = t % J.bricks[1];
        int64_t bz = t / J.bricks[1];
        affine_brick<T, INTERP>(J, bx, by, bz, red);
    }
}

template <typename T, int G, int INTERP>
cudaError_t launch_tps_t(const RJob *jobs, int njobs, int64_t total, cudaStream_t st, int sms)
{
    using Gm = Geom<G>;
    auto k = k_resample_tps<T, G, INTERP>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Gm::smem_bytes);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, Gm::smem_bytes);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > total) grid = total;
    if (grid < 1) grid = 1;
    k<<<(unsigned)grid, kThreads, Gm::smem_bytes, st>>>(jobs, njobs, total);
    return cudaGetLastError();
}

template <typename T, int INTERP>
cudaError_t launch_affine_t(const RJob *jobs, int njobs, int64_t total, cudaStream_t st, int sms)
{
    auto k = k_resample_affine<T, INTERP>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > total) grid = total;
    if (grid < 1) grid = 1;
    k<<<(unsigned)grid, kThreads, 0, st>>>(jobs, njobs, total);
    return cudaGetLastError();
}

template <typename T, int INTERP>
cudaError_t dispatch_g(const RJob *jobs, int njobs, int64_t total, int g, cudaStream_t st, int sms)
{
    switch (g) {
    case 4: return launch_tps_t<T, 4, INTERP>(jobs, njobs, total, st, sms);
    case 8: return launch_tps_t<T, 8, INTERP>(jobs, njobs, total, st, sms);
    case 16: return launch_tps_t<T, 16, INTERP>(jobs, njobs, total, st, sms);
    case 32: return launch_tps_t<T, 32, INTERP>(jobs, njobs, total, st, sms);
    case 64: return launch_tps_t<T, 64, INTERP>(jobs, njobs, total, st, sms);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

bool g_supported(int g) { return g == 4 || g == 8 || g == 16 || g == 32 || g == 64; }

void brick_dims(int kind, int g, int64_t out[3])
{
    if (kind == 0) {
        out[0] = kBX; out[1] = kABY; out[2] = kABZ;
        return;
    }
    out[0] = kBX;
    out[1] = g < 8 ? 8 : g;
    out[2] = g;
}

cudaError_t launch_resample(const RJob *jobs_dev, int njobs, int64_t total_bricks, int dtype, int kind, int g,
                            int interp, cudaStream_t st, int sm_count)
{
    if (total_bricks <= 0) return cudaSuccess;
    if (kind == 0) {
        if (dtype == 1) return interp ? launch_affine_t<uint8_t, 1>(jobs_dev, njobs, total_bricks, st, sm_count)
                                      : launch_affine_t<uint8_t, 0>(jobs_dev, njobs, total_bricks, st, sm_count);
        return interp ? launch_affine_t<uint16_t, 1>(jobs_dev, njobs, total_bricks, st, sm_count)
                      : launch_affine_t<uint16_t, 0>(jobs_dev, njobs, total_bricks, st, sm_count);
    }
    if (dtype == 1) return interp ? dispatch_g<uint8_t, 1>(jobs_dev, njobs, total_bricks, g, st, sm_count)
                                  : dispatch_g<uint8_t, 0>(jobs_dev, njobs, total_bricks, g, st, sm_count);
    return interp ? dispatch_g<uint16_t, 1>(jobs_dev, njobs, total_bricks, g, st, sm_count)
                  : dispatch_g<uint16_t, 0>(jobs_dev, njobs, total_bricks, g, st, sm_count);
}

}  // namespace tw
