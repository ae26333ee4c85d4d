// tw_resample.cu -- fused cubic B-spline expansion + trilinear/NN resampling
// of uint8/uint16 volumes on sm_100a, for TPS (node-grid) and affine warps.
//
// A launch covers the work units of one or more jobs that share (dtype,
// kind, g): the flattened unit index is mapped to its job by a binary search
// over the jobs' prefix sums, so uneven edge tiles and many small jobs run in
// one persistent launch.
//
// TPS units (reference: q_dfblcokinterp_bspline + q_imgblockwarp,
// q_imgwarp_tps_quicksmallmemory.cpp:85-203, and chazhi.cu:226-338, which
// does a dense 64x64x3 matvec per 4^3 cell and gathers every voxel from
// global memory): a column of 64 x 16 output voxels walks down its planes.
// The cubic B-spline is evaluated separably: per cell layer the 4 x (CY+3) x
// (CX+3) nodes are staged in shared memory as node' = DF + node position -
// frame origin (the B-spline reproduces linear functions, so the spline of
// node' is the sample position q itself), contracted along y once per layer
// (R), along z once per output plane (Q), and along x per voxel (12 FMA) --
// ~14 FMA per voxel instead of 192.  The column's source footprint is staged
// in shared memory by TMA, plane by plane, so that the eight taps of every
// voxel are shared-memory loads (see "TPS units" below).
//
// Affine bricks are 256 x 8 x 8 output voxels gathered from global memory.
//
// Sampling follows the reference exactly: a sample with any q_i < 0 or
// q_i > sz_i - 1 writes 0; weights come from floor(q); TPS rounds with +0.5
// and truncates, affine truncates (q_warp_affine_tps.cpp:1433).  A unit whose
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

// ---------------------------------------------------------------- packed FP32x2
// Blackwell issues two FP32 operations per instruction (FFMA2/FADD2).  The
// unchecked path of a lane's voxel pair is written in pairs: the B-spline
// taps as (x, y) per voxel and (z0, z1) across the pair (Q stores z twice),
// floor/frac on the same pairs, and the trilinear lerps across the pair.

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as one FFMA2 (b * -1 + a, a single rounding, so exact like a
// subtraction); negating both lanes first would cost two logic ops
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

// Packs the low halfword (u16) or byte (u8) of two words: voxel pair x, x+1.
template <typename T>
__device__ __forceinline__ uint32_t pack_pair(uint32_t a, uint32_t b)
{
    return sizeof(T) == 2 ? __byte_perm(a, b, 0x5410) : __byte_perm(a, b, 0x0040);
}

// Stores a packed voxel pair: one 2-element store when aligned, else per
// element within the row's valid extent.
template <typename T>
__device__ __forceinline__ void store_packed(T *p, uint32_t w, bool pair_ok, int nvalid)
{
    if (pair_ok && nvalid >= 2) {
        if (sizeof(T) == 2) *reinterpret_cast<uint32_t *>(p) = w;
        else *reinterpret_cast<uint16_t *>(p) = (uint16_t)w;
    } else {
        const int sh = 8 * (int)sizeof(T);
        if (nvalid >= 1) p[0] = (T)(w & ((1u << sh) - 1u));
        if (nvalid >= 2) p[1] = (T)((w >> sh) & ((1u << sh) - 1u));
    }
}

// Magic float 2^23 + v for a loaded voxel value v (exact for v < 2^23).
template <typename T>
__device__ __forceinline__ float mag(const T *p)
{
    return __int_as_float(0x4B000000 | (int)(uint32_t)__ldg(p));
}

// Per-lane constants of the packed path: weight pairs for the two voxels.
struct PairW {
    float2 w0[4];  // (w_a(0), w_a(0))
    float2 w1[4];  // (w_a(1), w_a(1))
    float2 wz[4];  // (w_a(0), w_a(1))
};

__device__ __forceinline__ PairW make_pairw(const float4 (&wx)[2])
{
    PairW p;
    const float a0[4] = {wx[0].x, wx[0].y, wx[0].z, wx[0].w};
    const float a1[4] = {wx[1].x, wx[1].y, wx[1].z, wx[1].w};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        p.w0[a] = f2(a0[a], a0[a]);
        p.w1[a] = f2(a1[a], a1[a]);
        p.wz[a] = f2(a0[a], a1[a]);
    }
    return p;
}

// Sample positions of a TPS voxel pair from its 4 x-taps: (qx, qy) of voxel
// 0 and of voxel 1, and (qz0, qz1).
__device__ __forceinline__ void pair_positions(const float4 n[4], const PairW &pw, float2 &p0, float2 &p1, float2 &pz2)
{
    p0 = make_float2(0.f, 0.f);
    p1 = p0;
    pz2 = p0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const float2 xy = f2(n[a].x, n[a].y);
        const float2 zz = f2(n[a].z, n[a].w);  // Q stores (x, y, z, z)
        p0 = fma2(pw.w0[a], xy, p0);
        p1 = fma2(pw.w1[a], xy, p1);
        pz2 = fma2(pw.wz[a], zz, pz2);
    }
}

// The four source rows a trilinear sample reads, (dy, dz) = (r & 1, r >> 1),
// as base pointers of one brick, plus the int32 pitches.  The bases sit at
// the low corner of the brick's sample hull, so every unchecked tap is a
// non-negative 32-bit element offset from them, and a tap address is one
// wide unsigned multiply-add onto a row base.
template <typename T>
struct Rows {
    const T *rb[4];
    int py, pz;
    uint32_t k;  // magic-number bias and the hull corner folded out of the offsets
};

// corner: the low corner (relative to `base`) of the box every tap of the
// brick lies in -- the clamp window of its checked samples, which also holds
// every unchecked tap -- so tap offsets from it are non-negative; used only
// when `valid` (offsets within the box fit 32 bits).
template <typename T>
__device__ __forceinline__ Rows<T> make_rows(const T *base, int py, int pz, const int (&corner)[3], bool valid)
{
    const int omin = valid ? corner[2] * pz + corner[1] * py + corner[0] : 0;
    const T *b = base + omin;
    Rows<T> r;
    r.rb[0] = b;
    r.rb[1] = b + py;
    r.rb[2] = b + pz;
    r.rb[3] = b + pz + py;
    r.py = py;
    r.pz = pz;
    r.k = (uint32_t)kMagicBits * (uint32_t)(pz + py + 1) + (uint32_t)omin;
    return r;
}

// Element offset of floor(q) from the rows' corner, from the
// magic-floor bit patterns (2^32 wrap arithmetic; exact because the result
// lies in [0, 2^31)).
template <typename T>
__device__ __forceinline__ uint32_t tap_offset(const Rows<T> &R, float mx, float my, float mz)
{
    return (uint32_t)__float_as_int(mz) * (uint32_t)R.pz + (uint32_t)__float_as_int(my) * (uint32_t)R.py +
           (uint32_t)__float_as_int(mx) - R.k;
}

// base + o elements as one wide unsigned multiply-add.
template <typename T>
__device__ __forceinline__ const T *wide_addr(const T *base, uint32_t o)
{
    const T *p;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(p) : "r"(o), "r"((uint32_t)sizeof(T)), "l"(base));
    return p;
}

// Trilinear value of a voxel pair from the magic floats 2^23 + v of its taps:
// lo[r] / hi[r] hold the x and x+1 taps of source row r = (dy, dz) =
// (r & 1, r >> 1), as (voxel 0, voxel 1).  Every sampler (global gathers,
// staged shared memory, checked or not) ends in this one sequence of
// operations, so a voxel's value does not depend on which path produced it.
__device__ __forceinline__ float2 trilerp2(const float2 (&lo)[4], const float2 (&hi)[4], float2 fx, float2 fy,
                                           float2 fz)
{
    float2 ax[4];
#pragma unroll
    for (int r = 0; r < 4; ++r)  // (2^23 + b) - (2^23 + a) = b - a exactly
        ax[r] = fma2(fx, sub2(hi[r], lo[r]), sub2(lo[r], f2(8388608.f, 8388608.f)));
    const float2 b0 = fma2(fy, sub2(ax[1], ax[0]), ax[0]);
    const float2 b1 = fma2(fy, sub2(ax[3], ax[2]), ax[2]);
    return fma2(fz, sub2(b1, b0), b0);
}

// Unchecked sample of a voxel pair at positions (p0, p1, pz2): every tap is
// known to be inside the volume and the buffer (hull test), offsets fit int32.
// Trilinear value of a voxel pair from the offsets of its (0,0,0) taps and
// its fractions (fx, fy, fz), as a pair (voxel 0, voxel 1).
template <typename T>
__device__ __forceinline__ float2 lerp_pair(const Rows<T> &R, uint32_t off0, uint32_t off1, float2 fx, float2 fy,
                                            float2 fz)
{
    // magic floats of the 8 taps of both voxels: one wide address per voxel,
    // the other rows at the brick's constant row / plane offsets
    float2 lo[4], hi[4];
    const T *a0 = wide_addr(R.rb[0], off0), *a1 = wide_addr(R.rb[0], off1);
    const int rofs[4] = {0, R.py, R.pz, R.py + R.pz};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const T *q0 = a0 + rofs[r], *q1 = a1 + rofs[r];
        lo[r] = f2(mag(q0), mag(q1));
        hi[r] = f2(mag(q0 + 1), mag(q1 + 1));
    }
    return trilerp2(lo, hi, fx, fy, fz);
}

// Output words of a voxel pair: TPS rounds (+0.5), affine truncates; v is a
// convex combination of voxel values (rounding can leave -0.0x), so
// 2^23 + floor(v) has the output in its low bits.
template <typename T, bool ROUND>
__device__ __forceinline__ float2 out_pair(float2 v)
{
    if (ROUND) v = add2(v, f2(0.5f, 0.5f));
    else v = f2(fmaxf(v.x, 0.f), fmaxf(v.y, 0.f));
    return __fadd2_rd(v, f2(8388608.f, 8388608.f));
}

template <typename T, bool ROUND>
__device__ __forceinline__ void pair_fast2(float2 p0, float2 p1, float2 pz2, const Rows<T> &R, uint32_t &packed)
{
    const float2 MM = f2(kMagic, kMagic);
    // floor via add.rm of 1.5*2^23, fractions
    const float2 m0 = __fadd2_rd(p0, MM), m1 = __fadd2_rd(p1, MM), mz = __fadd2_rd(pz2, MM);
    const float2 f0 = sub2(p0, sub2(m0, MM)), f1 = sub2(p1, sub2(m1, MM)), fz = sub2(pz2, sub2(mz, MM));
    const uint32_t off0 = tap_offset(R, m0.x, m0.y, mz.x);
    const uint32_t off1 = tap_offset(R, m1.x, m1.y, mz.y);
    const float2 t = out_pair<T, ROUND>(lerp_pair(R, off0, off1, f2(f0.x, f1.x), f2(f0.y, f1.y), fz));
    packed = pack_pair<T>(__float_as_uint(t.x), __float_as_uint(t.y));
}

// Checked sample of a voxel pair with 32-bit offsets: the reference's range
// test per voxel (0 <= q <= sz-1 in every axis, else 0), and floor(q) clamped
// to [cl, ch-1] of the clamp window so that both taps of every axis are
// inside it.  For a valid sample the clamp changes nothing except at q =
// sz-1 exactly, where floor sz-2 with fraction 1 gives the same value as the
// reference's floor sz-1 with fraction 0 (lo + 1 (hi - lo) = hi exactly).
// Needs ch > cl in every axis.
template <typename T, bool ROUND>
__device__ __forceinline__ void pair_clamped2(float2 p0, float2 p1, float2 pz2, const Rows<T> &R, const Frame &f,
                                              const int (&cl)[3], const int (&ch)[3], int nvalid, uint32_t &packed)
{
    const float2 MM = f2(kMagic, kMagic);
    const bool ok0 = nvalid >= 1 && p0.x >= f.lo[0] && p0.x <= f.hi[0] && p0.y >= f.lo[1] && p0.y <= f.hi[1] &&
                     pz2.x >= f.lo[2] && pz2.x <= f.hi[2];
    const bool ok1 = nvalid >= 2 && p1.x >= f.lo[0] && p1.x <= f.hi[0] && p1.y >= f.lo[1] && p1.y <= f.hi[1] &&
                     pz2.y >= f.lo[2] && pz2.y <= f.hi[2];
    const float lx = (float)cl[0], ly = (float)cl[1], lz = (float)cl[2];
    const float hx = (float)(ch[0] - 1), hy = (float)(ch[1] - 1), hz = (float)(ch[2] - 1);
    // floors (NaN or huge positions clamp into the window; such voxels are
    // rejected by the range test above)
    float2 l0 = sub2(__fadd2_rd(p0, MM), MM), l1 = sub2(__fadd2_rd(p1, MM), MM), lz2 = sub2(__fadd2_rd(pz2, MM), MM);
    l0 = f2(fminf(fmaxf(l0.x, lx), hx), fminf(fmaxf(l0.y, ly), hy));
    l1 = f2(fminf(fmaxf(l1.x, lx), hx), fminf(fmaxf(l1.y, ly), hy));
    lz2 = f2(fminf(fmaxf(lz2.x, lz), hz), fminf(fmaxf(lz2.y, lz), hz));
    const float2 f0 = sub2(p0, l0), f1 = sub2(p1, l1), fz = sub2(pz2, lz2);
    const float2 m0 = add2(l0, MM), m1 = add2(l1, MM), mz = add2(lz2, MM);  // exact: integers
    const uint32_t off0 = tap_offset(R, m0.x, m0.y, mz.x);
    const uint32_t off1 = tap_offset(R, m1.x, m1.y, mz.y);
    const float2 t = out_pair<T, ROUND>(lerp_pair(R, off0, off1, f2(f0.x, f1.x), f2(f0.y, f1.y), fz));
    // a rejected voxel writes 0: the bits of 2^23 have zero low bits
    packed = pack_pair<T>(ok0 ? __float_as_uint(t.x) : 0x4B000000u, ok1 ? __float_as_uint(t.y) : 0x4B000000u);
}

// Checked sample of a voxel pair near the volume or buffer border: the same
// packed arithmetic, plus the reference's range test per voxel (0 <= q <=
// sz-1, else 0) and taps clamped to [cl, ch] (the source buffer, narrowed to
// the brick's sample hull so that offsets stay 32-bit).  A tap clamped away
// from floor(q)+1 only happens where its weight is 0 (q integral at sz-1).
template <typename T, bool ROUND, typename OFF>
__device__ __forceinline__ void pair_checked2(float2 p0, float2 p1, float2 pz2, const T *__restrict__ base, OFF py,
                                              OFF pz, const Frame &f, const int (&cl)[3], const int (&ch)[3],
                                              int nvalid, uint32_t &packed)
{
    const float2 MM = f2(kMagic, kMagic);
    const bool ok0 = nvalid >= 1 && p0.x >= f.lo[0] && p0.x <= f.hi[0] && p0.y >= f.lo[1] && p0.y <= f.hi[1] &&
                     pz2.x >= f.lo[2] && pz2.x <= f.hi[2];
    const bool ok1 = nvalid >= 2 && p1.x >= f.lo[0] && p1.x <= f.hi[0] && p1.y >= f.lo[1] && p1.y <= f.hi[1] &&
                     pz2.y >= f.lo[2] && pz2.y <= f.hi[2];
    // positions of rejected voxels are replaced by the frame's low corner so
    // that the magic floor below stays exact (NaN or far-away q)
    if (!ok0) { p0 = f2(f.lo[0], f.lo[1]); pz2.x = f.lo[2]; }
    if (!ok1) { p1 = f2(f.lo[0], f.lo[1]); pz2.y = f.lo[2]; }
    const float2 m0 = __fadd2_rd(p0, MM), m1 = __fadd2_rd(p1, MM), mz = __fadd2_rd(pz2, MM);
    const float2 f0 = sub2(p0, sub2(m0, MM)), f1 = sub2(p1, sub2(m1, MM)), fz = sub2(pz2, sub2(mz, MM));
    const int ix0 = __float_as_int(m0.x) - kMagicBits, iy0 = __float_as_int(m0.y) - kMagicBits;
    const int ix1 = __float_as_int(m1.x) - kMagicBits, iy1 = __float_as_int(m1.y) - kMagicBits;
    const int iz0 = __float_as_int(mz.x) - kMagicBits, iz1 = __float_as_int(mz.y) - kMagicBits;
    const int xa0 = clampi(ix0, cl[0], ch[0]), xb0 = clampi(ix0 + 1, cl[0], ch[0]);
    const int xa1 = clampi(ix1, cl[0], ch[0]), xb1 = clampi(ix1 + 1, cl[0], ch[0]);
    const int ya0 = clampi(iy0, cl[1], ch[1]), yb0 = clampi(iy0 + 1, cl[1], ch[1]);
    const int ya1 = clampi(iy1, cl[1], ch[1]), yb1 = clampi(iy1 + 1, cl[1], ch[1]);
    const int za0 = clampi(iz0, cl[2], ch[2]), zb0 = clampi(iz0 + 1, cl[2], ch[2]);
    const int za1 = clampi(iz1, cl[2], ch[2]), zb1 = clampi(iz1 + 1, cl[2], ch[2]);
    const int ys0[2] = {ya0, yb0}, ys1[2] = {ya1, yb1}, zs0[2] = {za0, zb0}, zs1[2] = {za1, zb1};
    float2 lo[4], hi[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const T *r0 = base + ((OFF)zs0[r >> 1] * pz + (OFF)ys0[r & 1] * py);
        const T *r1 = base + ((OFF)zs1[r >> 1] * pz + (OFF)ys1[r & 1] * py);
        lo[r] = f2(mag(r0 + xa0), mag(r1 + xa1));
        hi[r] = f2(mag(r0 + xb0), mag(r1 + xb1));
    }
    const float2 t = out_pair<T, ROUND>(trilerp2(lo, hi, f2(f0.x, f1.x), f2(f0.y, f1.y), fz));
    // a rejected voxel writes 0: the bits of 2^23 have zero low bits
    packed = pack_pair<T>(ok0 ? __float_as_uint(t.x) : 0x4B000000u, ok1 ? __float_as_uint(t.y) : 0x4B000000u);
}

// Clamp window of a brick's checked taps: the source buffer narrowed to the
// brick's sample hull (+1), and whether offsets inside it fit int32.
struct Clamp {
    int cl[3], ch[3];
    bool span32;   // offsets within the window fit 32 bits (the rows' corner is cl)
    bool clamped;  // span32 and at least two taps wide in every axis: pair_clamped2 applies
};

__device__ __forceinline__ Clamp make_clamp(const RJob &J, const Frame &f, const float (&mn)[3], const float (&mx)[3])
{
    Clamp c;
    double span = 0.0;
    const double pitch[3] = {1.0, (double)J.src_py, (double)J.src_pz};
    for (int a = 0; a < 3; ++a) {
        const double lo = fmax(-1.0e9, fmin(1.0e9, floor((double)mn[a]) - 1.0));
        const double hi = fmax(-1.0e9, fmin(1.0e9, floor((double)mx[a]) + 2.0));
        int l = max(f.bl[a], (int)lo), h = min(f.bh[a], (int)hi);
        if (l > h) l = h = f.bl[a];  // no sample can be valid here; any in-buffer tap will do
        c.cl[a] = l;
        c.ch[a] = h;
        span += fmax(fabs((double)l), fabs((double)h)) * pitch[a];
    }
    c.span32 = span < 1.0e9 && J.src_pz < 0x3fffffff;
    c.clamped = c.span32 && c.ch[0] > c.cl[0] && c.ch[1] > c.cl[1] && c.ch[2] > c.cl[2];
    return c;
}

// ------------------------------------------------------------- TPS units
//
// A TPS work unit is a column of 64 x 16 output voxels (x, y) over a run of
// output planes: part of one control-cell layer (small jobs) or several
// whole layers.  The unit walks its planes in order.  Each cell layer is
// evaluated in its own frame -- origin at the column's corner on the layer's
// first plane -- so a voxel's position and value do not depend on how the
// volume is cut into units or how units are batched.  Lane l of warp w owns
// the voxel pair (2l, 2l+1) of rows w and w+8: a warp covers one whole row,
// so its taps for one source row are 64 consecutive-ish voxels.
//
// Staged walks.  The column's source footprint over a walk -- the convex
// hull of its B-spline nodes' displacements (weights >= 0, sum 1) plus the
// +1 tap -- is a box of at most kBoxW x kHMax elements per source plane and
// a window of planes that slides down one plane per output plane.  The box's
// rows are copied into a ring of plane slots in shared memory by TMA
// (cp.async.bulk.tensor, one row per copy from this GPU's own memory,
// completion counted on one mbarrier per slot), kAhead planes ahead of the
// plane being sampled, and every tap becomes a shared-memory load.  Slot 0
// also has a copy one slot past the end, so the z+1 tap of any plane is at a
// fixed offset.  The slots' row pitch is 128 elements: a step of a row or a
// plane then moves an address by a multiple of 32 banks, so the loads of a
// warp's 64 voxels hit 32 distinct banks whichever rows and planes the lanes
// read.  A walk whose box or window does not fit, a nearest-neighbour job,
// or a source buffer TMA cannot describe gathers from global memory instead,
// with the same positions and the same trilinear arithmetic (trilerp2).

constexpr int kTBX = 64;               // unit width (x): 32 lanes x 2 voxels
constexpr int kTBY = 16;               // unit height (y)
constexpr int kTRows = kTBY / kTY;     // rows per warp
constexpr int kBoxW = kStageBoxW;      // TMA box: source elements per row copy
constexpr int kRowP = 128;             // shared-memory row pitch (elements)
constexpr int kHMax = 28;              // staged rows per plane
constexpr int kAhead = 2;              // planes copied ahead of the plane being sampled
// a staged plane that has not landed after this long is an error (the wait
// gives up, the kernel reports kKernErrTimeout and returns)
constexpr unsigned long long kStageWaitNs = 2000000000ull;

template <typename T, int G>
struct TGeom {
    static constexpr int CX = kTBX / G;               // cells along x (G <= 64)
    static constexpr int CY = G < kTBY ? kTBY / G : 1; // cell rows a unit's 16 rows touch
    static constexpr int NX = CX + 3;
    static constexpr int NY = CY + 3;
    static constexpr int ND = 4 * NY * NX;            // staged nodes of one layer
    static constexpr int NR = kTBY * 4 * NX;          // y-contracted
    static constexpr int NQ = 2 * kTBY * NX;          // z-contracted, double-buffered
    static constexpr int UNION = ND > NQ ? ND : NQ;
    static constexpr int R = G == 4 ? 10 : 12;        // ring slots (plus the mirror of slot 0)
    static constexpr int ES = (int)sizeof(T);
    static constexpr int ROW_B = kRowP * ES;
    static constexpr int PLANE_B = kHMax * ROW_B;
    static constexpr int RING_B = (R + 1) * PLANE_B;
    static constexpr int MBAR_B = 8 * 16;
    static constexpr size_t smem_bytes = 128 + (size_t)RING_B + MBAR_B + sizeof(float4) * (size_t)(UNION + NR + G);
    static_assert(R <= 16, "one mbarrier per slot, 16 at most");
};

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of parity `parity` of the mbarrier at `a`; gives up
// (false) after kStageWaitNs.
__device__ __noinline__ bool mbar_wait_slow(uint32_t a, uint32_t parity)
{
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned i = 1;; ++i) {
        if (mbar_try(a, parity)) return true;
        if ((i & 255u) == 0 && globaltimer_ns() - t0 > kStageWaitNs) return false;
    }
}

__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity)
{
    return mbar_try(a, parity) || mbar_wait_slow(a, parity);
}

// One row of a staged plane: kBoxW elements at tensor coordinates (x, y, z)
// of the job's source buffer (elements outside it read as 0) into shared
// memory at dst; completion is counted on the mbarrier at mbar.
__device__ __forceinline__ void tma_row(uint32_t dst, const CUtensorMap *map, int x, int y, int z, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ int pmod(int64_t p, int r)
{
    const int64_t m = p % r;
    return (int)(m < 0 ? m + r : m);
}

// Shared memory of a TPS CTA.
template <typename T, int G>
struct TSmem {
    unsigned char *base;  // 128-byte aligned start of the ring
    uint32_t sring;       // shared-window address of slot 0
    uint32_t smbar;       // shared-window address of slot 0's mbarrier (8 bytes each)
    float4 *Nd, *Qb, *R, *W;
};

// State of a staged walk; every thread holds the same values.
struct Stage {
    int a, b;             // output plane z reads source planes [z + a, z + b]
    int rx0, ry0, rows;   // staged box: buffer column and row of its first element, rows per plane
    int DX, DY;           // box column / row of frame x = 0 / y = 0
    int64_t issued;       // last plane copied (buffer z)
    int64_t waited;       // last plane this thread waited for (buffer z)
    int64_t last;         // last plane the walk reads (buffer z)
    uint32_t kxy;         // offset (from base) of frame x = y = 0 in slot 0, magic-float bias folded in
    uint32_t omax;        // largest offset whose 8 taps all stay inside the ring
};

// Copies staged plane p (buffer z) into its slot; executed by warp 0.
template <typename T, int G>
__device__ __forceinline__ void stage_issue(const RJob &J, const TSmem<T, G> &S, const Stage &st, int64_t p, int lane)
{
    using Gm = TGeom<T, G>;
    const int s = pmod(p, Gm::R);
    const uint32_t mb = S.smbar + 8u * (uint32_t)s;
    const uint32_t bytes = (uint32_t)(kBoxW * Gm::ES) * (uint32_t)st.rows * (s == 0 ? 2u : 1u);
    if (lane == 0) mbar_expect_tx(mb, bytes);
    __syncwarp();
    if (lane < st.rows) {
        // the slot's previous plane was read by every thread before the
        // barrier that precedes this call; order those generic-proxy reads
        // before the asynchronous write
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint32_t d = S.sring + (uint32_t)(s * Gm::PLANE_B + lane * Gm::ROW_B);
        tma_row(d, &J.tmap, st.rx0, st.ry0 + lane, (int)p, mb);
        if (s == 0) tma_row(d + (uint32_t)(Gm::R * Gm::PLANE_B), &J.tmap, st.rx0, st.ry0 + lane, (int)p, mb);
    }
}

// Waits for every plane up to `upto` (buffer z); false if a wait gave up.
template <typename T, int G>
__device__ __forceinline__ bool stage_wait(const TSmem<T, G> &S, Stage &st, uint32_t &parity, int64_t upto)
{
    using Gm = TGeom<T, G>;
    while (st.waited < upto) {
        const int64_t p = st.waited + 1;
        const int s = pmod(p, Gm::R);
        if (!mbar_wait(S.smbar + 8u * (uint32_t)s, (parity >> s) & 1u)) return false;
        parity ^= 1u << s;
        st.waited = p;
    }
    return true;
}

// Offset (from base) of the (x, y, z) = floor tap of a staged sample, from the
// magic-floor bit patterns; clamped so that all 8 taps stay in the ring.
template <typename T, int G>
__device__ __forceinline__ uint32_t staged_off(const Stage &st, uint32_t cz, float mx, float my, float mz)
{
    using Gm = TGeom<T, G>;
    const uint32_t t = __float_as_uint(mz) + cz;  // slot + (0 or R) for the planes of the window
    const uint32_t slot = min(t, t - (uint32_t)Gm::R);
    const uint32_t o = slot * (uint32_t)Gm::PLANE_B + __float_as_uint(my) * (uint32_t)Gm::ROW_B +
                       __float_as_uint(mx) * (uint32_t)Gm::ES + st.kxy;
    return min(o, st.omax);
}

// Magic float 2^23 + v of the staged voxel at offset o.
template <typename T>
__device__ __forceinline__ float smag(const unsigned char *sm, uint32_t o)
{
    return __int_as_float(0x4B000000 | (int)(uint32_t)*reinterpret_cast<const T *>(sm + o));
}

// A voxel pair sampled from the staged planes.  CHECKED applies the
// reference's range rule per voxel (0 <= q <= sz-1, else 0) and clamps floor(q)
// into the staged window (wl, wh: frame coordinates) so that no tap of an
// invalid sample leaves it; for a valid sample the clamp changes nothing (the
// window holds the whole footprint), so both variants give the same bits.
template <typename T, int G, bool ROUND, bool CHECKED>
__device__ __forceinline__ uint32_t pair_staged(const unsigned char *sm, const Stage &st, uint32_t cz, float2 p0,
                                                float2 p1, float2 pz2, const Frame &f, const float (&wl)[3],
                                                const float (&wh)[3], int nvalid)
{
    using Gm = TGeom<T, G>;
    const float2 MM = f2(kMagic, kMagic);
    float2 m0, m1, mz, f0, f1, fz;
    bool ok0 = true, ok1 = true;
    if (CHECKED) {
        ok0 = nvalid >= 1 && p0.x >= f.lo[0] && p0.x <= f.hi[0] && p0.y >= f.lo[1] && p0.y <= f.hi[1] &&
              pz2.x >= f.lo[2] && pz2.x <= f.hi[2];
        ok1 = nvalid >= 2 && p1.x >= f.lo[0] && p1.x <= f.hi[0] && p1.y >= f.lo[1] && p1.y <= f.hi[1] &&
              pz2.y >= f.lo[2] && pz2.y <= f.hi[2];
        float2 l0 = sub2(__fadd2_rd(p0, MM), MM), l1 = sub2(__fadd2_rd(p1, MM), MM);
        float2 lz2 = sub2(__fadd2_rd(pz2, MM), MM);
        l0 = f2(fminf(fmaxf(l0.x, wl[0]), wh[0]), fminf(fmaxf(l0.y, wl[1]), wh[1]));
        l1 = f2(fminf(fmaxf(l1.x, wl[0]), wh[0]), fminf(fmaxf(l1.y, wl[1]), wh[1]));
        lz2 = f2(fminf(fmaxf(lz2.x, wl[2]), wh[2]), fminf(fmaxf(lz2.y, wl[2]), wh[2]));
        f0 = sub2(p0, l0);
        f1 = sub2(p1, l1);
        fz = sub2(pz2, lz2);
        m0 = add2(l0, MM);  // exact: integers
        m1 = add2(l1, MM);
        mz = add2(lz2, MM);
    } else {
        m0 = __fadd2_rd(p0, MM);
        m1 = __fadd2_rd(p1, MM);
        mz = __fadd2_rd(pz2, MM);
        f0 = sub2(p0, sub2(m0, MM));
        f1 = sub2(p1, sub2(m1, MM));
        fz = sub2(pz2, sub2(mz, MM));
    }
    const uint32_t o0 = staged_off<T, G>(st, cz, m0.x, m0.y, mz.x);
    const uint32_t o1 = staged_off<T, G>(st, cz, m1.x, m1.y, mz.y);
    constexpr uint32_t rofs[4] = {0u, (uint32_t)Gm::ROW_B, (uint32_t)Gm::PLANE_B, (uint32_t)(Gm::PLANE_B + Gm::ROW_B)};
    float2 lo[4], hi[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        lo[r] = f2(smag<T>(sm, o0 + rofs[r]), smag<T>(sm, o1 + rofs[r]));
        hi[r] = f2(smag<T>(sm, o0 + rofs[r] + Gm::ES), smag<T>(sm, o1 + rofs[r] + Gm::ES));
    }
    const float2 t = out_pair<T, ROUND>(trilerp2(lo, hi, f2(f0.x, f1.x), f2(f0.y, f1.y), fz));
    if (CHECKED)  // a rejected voxel writes 0: the bits of 2^23 have zero low bits
        return pack_pair<T>(ok0 ? __float_as_uint(t.x) : 0x4B000000u, ok1 ? __float_as_uint(t.y) : 0x4B000000u);
    return pack_pair<T>(__float_as_uint(t.x), __float_as_uint(t.y));
}

// Everything a lane needs about its unit's current layer.
template <typename T>
struct BrickCtx {
    const T *base;      // source element at the frame origin (may lie outside the buffer)
    int py32, pz32;     // source pitches as int (valid when the brick's offsets fit int32)
    int64_t py, pz;     // source pitches
    Frame frame;
    Clamp cw;
    Rows<T> rows;
    PairW pw;           // packed x weights of the lane's voxel pair
    float4 wx[2];       // scalar x weights (nearest-neighbour path)
    bool pair_ok;       // a voxel pair can be stored as one 2-element word
    int xe, ye;         // valid x / y extent of the unit's output region
};

// A voxel pair gathered from global memory (every path but the staged one).
template <typename T, int G, int INTERP>
__device__ __forceinline__ void tps_pair(const float4 (&n)[4], const BrickCtx<T> &B, int x, bool fast, T *drow)
{
    if constexpr (INTERP == 0) {
        float2 p0, p1, pz2;
        pair_positions(n, B.pw, p0, p1, pz2);
        uint32_t w;
        if (fast) {
            pair_fast2<T, true>(p0, p1, pz2, B.rows, w);
            store_packed<T>(drow + x, w, B.pair_ok, 2);
        } else {
            const int nv = B.xe - x;
            if (B.cw.clamped)
                pair_clamped2<T, true>(p0, p1, pz2, B.rows, B.frame, B.cw.cl, B.cw.ch, nv, w);
            else if (B.cw.span32)
                pair_checked2<T, true, int>(p0, p1, pz2, B.base, B.py32, B.pz32, B.frame, B.cw.cl, B.cw.ch, nv, w);
            else
                pair_checked2<T, true, int64_t>(p0, p1, pz2, B.base, B.py, B.pz, B.frame, B.cw.cl, B.cw.ch, nv, w);
            store_packed<T>(drow + x, w, B.pair_ok, nv);
        }
    } else {
        uint32_t outv[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float4 w = B.wx[j];
            const float qx = fmaf(w.x, n[0].x, fmaf(w.y, n[1].x, fmaf(w.z, n[2].x, w.w * n[3].x)));
            const float qy = fmaf(w.x, n[0].y, fmaf(w.y, n[1].y, fmaf(w.z, n[2].y, w.w * n[3].y)));
            const float qz = fmaf(w.x, n[0].z, fmaf(w.y, n[1].z, fmaf(w.z, n[2].z, w.w * n[3].z)));
            float v;
            if (fast) {
                v = sample_fast<T, INTERP>(B.base, B.py32, B.pz32, qx, qy, qz);
                outv[j] = INTERP == 1 ? (uint32_t)v : to_out<T, true>(v);
            } else {
                const bool ok =
                    (x + j) < B.xe && sample_checked<T, INTERP>(B.base, B.py, B.pz, B.frame, qx, qy, qz, v);
                outv[j] = ok ? (INTERP == 1 ? (uint32_t)v : to_out<T, true>(v)) : 0u;
            }
        }
        store_pair<T>(drow + x, outv[0], outv[1], B.pair_ok, fast ? 2 : B.xe - x);
    }
}

// Planes [zf, zf + zn) of one cell layer of a unit (global output z), in the
// layer's frame.  STAGED: the taps come from the walk's staged planes (the
// walk's copies are issued and waited for here, one plane per output plane).
// Returns false when a staged wait gave up (tmo set); every thread returns
// the same.
template <typename T, int G, int INTERP, bool STAGED>
__device__ bool tps_layer(const RJob &J, int64_t Ox, int64_t Oy, int64_t zf, int zn, const TSmem<T, G> &S, Stage &st,
                          uint32_t &parity, int &tmo, float *red, unsigned char *segf)
{
    using Gm = TGeom<T, G>;
    float4 *Nd = S.Nd;  // [4][NY][NX]   (aliases Qb)
    float4 *Qb = S.Qb;  // [2][kTBY][NX]
    float4 *R = S.R;    // [kTBY][4][NX]
    const float4 *W = S.W;
    const int tid = threadIdx.x;
    const int tx = tid & 31, ty = tid >> 5;

    // frame: the column's corner on the layer's first plane
    const int64_t Oz = (zf / G) * G;
    const int64_t O[3] = {Ox, Oy, Oz};
    const int64_t c0[3] = {Ox / G, Oy / G, Oz / G};  // first node index per axis
    const int yoff = (int)(Oy - c0[1] * G);           // rows of the first cell above the unit (G > 16)
    const int zoff = (int)(zf - Oz);                  // first plane within the cell layer

    // 1. stage node' = DF + node position - O, and the range of DF (a
    // non-finite node forces the checked path)
    float dmn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, dmx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = tid; i < Gm::ND; i += kThreads) {
        const int nx = i % Gm::NX, t = i / Gm::NX;
        const int ny = t % Gm::NY, nz = t / Gm::NY;
        int64_t gx = c0[0] + nx, gy = c0[1] + ny, gz = c0[2] + nz;
        gx = gx < J.gsz[0] ? gx : J.gsz[0] - 1;
        gy = gy < J.gsz[1] ? gy : J.gsz[1] - 1;
        gz = gz < J.gsz[2] ? gz : J.gsz[2] - 1;
        const float4 d = J.nodes[(gz * J.gsz[1] + gy) * J.gsz[0] + gx];
        // node gx sits at (gx-1)*G; relative to O that is (gx-1)*G - O (exact in float)
        float4 v;
        v.x = d.x + (float)((gx - 1) * G - O[0]);
        v.y = d.y + (float)((gy - 1) * G - O[1]);
        v.z = d.z + (float)((gz - 1) * G - O[2]);
        v.w = 0.f;
        Nd[i] = v;
        if (isfinite(v.x) && isfinite(v.y) && isfinite(v.z)) {
            dmn[0] = fminf(dmn[0], d.x); dmn[1] = fminf(dmn[1], d.y); dmn[2] = fminf(dmn[2], d.z);
            dmx[0] = fmaxf(dmx[0], d.x); dmx[1] = fmaxf(dmx[1], d.y); dmx[2] = fmaxf(dmx[2], d.z);
        } else {
            dmn[0] = dmn[1] = dmn[2] = -3.4e38f;
            dmx[0] = dmx[1] = dmx[2] = 3.4e38f;
        }
    }
    block_minmax(dmn, dmx, red);  // contains __syncthreads (Nd visible after it)

    // Sample hull: a voxel at frame position p samples p + (a convex
    // combination of DF), so per axis q lies in [p + min DF, p + max DF].
    const float plo[3] = {0.f, 0.f, (float)zoff};
    const float phi[3] = {(float)(kTBX - 1), (float)(kTBY - 1), (float)(zoff + zn - 1)};
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = dmn[a] <= -3.0e38f ? -3.4e38f : plo[a] + dmn[a];
        mx[a] = dmx[a] >= 3.0e38f ? 3.4e38f : phi[a] + dmx[a];
    }
    const Frame frame = make_frame(J, O);
    const bool span_ok = offsets_fit_32(J, mn, mx);
    const Clamp cw = make_clamp(J, frame, mn, mx);

    // 2. R[y][c][nx] = sum_b wy_b(yoff + y) Nd[c][(yoff + y)/G + b][nx]
    for (int i = tid; i < Gm::NR; i += kThreads) {
        const int nx = i % Gm::NX, t = i / Gm::NX;
        const int c = t & 3, y = t >> 2;
        const int yy = yoff + y;
        const float4 w = W[yy % G];
        const float4 *n0 = Nd + (c * Gm::NY + yy / G) * Gm::NX + nx;
        const float4 a = n0[0], b = n0[Gm::NX], e = n0[2 * Gm::NX], f = n0[3 * Gm::NX];
        float4 r;
        r.x = fmaf(w.x, a.x, fmaf(w.y, b.x, fmaf(w.z, e.x, w.w * f.x)));
        r.y = fmaf(w.x, a.y, fmaf(w.y, b.y, fmaf(w.z, e.y, w.w * f.y)));
        r.z = fmaf(w.x, a.z, fmaf(w.y, b.z, fmaf(w.z, e.z, w.w * f.z)));
        r.w = 0.f;
        R[i] = r;
    }

    // Unchecked-path bounds per axis: every tap of a sample q with
    // lb <= q < hb lies inside the volume and the source buffer.
    float lb[3], hb[3];
    for (int a = 0; a < 3; ++a) {
        lb[a] = fmaxf(frame.lo[a], (float)frame.bl[a]) + 1.0f / 64.0f;
        hb[a] = fminf(frame.hi[a], (float)frame.bh[a]) - 1.0f / 64.0f;
    }
    // per row (64 voxels): may it skip the bounds checks in x and y?  (z is
    // decided per output plane below.)
    const int64_t xe = J.out_o[0] + J.out_n[0] - O[0];  // valid x extent in this unit
    const int64_t ye = J.out_o[1] + J.out_n[1] - O[1];
    if (tid < kTBY) {
        const int y = tid;
        const float qx0 = dmn[0], qx1 = (float)(kTBX - 1) + dmx[0];
        const float qy0 = (float)y + dmn[1], qy1 = (float)y + dmx[1];
        // (rows at or beyond ye are never written, so they need no test)
        const bool ok = (y >= ye) || (span_ok && cw.span32 && (kTBX <= xe) && qx0 >= lb[0] && qx1 < hb[0] &&
                                      qy0 >= lb[1] && qy1 < hb[1]);
        segf[y] = ok ? 1 : 0;
    }
    // plane z (at frame position pz) is unchecked in z when zlo <= pz < zhi
    const float zlo = lb[2] - dmn[2], zhi = hb[2] - dmx[2];

    const T *src = static_cast<const T *>(J.src);
    T *dst = static_cast<T *>(J.dst);
    const int64_t sbase = (O[2] - J.src_o[2]) * J.src_pz + (O[1] - J.src_o[1]) * J.src_py + (O[0] - J.src_o[0]);
    // output plane z of the loop below is zf + z
    const int64_t dbase0 = (zf - J.out_o[2]) * J.dst_pz + (O[1] - J.out_o[1]) * J.dst_py + (O[0] - J.out_o[0]);
    BrickCtx<T> B;
    B.base = src + sbase;
    B.py32 = (int)J.src_py;
    B.pz32 = (int)J.src_pz;
    B.py = J.src_py;
    B.pz = J.src_pz;
    B.frame = frame;
    B.cw = cw;
    B.rows = make_rows(B.base, B.py32, B.pz32, cw.cl, cw.span32);
    // x weights of the lane's voxel pair (2l, 2l+1): the unit's origin is a
    // multiple of G (G <= 64 divides 64)
    B.wx[0] = W[(2 * tx) % G];
    B.wx[1] = W[(2 * tx + 1) % G];
    B.pw = make_pairw(B.wx);
    // a voxel pair (even x) can be written as one 2-element store
    B.pair_ok = ((((uintptr_t)(dst + dbase0)) % (2 * sizeof(T))) == 0) && (J.dst_py % 2 == 0) && (J.dst_pz % 2 == 0);
    B.xe = (int)min(xe, (int64_t)kTBX);
    B.ye = (int)min(ye, (int64_t)kTBY);

    // staged window in frame coordinates (checked samples clamp into it)
    float wl[3] = {0.f, 0.f, 0.f}, wh[3] = {0.f, 0.f, 0.f};
    if (STAGED) {
        wl[0] = (float)(-st.DX);
        wh[0] = (float)(kBoxW - 2 - st.DX);
        wl[1] = (float)(-st.DY);
        wh[1] = (float)(st.rows - 2 - st.DY);
    }
    const unsigned char *sm = S.base;
    // R and the row flags are visible, and Nd (which Q overwrites) is no
    // longer read
    __syncthreads();

    for (int z = 0; z < zn; ++z) {
        float4 *Q = Qb + (z & 1) * (kTBY * Gm::NX);
        const float4 wz = W[zoff + z];
        for (int i = tid; i < kTBY * Gm::NX; i += kThreads) {
            const int nx = i % Gm::NX, y = i / Gm::NX;
            const float4 *r = R + (y * 4) * Gm::NX + nx;
            const float4 a = r[0], b = r[Gm::NX], e = r[2 * Gm::NX], f = r[3 * Gm::NX];
            float4 q;
            q.x = fmaf(wz.x, a.x, fmaf(wz.y, b.x, fmaf(wz.z, e.x, wz.w * f.x)));
            q.y = fmaf(wz.x, a.y, fmaf(wz.y, b.y, fmaf(wz.z, e.y, wz.w * f.y)));
            q.z = fmaf(wz.x, a.z, fmaf(wz.y, b.z, fmaf(wz.z, e.z, wz.w * f.z)));
            q.w = q.z;  // z twice: the packed path reads (z, z) as one pair
            Q[i] = q;
        }
        // every thread is done with the previous plane (its Q buffer, and for
        // a staged walk the slot the next copy overwrites); Q is visible
        if (__syncthreads_or(tmo)) return false;
        const int64_t zg = zf + z;
        uint32_t cz = 0;
        if (STAGED) {
            if (st.issued < st.last) {
                if (ty == 0) stage_issue<T, G>(J, S, st, st.issued + 1, tx);
                ++st.issued;
            }
            const int64_t sz0 = J.src_o[2];
            if (!stage_wait<T, G>(S, st, parity, zg + st.b - sz0)) {
                tmo = 1;
                continue;  // the next barrier ends the unit
            }
            // slot of a tap plane: t = (plane - window start) + slot(window start)
            const int64_t ws = zg + st.a - sz0;
            const int sws = pmod(ws, Gm::R);
            cz = (uint32_t)(int32_t)(Oz - zg - st.a + sws) - (uint32_t)kMagicBits;
            wl[2] = (float)(zg + st.a - Oz);
            wh[2] = (float)(zg + st.b - 1 - Oz);
        }
        // z of this plane: q_z lies in zoff + z + [min DF_z, max DF_z]
        const float pz = (float)(zoff + z);
        const bool z_fast = pz >= zlo && pz < zhi;
        T *dslice = dst + dbase0 + (int64_t)z * J.dst_pz;
#pragma unroll 1
        for (int r = 0; r < kTRows; ++r) {
            const int y = ty + kTY * r;
            if (y >= B.ye) continue;
            const int x = 2 * tx;
            const bool fast = z_fast && segf[y];  // uniform across the warp (one row)
            if (!fast && x >= B.xe) continue;
            T *drow = dslice + (int64_t)y * J.dst_py;
            const float4 *qn = Q + y * Gm::NX + x / G;
            const float4 n[4] = {qn[0], qn[1], qn[2], qn[3]};
            if constexpr (STAGED && INTERP == 0) {
                float2 p0, p1, pz2;
                pair_positions(n, B.pw, p0, p1, pz2);
                if (fast) {
                    const uint32_t w = pair_staged<T, G, true, false>(sm, st, cz, p0, p1, pz2, frame, wl, wh, 2);
                    store_packed<T>(drow + x, w, B.pair_ok, 2);
                } else {
                    const int nv = B.xe - x;
                    const uint32_t w = pair_staged<T, G, true, true>(sm, st, cz, p0, p1, pz2, frame, wl, wh, nv);
                    store_packed<T>(drow + x, w, B.pair_ok, nv);
                }
            } else {
                tps_pair<T, G, INTERP>(n, B, x, fast, drow);
            }
        }
    }
    // shared memory (Nd / Q) is reused by the next layer; a wait that gave up
    // on the last plane ends the unit here
    return !__syncthreads_or(tmo);
}

// Plans a staged walk over output planes [z0, z1) of the column at (Ox, Oy):
// the hull of the DF over the walk's node support gives the staged box and
// the plane window.  false when they do not fit (every thread agrees).
template <typename T, int G>
__device__ bool plan_walk(const RJob &J, int64_t Ox, int64_t Oy, int64_t z0, int64_t z1, float *red, Stage &st)
{
    using Gm = TGeom<T, G>;
    const int64_t cx0 = Ox / G, cy0 = Oy / G, cz0 = z0 / G;
    const int nzn = (int)((z1 - 1) / G - cz0) + 4;
    const int tot = Gm::NX * Gm::NY * nzn;
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = threadIdx.x; i < tot; i += kThreads) {
        const int nx = i % Gm::NX, t = i / Gm::NX;
        const int ny = t % Gm::NY, nz = t / Gm::NY;
        const int64_t gx = min(cx0 + nx, J.gsz[0] - 1), gy = min(cy0 + ny, J.gsz[1] - 1);
        const int64_t gz = min(cz0 + nz, J.gsz[2] - 1);
        const float4 d = J.nodes[(gz * J.gsz[1] + gy) * J.gsz[0] + gx];
        if (isfinite(d.x) && isfinite(d.y) && isfinite(d.z)) {
            mn[0] = fminf(mn[0], d.x); mn[1] = fminf(mn[1], d.y); mn[2] = fminf(mn[2], d.z);
            mx[0] = fmaxf(mx[0], d.x); mx[1] = fmaxf(mx[1], d.y); mx[2] = fmaxf(mx[2], d.z);
        } else {
            mn[0] = mn[1] = mn[2] = -3.4e38f;
            mx[0] = mx[1] = mx[2] = 3.4e38f;
        }
    }
    block_minmax(mn, mx, red);
    __syncthreads();  // `red` is written again by the next reduction
    for (int a = 0; a < 3; ++a)
        if (!(mn[a] > -1.0e6f && mx[a] < 1.0e6f)) return false;
    // taps of the walk, frame coordinates: x in [fx0, 63 + fx1 + 1], y in
    // [fy0, 15 + fy1 + 1], z in [z + fz0, z + fz1 + 1] for output plane z (a
    // margin of 1/64 covers the FP32 rounding of the spline)
    const float e = 1.0f / 64.0f;
    const int fx0 = (int)floorf(mn[0] - e), fx1 = (int)floorf(mx[0] + e);
    const int fy0 = (int)floorf(mn[1] - e), fy1 = (int)floorf(mx[1] + e);
    const int fz0 = (int)floorf(mn[2] - e), fz1 = (int)floorf(mx[2] + e);
    // the box's first column, in source-buffer coordinates, on a 16-byte boundary
    constexpr int A = 16 / Gm::ES;
    const int64_t xlo = Ox - J.src_o[0] + fx0;
    const int64_t xhi = Ox - J.src_o[0] + kTBX + fx1;
    const int64_t rx0 = xlo >= 0 ? (xlo / A) * A : -(((-xlo) + A - 1) / A) * A;
    if (xhi - rx0 + 1 > kBoxW) return false;
    const int rows = kTBY + fy1 - fy0 + 1;
    if (rows > kHMax) return false;
    const int a = fz0, b = fz1 + 1;
    if (b - a + 1 + kAhead > Gm::R) return false;
    const int64_t ry0 = Oy - J.src_o[1] + fy0;
    const int64_t p0 = z0 + a - J.src_o[2], p1 = z1 - 1 + b - J.src_o[2];
    const int64_t lim = (int64_t)1 << 30;  // TMA coordinates are int32
    if (rx0 < -lim || rx0 > lim || ry0 < -lim || ry0 + rows > lim || p0 < -lim || p1 > lim) return false;
    st.a = a;
    st.b = b;
    st.rx0 = (int)rx0;
    st.ry0 = (int)ry0;
    st.rows = rows;
    st.DX = (int)(Ox - J.src_o[0] - rx0);
    st.DY = -fy0;
    return true;
}

// A staged walk over output planes [z0, z1) (planned by plan_walk).
template <typename T, int G, int INTERP>
__device__ bool tps_walk(const RJob &J, int64_t Ox, int64_t Oy, int64_t z0, int64_t z1, const TSmem<T, G> &S,
                         Stage &st, uint32_t &parity, int &tmo, float *red, unsigned char *segf)
{
    using Gm = TGeom<T, G>;
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t sz0 = J.src_o[2];
    const uint32_t ring = 0;  // slots start at S.base
    // offset of frame (x, y) = (0, 0) in slot 0, minus the magic-float bias
    // of the floor bit patterns (2^32 wrap arithmetic)
    st.kxy = ring + (uint32_t)(st.DY - kMagicBits) * (uint32_t)Gm::ROW_B +
             (uint32_t)(st.DX - kMagicBits) * (uint32_t)Gm::ES;
    st.omax = ring + (uint32_t)(Gm::R * Gm::PLANE_B - Gm::ROW_B - 2 * Gm::ES);
    const int64_t first = z0 + st.a - sz0;
    st.last = z1 - 1 + st.b - sz0;
    st.waited = first - 1;
    // prologue: the first plane's window and kAhead - 1 planes beyond it
    const int64_t pro = min(st.last, z0 + st.b + kAhead - 1 - sz0);
    for (int64_t p = first; p <= pro; ++p)
        if ((tid >> 5) == 0) stage_issue<T, G>(J, S, st, p, lane);
    st.issued = pro;
    for (int64_t zf = z0; zf < z1;) {
        const int64_t ze = min(z1, (zf / G + 1) * G);
        if (!tps_layer<T, G, INTERP, true>(J, Ox, Oy, zf, (int)(ze - zf), S, st, parity, tmo, red, segf))
            return false;
        zf = ze;
    }
    return true;
}

// One work unit: output planes [z0, z1) of the column at (Ox, Oy).
template <typename T, int G, int INTERP>
__device__ bool tps_unit(const RJob &J, int64_t Ox, int64_t Oy, int64_t z0, int64_t z1, const TSmem<T, G> &S,
                         Stage &st, uint32_t &parity, int &tmo, float *red, unsigned char *segf)
{
    if (INTERP == 0 && J.tma_ok) {
        if (plan_walk<T, G>(J, Ox, Oy, z0, z1, red, st))
            return tps_walk<T, G, INTERP>(J, Ox, Oy, z0, z1, S, st, parity, tmo, red, segf);
        if ((z1 - 1) / G != z0 / G) {
            // several layers: plan each on its own
            for (int64_t zf = z0; zf < z1;) {
                const int64_t ze = min(z1, (zf / G + 1) * G);
                bool ok;
                if (plan_walk<T, G>(J, Ox, Oy, zf, ze, red, st))
                    ok = tps_walk<T, G, INTERP>(J, Ox, Oy, zf, ze, S, st, parity, tmo, red, segf);
                else
                    ok = tps_layer<T, G, INTERP, false>(J, Ox, Oy, zf, (int)(ze - zf), S, st, parity, tmo, red, segf);
                if (!ok) return false;
                zf = ze;
            }
            return true;
        }
    }
    for (int64_t zf = z0; zf < z1;) {
        const int64_t ze = min(z1, (zf / G + 1) * G);
        if (!tps_layer<T, G, INTERP, false>(J, Ox, Oy, zf, (int)(ze - zf), S, st, parity, tmo, red, segf))
            return false;
        zf = ze;
    }
    return true;
}

// ---------------------------------------------------------------- affine

constexpr int kABY = 8, kABZ = 8;

// Rows of an affine brick with the same lane-pair layout as the TPS path:
// lane l owns voxels (x, x+1), x = 2l + 64k; q = fo + M_lin l in FP32.
template <typename T, int INTERP, bool FAST>
__device__ __forceinline__ void affine_rows(const float (&m)[3][3], const float (&fo)[3], int lane, int ty, int ye,
                                            int ze, int xe, const T *base, int py32, int pz32, int64_t py, int64_t pz,
                                            const Frame &frame, const Clamp &cw, T *dbrick, int64_t dpy, int64_t dpz,
                                            bool pair_ok, const Rows<T> &rows)
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
            if constexpr (INTERP == 0) {  // packed pair path, truncation (no +0.5)
                const float lx = (float)x;
                const float2 p0 = f2(fmaf(m[0][0], lx, bx0), fmaf(m[1][0], lx, by0));
                const float2 p1 = add2(p0, f2(m[0][0], m[1][0]));
                const float qz0 = fmaf(m[2][0], lx, bz0);
                const float2 pz2 = f2(qz0, qz0 + m[2][0]);
                uint32_t w;
                if (FAST)
                    pair_fast2<T, false>(p0, p1, pz2, rows, w);
                else if (cw.clamped)
                    pair_clamped2<T, false>(p0, p1, pz2, rows, frame, cw.cl, cw.ch, xe - x, w);
                else if (cw.span32)
                    pair_checked2<T, false, int>(p0, p1, pz2, base, py32, pz32, frame, cw.cl, cw.ch, xe - x, w);
                else
                    pair_checked2<T, false, int64_t>(p0, p1, pz2, base, py, pz, frame, cw.cl, cw.ch, xe - x, w);
                store_packed<T>(drow + x, w, pair_ok, FAST ? 2 : xe - x);
            } else {
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
    const Clamp cw = make_clamp(J, frame, lo, hi);
    const Rows<T> rows = make_rows(base, py32, pz32, cw.cl, cw.span32);
    if (fast && cw.span32)  // the unchecked path addresses taps from the rows' corner
        affine_rows<T, INTERP, true>(m, fo, tx, ty, (int)ye, (int)ze, (int)xe, base, py32, pz32, J.src_py, J.src_pz,
                                     frame, cw, dst + dbase0, J.dst_py, J.dst_pz, pair_ok, rows);
    else
        affine_rows<T, INTERP, false>(m, fo, tx, ty, (int)ye, (int)ze, (int)xe, base, py32, pz32, J.src_py, J.src_pz,
                                      frame, cw, dst + dbase0, J.dst_py, J.dst_pz, pair_ok, rows);
}

// ---------------------------------------------------------------- kernels

template <typename T, int G, int INTERP>
__global__ void __launch_bounds__(kThreads, 2) k_resample_tps(const RJob *__restrict__ jobs, int njobs,
                                                               int64_t total_units, int *err)
{
    using Gm = TGeom<T, G>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ float red[6 * (kThreads / 32)];
    __shared__ unsigned char segf[kTBY];
    // ring slots first, on a 128-byte boundary (TMA destinations), then the
    // slots' mbarriers, then the node / R / Q / weight arrays
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = (128u - (raw & 127u)) & 127u;
    TSmem<T, G> S;
    S.base = smem_raw + pad;
    S.sring = raw + pad;
    S.smbar = S.sring + (uint32_t)Gm::RING_B;
    float4 *f4 = reinterpret_cast<float4 *>(S.base + Gm::RING_B + Gm::MBAR_B);
    S.Nd = f4;
    S.Qb = f4;
    S.R = f4 + Gm::UNION;
    S.W = S.R + Gm::NR;
    const int tid = threadIdx.x;
    if (tid < G) S.W[tid] = bspline_w(tid, G);
    if (tid < Gm::R) mbar_init(S.smbar + 8u * (uint32_t)tid, 1);
    if (tid == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    uint32_t parity = 0;  // bit s: parity of the next phase of slot s's mbarrier
    int tmo = 0;
    Stage st;
    st.a = st.b = st.rx0 = st.ry0 = st.rows = st.DX = st.DY = 0;
    st.issued = st.waited = st.last = 0;
    st.kxy = st.omax = 0;
    int last_job = -1;
    bool aborted = false;
    for (int64_t u = blockIdx.x; u < total_units; u += gridDim.x) {
        const int j = find_job(jobs, njobs, u);
        const RJob &J = jobs[j];
        if (INTERP == 0 && j != last_job && J.tma_ok && tid < 32)  // the descriptor was written by a copy
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&J.tmap) : "memory");
        last_job = j;
        const int64_t lu = u - J.brick_begin;
        const int64_t bx = lu % J.bricks[0], t = lu / J.bricks[0];
        const int64_t by = t % J.bricks[1], bz = t / J.bricks[1];
        const int64_t Ox = J.out_o[0] + bx * kTBX, Oy = J.out_o[1] + by * kTBY;
        const int64_t z0 = J.out_o[2] + bz * J.zs;
        const int64_t z1 = min(z0 + (int64_t)J.zs, J.out_o[2] + J.out_n[2]);
        if (!tps_unit<T, G, INTERP>(J, Ox, Oy, z0, z1, S, st, parity, tmo, red, segf)) {
            aborted = true;
            break;
        }
    }
    if (aborted && tid == 0) {
        if (err) atomicOr(err, kKernErrTimeout);
        // let the copies still in flight land (each wait bounded) before the CTA exits
        while (st.waited < st.issued) {
            const int64_t p = st.waited + 1;
            const int s = pmod(p, Gm::R);
            if (!mbar_wait(S.smbar + 8u * (uint32_t)s, (parity >> s) & 1u)) break;
            parity ^= 1u << s;
            st.waited = p;
        }
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
cudaError_t launch_tps_t(const RJob *jobs, int njobs, int64_t total, cudaStream_t st, int sms, int *err)
{
    using Gm = TGeom<T, G>;
    auto k = k_resample_tps<T, G, INTERP>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Gm::smem_bytes);
    if (e != cudaSuccess) return e;
    // two CTAs per SM need the largest shared-memory carveout
    e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, Gm::smem_bytes);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > total) grid = total;
    if (grid < 1) grid = 1;
    k<<<(unsigned)grid, kThreads, Gm::smem_bytes, st>>>(jobs, njobs, total, err);
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
cudaError_t dispatch_g(const RJob *jobs, int njobs, int64_t total, int g, cudaStream_t st, int sms, int *err)
{
    switch (g) {
    case 4: return launch_tps_t<T, 4, INTERP>(jobs, njobs, total, st, sms, err);
    case 8: return launch_tps_t<T, 8, INTERP>(jobs, njobs, total, st, sms, err);
    case 16: return launch_tps_t<T, 16, INTERP>(jobs, njobs, total, st, sms, err);
    case 32: return launch_tps_t<T, 32, INTERP>(jobs, njobs, total, st, sms, err);
    case 64: return launch_tps_t<T, 64, INTERP>(jobs, njobs, total, st, sms, err);
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
    out[0] = kTBX;
    out[1] = kTBY;
    out[2] = g;
}

cudaError_t launch_resample(const RJob *jobs_dev, int njobs, int64_t total_bricks, int dtype, int kind, int g,
                            int interp, cudaStream_t st, int sm_count, int *err)
{
    if (total_bricks <= 0) return cudaSuccess;
    if (kind == 0) {
        if (dtype == 1) return interp ? launch_affine_t<uint8_t, 1>(jobs_dev, njobs, total_bricks, st, sm_count)
                                      : launch_affine_t<uint8_t, 0>(jobs_dev, njobs, total_bricks, st, sm_count);
        return interp ? launch_affine_t<uint16_t, 1>(jobs_dev, njobs, total_bricks, st, sm_count)
                      : launch_affine_t<uint16_t, 0>(jobs_dev, njobs, total_bricks, st, sm_count);
    }
    if (dtype == 1) return interp ? dispatch_g<uint8_t, 1>(jobs_dev, njobs, total_bricks, g, st, sm_count, err)
                                  : dispatch_g<uint8_t, 0>(jobs_dev, njobs, total_bricks, g, st, sm_count, err);
    return interp ? dispatch_g<uint16_t, 1>(jobs_dev, njobs, total_bricks, g, st, sm_count, err)
                  : dispatch_g<uint16_t, 0>(jobs_dev, njobs, total_bricks, g, st, sm_count, err);
}

}  // namespace tw
