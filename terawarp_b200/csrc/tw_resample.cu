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
// global memory): a column of 64 x 16 output voxels walks down its planes,
// one warp per output row.  The cubic B-spline is evaluated separably: per
// cell layer a row warp contracts its row's nodes, taken as node' = DF +
// node position - frame origin (the B-spline reproduces linear functions, so
// the spline of node' is the sample position q itself), along y and then
// along x into four position pairs per lane; per output plane the positions
// are their z contraction -- 12 FFMA2 per voxel pair instead of 192 FMA per
// voxel.  A copy warp stages the column's source footprint in shared memory
// by TMA, plane by plane, so that the eight taps of every voxel are
// shared-memory loads (see "TPS units" below).
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
// A TPS work unit is a column of 64 x 16 output voxels (x, y) walking down a
// run of output planes: part of one control-cell layer (small jobs) or
// several whole layers.  Each cell layer is evaluated in its own frame --
// origin at the column's corner on the layer's first plane -- so a voxel's
// position and value do not depend on how the volume is cut into units or
// how units are batched.
//
// A CTA is 16 warps, one per output row of the unit; lane l owns the voxel
// pair (2l, 2l+1), so a warp covers one whole 64-voxel row.  Per cell layer a
// warp contracts the 4 x 4 x (64/G + 3) nodes of its row along y (into
// warp-private shared memory), then every lane contracts them along x for
// its voxel pair: four (one per node layer along z) position pairs P_c kept
// in registers.  Per output plane the positions are sum_c wz_c P_c (12 FFMA2
// per pair); no node data is touched and no barrier is taken.
//
// Staged walks.  The column's source footprint over a walk -- the convex
// hull of its nodes' displacements (B-spline weights are >= 0 and sum to 1)
// plus the +1 tap -- is a box of at most kBoxW x kHMax elements per source
// plane and a window of W planes that slides down one plane per output
// plane.  A planning kernel (one warp per walk) computes every walk's plan
// first and lists the walks that do not fit.  The staged kernel's CTA has
// one producer warp next to the 16 row warps: it copies the box of every
// source plane its CTA's walks read, in order, into a ring of kRing plane
// slots by TMA (cp.async.bulk.tensor, one kBoxW x kHMax box per plane, from
// this GPU's own memory; no multicast).  Each slot has a "full" mbarrier
// (transaction count of the copies) and an "empty" mbarrier (one arrival per
// row warp once no later plane of that warp reads the slot); the producer
// waits on "empty" before it reuses a slot, so copies run up to kRing - W
// planes ahead of the slowest row warp and no row warp waits for another
// except through the data.  Slot 0 is copied a second time past the last
// slot, so the z+1 tap of any plane is at a fixed offset.  A slot holds the
// box densely (row pitch kBoxW).  Units are numbered x-fastest, then y,
// then z, so the walks in flight at one time are a slab of neighbouring
// columns at the same depth: their boxes overlap in x and y and meet in L2,
// and each source plane comes from DRAM about once.  (Numbered z-fastest,
// the walks in flight were a few columns at 16 depths and the y-neighbours'
// halo rows were fetched again later: 3x the source bytes read from DRAM on
// a 1024^3 u16 job.)  A walk whose box or window does not fit, a nearest-neighbour job,
// or a source buffer TMA cannot describe gathers from global memory instead
// (the gather kernel), with the same positions and the same trilinear
// arithmetic (trilerp2).
//
// Interior walks.  The planning kernel also marks a walk "interior" when
// every tap of every voxel lies inside the subject volume and the source
// buffer and the unit lies wholly inside the output region.  Row warps then
// skip every range test: per cell layer only the node contractions, per
// output plane only positions, staged taps, lerps and one store.  Other
// walks apply the reference's range rule voxel by voxel.

constexpr int kTBX = 64;                     // unit width (x): 32 lanes x 2 voxels
constexpr int kTBY = 16;                     // unit height (y): one warp per row
constexpr int kTpsThreads = 32 * kTBY;        // gather kernel: one warp per output row
// staged kernel: output rows per row warp.  One row per warp, 16 row warps
// and the producer (17 warps, 96 registers a thread) measured 17.9 ms on the
// 2048 x 2048 x 1024 u16 job against 20.5 ms for two rows per warp (9 warps,
// 168 registers): more warps hide the dependency chains better than the
// second row's independent work does.
constexpr int kRowsPerWarp = 1;
constexpr int kRowWarps = kTBY / kRowsPerWarp;  // row warp y owns rows y + k kRowWarps
constexpr int kStagedThreads = 32 * kRowWarps + 32;  // row warps + the producer warp
constexpr int kBoxW = kStageBoxW;            // TMA box: source elements per row copy
constexpr int kHMax = kStageBoxH;            // TMA box: rows per staged plane
constexpr int kRing = 16;                    // plane slots (plus the mirror of slot 0); a power of 2
constexpr int kMinAhead = 3;                 // slots a walk's window leaves for copies in flight
static_assert((kRing & (kRing - 1)) == 0, "slot = sequence & (kRing - 1)");
// a wait on a copy or on another warp that has not ended after this long is
// an error (the kernel reports kKernErrTimeout and returns)
constexpr unsigned long long kStageWaitNs = 2000000000ull;

// A walk's staging plan (planning kernel), with the walk itself decoded
// (job, column corner, output planes) so the staged kernel's warps need no
// 64-bit divisions to find it.
struct alignas(16) Plan {
    int staged;    // 1: the walk's source footprint is staged
    int a, b;      // output plane z reads source planes [z + a, z + b]
    int rx0, ry0;  // buffer column / row of the staged box's first element
    int rows;      // staged rows per plane
    int DX, DY;    // box column / row of frame x = 0 / y = 0
    int nplanes;   // source planes staged for the walk
    int interior;  // 1: every sample of the walk is inside (no range tests)
    int j;         // job
    int ox, oy;    // global output voxel of the column's corner
    int z0, z1;    // output planes [z0, z1)
    int pad;
};

template <typename T, int G>
struct TGeom {
    static constexpr int NX = kTBX / G + 3;       // node columns of a unit (G <= 64)
    static constexpr int NRW = 4 * NX;            // y-contracted nodes of one row and layer
    static constexpr int ES = (int)sizeof(T);
    static constexpr int ROW_B = kBoxW * ES;
    static constexpr int PLANE_B = kHMax * ROW_B;
    static constexpr int RING_B = (kRing + 1) * PLANE_B;
    static constexpr int NBAR = 2 * kRing;        // full[kRing], empty[kRing]
    // ring, barriers, then the weight tables: W[G] (float4) and W2[G][2]
    // (float4 pairs (w0, w0, w1, w1), (w2, w2, w3, w3)), then the row warps'
    // nodes (two float4 per y-contracted node: the interior walks keep them
    // as duplicated pairs)
    static constexpr size_t smem_bytes =
        128 + (size_t)RING_B + 8 * NBAR + sizeof(float4) * (size_t)(3 * G + kRowWarps * 2 * NRW);
    static_assert(PLANE_B % 128 == 0, "TMA destinations are 128-byte aligned");
    static_assert((8 * NBAR) % 16 == 0 && sizeof(Plan) % 16 == 0, "the weight tables are float4-aligned");
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

__device__ __forceinline__ void mbar_arrive(uint32_t a)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
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

// try_wait with a suspend-time hint: a thread whose phase is not complete
// sleeps until it completes or about hint_ns pass, instead of returning at
// once, so a waiting warp takes almost no issue slots from the other warps
// of its SM sub-partition.
__device__ __forceinline__ bool mbar_try_sleep(uint32_t a, uint32_t parity, uint32_t hint_ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// The producer's wait for a free slot (bounded like mbar_wait_slow): it
// sleeps between tries, since it has nothing else to do meanwhile.
__device__ __forceinline__ bool mbar_wait_producer(uint32_t a, uint32_t parity, const volatile int *abort)
{
    if (mbar_try(a, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_sleep(a, parity, 20000u)) return true;
        if (*abort || globaltimer_ns() - t0 > kStageWaitNs) return false;
    }
}

// Waits for the phase of parity `parity` of the mbarrier at `a`; gives up
// (false) after kStageWaitNs, or early once another warp has given up
// (*abort set) unless `drain`.  Inlined: a call would make the hot loops
// keep registers on the stack around it.
__device__ __forceinline__ bool mbar_wait_slow(uint32_t a, uint32_t parity, const volatile int *abort, bool drain)
{
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned i = 1;; ++i) {
        if (mbar_try(a, parity)) return true;
        if ((i & 63u) == 0 && ((!drain && *abort) || globaltimer_ns() - t0 > kStageWaitNs)) return false;
    }
}

__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, const volatile int *abort)
{
    return mbar_try(a, parity) || mbar_wait_slow(a, parity, abort, false);
}

// One staged plane: the kBoxW x kHMax box at tensor coordinates (x, y, z) of
// the job's source buffer (elements outside it read as 0) into shared memory
// at dst; completion is counted on the mbarrier at mbar.
__device__ __forceinline__ void tma_plane(uint32_t dst, const CUtensorMap *map, int x, int y, int z, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(mbar)
        : "memory");
}

// Shared memory of a TPS CTA.
struct TSmem {
    unsigned char *base;  // 128-byte aligned start of the ring
    uint32_t sring;       // shared-window address of slot 0
    uint32_t sfull;       // shared-window address of full[0] (8 bytes each); empty[s] = full[s] + 8 kRing
    float4 *W;            // B-spline weights at t = i / G
    float4 *W2;           // the same as duplicated pairs: W2[2i] = (w0, w0, w1, w1), W2[2i+1] = (w2, w2, w3, w3)
    float4 *Rw;           // per row warp: y-contracted nodes of its row
    int *abort;           // set by a warp that gave up waiting
};

// Job and unit of flattened unit index u (x fastest, then y, then z: the
// units that run at the same time are a compact slab of neighbouring
// columns at the same depth, whose overlapping source footprints meet in L2).
struct Walk {
    int j;
    int64_t Ox, Oy, z0, z1;
};

__device__ __forceinline__ Walk walk_of(const RJob *jobs, int njobs, int64_t u)
{
    Walk w;
    w.j = find_job(jobs, njobs, u);
    const RJob &J = jobs[w.j];
    const int64_t lu = u - J.brick_begin;
    const int64_t bx = lu % J.bricks[0], t = lu / J.bricks[0];
    const int64_t by = t % J.bricks[1], bz = t / J.bricks[1];
    w.Ox = J.out_o[0] + bx * kTBX;
    w.Oy = J.out_o[1] + by * kTBY;
    w.z0 = J.out_o[2] + bz * J.zs;
    w.z1 = min(w.z0 + (int64_t)J.zs, J.out_o[2] + J.out_n[2]);
    return w;
}

// Warp-wide min / max of 3 components.
__device__ __forceinline__ void warp_minmax(float (&mn)[3], float (&mx)[3])
{
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
}

// Plans walk w (one warp): the hull of the DF over the walk's node support
// gives the staged box and the plane window.  staged = 0 when they do not
// fit.  Every lane returns the same plan.
template <typename T, int G>
__device__ Plan plan_walk(const RJob &J, const Walk &w)
{
    constexpr int NX = TGeom<T, G>::NX;
    constexpr int NY = (G < kTBY ? kTBY / G : 1) + 3;
    Plan P = {};
    const int lane = threadIdx.x & 31;
    const int64_t cx0 = w.Ox / G, cy0 = w.Oy / G, cz0 = w.z0 / G;
    const int nzn = (int)((w.z1 - 1) / G - cz0) + 4;
    const int tot = NX * NY * nzn;
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = lane; i < tot; i += 32) {
        const int nx = i % NX, t = i / NX;
        const int ny = t % NY, nz = t / NY;
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
    warp_minmax(mn, mx);
    for (int a = 0; a < 3; ++a)
        if (!(mn[a] > -1.0e6f && mx[a] < 1.0e6f)) return P;
    // taps of the walk, frame coordinates: x in [fx0, 63 + fx1 + 1], y in
    // [fy0, 15 + fy1 + 1], z in [z + fz0, z + fz1 + 1] for output plane z (a
    // margin of 1/64 covers the FP32 rounding of the spline)
    const float e = 1.0f / 64.0f;
    const int fx0 = (int)floorf(mn[0] - e), fx1 = (int)floorf(mx[0] + e);
    const int fy0 = (int)floorf(mn[1] - e), fy1 = (int)floorf(mx[1] + e);
    const int fz0 = (int)floorf(mn[2] - e), fz1 = (int)floorf(mx[2] + e);
    // the box's first column, in source-buffer coordinates, on a 16-byte boundary
    constexpr int A = 16 / (int)sizeof(T);
    const int64_t xlo = w.Ox - J.src_o[0] + fx0;
    const int64_t xhi = w.Ox - J.src_o[0] + kTBX + fx1;
    const int64_t rx0 = xlo >= 0 ? (xlo / A) * A : -(((-xlo) + A - 1) / A) * A;
    if (xhi - rx0 + 1 > kBoxW) return P;
    const int rows = kTBY + fy1 - fy0 + 1;
    if (rows > kHMax) return P;
    const int a = fz0, b = fz1 + 1;
    if (b - a + 1 + kMinAhead > kRing) return P;
    const int64_t ry0 = w.Oy - J.src_o[1] + fy0;
    const int64_t p0 = w.z0 + a - J.src_o[2], p1 = w.z1 - 1 + b - J.src_o[2];
    const int64_t lim = (int64_t)1 << 30;  // TMA coordinates and the plan's coordinates are int32
    if (rx0 < -lim || rx0 > lim || ry0 < -lim || ry0 + rows > lim || p0 < -lim || p1 > lim) return P;
    if (w.Ox > lim || w.Oy > lim || w.z1 > lim) return P;
    // staged walks index the node grid with 32 bits
    if (J.gsz[0] * J.gsz[1] * J.gsz[2] >= ((int64_t)1 << 31)) return P;
    P.staged = 1;
    P.a = a;
    P.b = b;
    P.rx0 = (int)rx0;
    P.ry0 = (int)ry0;
    P.rows = rows;
    P.DX = (int)(w.Ox - J.src_o[0] - rx0);
    P.DY = -fy0;
    P.nplanes = (int)(w.z1 - w.z0) + b - a;
    P.j = w.j;
    P.ox = (int)w.Ox;
    P.oy = (int)w.Oy;
    P.z0 = (int)w.z0;
    P.z1 = (int)w.z1;
    // interior: the unit lies wholly inside the output region, its voxel
    // pairs can be stored as one word each, and every sample q (with the
    // margin) has 0 <= floor(q) and floor(q) + 1 <= sz - 1 inside both the
    // subject volume and the source buffer, so no range test can fail
    const int64_t pe[3] = {w.Ox + kTBX - 1, w.Oy + kTBY - 1, w.z1 - 1};
    const int64_t ps[3] = {w.Ox, w.Oy, w.z0};
    bool in = w.Ox + kTBX <= J.out_o[0] + J.out_n[0] && w.Oy + kTBY <= J.out_o[1] + J.out_n[1];
    in = in && ((uintptr_t)J.dst) % (2 * sizeof(T)) == 0 && J.dst_py % 2 == 0 && J.dst_pz % 2 == 0;
    for (int ax = 0; ax < 3; ++ax) {
        const double lo = (double)ps[ax] + (double)mn[ax] - (double)e;
        const double hi = (double)pe[ax] + (double)mx[ax] + (double)e;
        const double vlo = (double)max((int64_t)0, J.src_o[ax]);
        const double vhi = (double)min(J.glob[ax] - 1, J.src_o[ax] + J.src_n[ax] - 1);
        in = in && lo >= vlo && hi < vhi;
    }
    P.interior = in ? 1 : 0;
    return P;
}

// The staged kernel runs in two launches: MODE 0 takes the interior walks,
// MODE 1 the other staged walks (the reference's range rule as a mask).
// Each launch strides over its own list of walks, in unit order, which
// k_tps_lists builds: strided over all units, the CTAs met the border walks
// unevenly (148 CTAs and 32 columns per row of a 2048-wide job share the
// factor 4, so half the CTAs took every x-face walk), and the launch waited
// for the busiest CTA.
// A walk list: n at [0], then the unit indices.
__device__ __forceinline__ int list_count(const int *list) { return list[0]; }

// Ring barriers come in plane pairs: planes 2p and 2p + 1 (sequence numbers)
// share the "full" and "empty" mbarriers of pair slot p & (kPairs - 1), so a
// row warp waits and releases once per two planes.
constexpr int kPairs = kRing / 2;

__device__ __forceinline__ uint32_t full_bar(const TSmem &S, uint32_t pair)
{
    return S.sfull + 8u * (pair & (uint32_t)(kPairs - 1));
}

__device__ __forceinline__ uint32_t empty_bar(const TSmem &S, uint32_t pair)
{
    return S.sfull + 8u * (kRing + (pair & (uint32_t)(kPairs - 1)));
}

// The producer (lane 0 of the producer warp): copies every source plane of
// the CTA's staged walks, in walk order, into the ring; plane sequence s
// goes to slot s & (kRing - 1) and completes on the "full" barrier of its
// pair s / 2 (two arrivals per phase, one per plane, with the planes'
// bytes).  Before it reuses a pair slot it waits for the slot's "empty"
// phase: every row warp's reads of the two planes before happen before its
// arrival there (a release), which the wait observes (an acquire) before the
// asynchronous writes.  seq returns the number of planes issued; false if a
// wait gave up (or another warp did).
template <typename T, int G>
__device__ bool produce(const RJob *__restrict__ jobs, const int *__restrict__ list, const Plan *__restrict__ plans,
                        const TSmem &S, uint32_t &seq)
{
    using Gm = TGeom<T, G>;
    seq = 0;
    int last_job = -1;
    const int n = list_count(list);
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const Plan P = plans[list[1 + i]];
        const RJob &J = jobs[P.j];
        if (P.j != last_job) {  // the descriptor was written by a copy
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&J.tmap) : "memory");
            last_job = P.j;
        }
        const int pfirst = (int)((int64_t)P.z0 + P.a - J.src_o[2]);
        for (int i = 0; i < P.nplanes; ++i, ++seq) {
            const uint32_t slot = seq & (uint32_t)(kRing - 1), pair = seq >> 1;
            const uint32_t full = full_bar(S, pair);
            if ((seq & 1u) == 0 && pair >= (uint32_t)kPairs &&
                !mbar_wait_producer(empty_bar(S, pair), ((pair / kPairs) - 1u) & 1u, S.abort))
                return false;
            mbar_expect_tx(full, (uint32_t)(slot == 0 ? 2 : 1) * (uint32_t)Gm::PLANE_B);
            const uint32_t d = S.sring + slot * (uint32_t)Gm::PLANE_B;
            tma_plane(d, &J.tmap, P.rx0, P.ry0, pfirst + i, full);
            if (slot == 0) tma_plane(d + (uint32_t)(kRing * Gm::PLANE_B), &J.tmap, P.rx0, P.ry0, pfirst + i, full);
        }
    }
    return true;
}

// The producer on its way out.  An odd number of planes leaves the last
// pair's barrier one arrival short: it gets a plain arrival, so the phase
// completes once the copy lands.  Then every copy issued has landed before
// the CTA exits (the row warps waited for all of them unless a wait gave
// up; bounded waits).
__device__ void drain_copies(const TSmem &S, uint32_t seq)
{
    if (seq & 1u) mbar_arrive(full_bar(S, seq >> 1));
    const uint32_t npairs = (seq + 1u) >> 1;
    const uint32_t n0 = npairs > (uint32_t)kPairs ? npairs - kPairs : 0u;
    for (uint32_t n = n0; n < npairs; ++n)
        if (!mbar_try(full_bar(S, n), (n / kPairs) & 1u))
            mbar_wait_slow(full_bar(S, n), (n / kPairs) & 1u, S.abort, true);
}

// A row warp's place in the ring: the next plane pair to wait for and the
// next plane sequence to release.  A walk's planes are consecutive
// sequences, so at the start of a walk rseq = the sequence of its first
// plane.
struct RingPos {
    uint32_t wpair, rseq;
};

// Waits (bounded) for the planes before sequence `need` (their pairs);
// false if a wait gave up.  Every lane waits; the outcome is made uniform
// across the warp.
__device__ __forceinline__ bool wait_planes(const TSmem &S, RingPos &R, uint32_t need)
{
    const uint32_t last = (need - 1u) >> 1;  // the pair of plane need - 1
    for (; R.wpair <= last; ++R.wpair) {
        const bool ok = mbar_wait(full_bar(S, R.wpair), (R.wpair / kPairs) & 1u, S.abort);
        if (!__all_sync(0xffffffffu, ok)) return false;
    }
    return true;
}

// Releases the oldest plane the warp holds.  When it is the second plane of
// its pair, every lane arrives on the pair's "empty" barrier (32 arrivals
// per row warp), each arrival a release of that lane's reads of both planes.
__device__ __forceinline__ void release_plane(const TSmem &S, RingPos &R)
{
    if (R.rseq & 1u) mbar_arrive(empty_bar(S, R.rseq >> 1));
    ++R.rseq;
}

// Releases the two oldest planes the warp holds, s and s + 1, without a
// test of their parity: whichever of them is the second plane of its pair
// completes pair s / 2 (planes s, s + 1 when s is even; s - 1, released
// before, and s when s is odd), and every lane arrives on that pair's
// "empty" barrier.  A pair is completed by exactly one release, single or
// double, so each lane arrives once per pair.
__device__ __forceinline__ void release_two_planes(const TSmem &S, RingPos &R)
{
    mbar_arrive(empty_bar(S, R.rseq >> 1));
    R.rseq += 2;
}

// The row warps' state of one cell layer (uniform across the warp except
// the position pairs).
struct RowLayer {
    float2 P[4][3];   // per node layer c: (x, y) of voxel 0, (x, y) of voxel 1, (z0, z1)
    float mn[3], mx[3];  // the row's sample hull over the layer (frame coordinates)
    float zlo, zhi;   // a plane at frame z pz is unchecked in z when zlo <= pz < zhi
    bool row_fast;    // the row is unchecked in x and y
};

// Layer setup of row warp `y` of the unit at (Ox, Oy), layer frame origin
// Oz: y-contraction of the row's nodes into Rw, x-contraction into the
// lane's position pairs, and the row's sample hull.
template <typename T, int G>
__device__ __forceinline__ void row_layer(const RJob &J, int64_t Ox, int64_t Oy, int64_t Oz, int zoff, int zn, int y,
                                          int xe, const float4 *W, float4 *Rw, const float4 (&wx)[2], RowLayer &L)
{
    using Gm = TGeom<T, G>;
    const int lane = threadIdx.x & 31;
    const int64_t O[3] = {Ox, Oy, Oz};
    const int64_t c0[3] = {Ox / G, Oy / G, Oz / G};
    const int yy = (int)(Oy - c0[1] * G) + y;
    const int cyb = yy / G;
    const float4 wy = W[yy % G];
    __syncwarp();  // every lane is done with the previous layer's Rw
    // R[c][nx] = sum_b wy_b node'[c][cyb + b][nx], node' = DF + node position - O
    for (int i = lane; i < Gm::NRW; i += 32) {
        const int c = i / Gm::NX, nx = i % Gm::NX;
        const int64_t gx = min(c0[0] + nx, J.gsz[0] - 1), gz = min(c0[2] + c, J.gsz[2] - 1);
        // node g sits at (g-1)*G; relative to O that is exact in float
        const float ox = (float)((gx - 1) * G - O[0]), oz = (float)((gz - 1) * G - O[2]);
        float4 v[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int64_t gy = min(c0[1] + cyb + b, J.gsz[1] - 1);
            const float4 d = J.nodes[(gz * J.gsz[1] + gy) * J.gsz[0] + gx];
            v[b] = make_float4(d.x + ox, d.y + (float)((gy - 1) * G - O[1]), d.z + oz, 0.f);
        }
        float4 r;
        r.x = fmaf(wy.x, v[0].x, fmaf(wy.y, v[1].x, fmaf(wy.z, v[2].x, wy.w * v[3].x)));
        r.y = fmaf(wy.x, v[0].y, fmaf(wy.y, v[1].y, fmaf(wy.z, v[2].y, wy.w * v[3].y)));
        r.z = fmaf(wy.x, v[0].z, fmaf(wy.y, v[1].z, fmaf(wy.z, v[2].z, wy.w * v[3].z)));
        r.w = 0.f;
        Rw[i] = r;
    }
    __syncwarp();
    // x-contraction for the lane's voxel pair (2 lane, 2 lane + 1: one cell)
    const int xn = (2 * lane) / G;
    float dmn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, dmx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    bool fin = true;
    const float x0 = (float)(2 * lane), fy = (float)y;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float2 p0 = f2(0.f, 0.f), p1 = p0, pz = p0;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const float4 n = Rw[c * Gm::NX + xn + a];
            const float w0 = (&wx[0].x)[a], w1 = (&wx[1].x)[a];
            p0 = fma2(f2(w0, w0), f2(n.x, n.y), p0);
            p1 = fma2(f2(w1, w1), f2(n.x, n.y), p1);
            pz = fma2(f2(w0, w1), f2(n.z, n.z), pz);
        }
        L.P[c][0] = p0;
        L.P[c][1] = p1;
        L.P[c][2] = pz;
        // displacement part (the spline of the node positions is the voxel
        // position; node layer c sits at frame z (c - 1) G)
        const float zc = (float)((c - 1) * G);
        const float d[6] = {p0.x - x0, p1.x - (x0 + 1.f), p0.y - fy, p1.y - fy, pz.x - zc, pz.y - zc};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            fin = fin && isfinite(d[k]);
            dmn[k >> 1] = fminf(dmn[k >> 1], d[k]);
            dmx[k >> 1] = fmaxf(dmx[k >> 1], d[k]);
        }
    }
    warp_minmax(dmn, dmx);
    if (!__all_sync(0xffffffffu, fin))
        for (int a = 0; a < 3; ++a) {
            dmn[a] = -3.4e38f;
            dmx[a] = 3.4e38f;
        }
    // sample hull of the row over the layer's planes (frame coordinates)
    const float plo[3] = {0.f, fy, (float)zoff};
    const float phi[3] = {(float)(kTBX - 1), fy, (float)(zoff + zn - 1)};
    float *mn = L.mn, *mx = L.mx;
    for (int a = 0; a < 3; ++a) {
        mn[a] = dmn[a] <= -3.0e38f ? -3.4e38f : plo[a] + dmn[a];
        mx[a] = dmx[a] >= 3.0e38f ? 3.4e38f : phi[a] + dmx[a];
    }
    const Frame frame = make_frame(J, O);
    const bool span_ok = offsets_fit_32(J, L.mn, L.mx);
    const Clamp cw = make_clamp(J, frame, L.mn, L.mx);
    // unchecked-path bounds per axis: every tap of a sample q with
    // lb <= q < hb lies inside the volume and the source buffer
    float lb[3], hb[3];
    for (int a = 0; a < 3; ++a) {
        lb[a] = fmaxf(frame.lo[a], (float)frame.bl[a]) + 1.0f / 64.0f;
        hb[a] = fminf(frame.hi[a], (float)frame.bh[a]) - 1.0f / 64.0f;
    }
    L.row_fast = span_ok && cw.span32 && (kTBX <= xe) && mn[0] >= lb[0] && mx[0] < hb[0] && mn[1] >= lb[1] &&
                 mx[1] < hb[1];
    L.zlo = lb[2] - dmn[2];
    L.zhi = hb[2] - dmx[2];
}

// Positions of the lane's voxel pair on a plane with z weights wz.
__device__ __forceinline__ void plane_positions(const RowLayer &L, float4 wz, float2 &p0, float2 &p1, float2 &pz)
{
    const float2 w0 = f2(wz.x, wz.x), w1 = f2(wz.y, wz.y), w2 = f2(wz.z, wz.z), w3 = f2(wz.w, wz.w);
    p0 = fma2(w0, L.P[0][0], fma2(w1, L.P[1][0], fma2(w2, L.P[2][0], fma2(w3, L.P[3][0], f2(0.f, 0.f)))));
    p1 = fma2(w0, L.P[0][1], fma2(w1, L.P[1][1], fma2(w2, L.P[2][1], fma2(w3, L.P[3][1], f2(0.f, 0.f)))));
    pz = fma2(w0, L.P[0][2], fma2(w1, L.P[1][2], fma2(w2, L.P[2][2], fma2(w3, L.P[3][2], f2(0.f, 0.f)))));
}

// Offset (from the ring base) of the (x, y, z) = floor tap of a staged
// sample: the in-plane byte offset comes as the magic float kMagic + offset
// (exact for offsets below 2^22 in magnitude, and every tap of the staged
// window is), the slot from the z floor's magic bit pattern; cz maps a tap
// plane to its plane sequence (mod kRing: the slot).  Clamped so that all 8
// taps stay in the ring whatever the position (an out-of-range or NaN
// position gives some offset in the ring, for a sample whose value the
// range rule discards).
template <typename T>
__device__ __forceinline__ uint32_t staged_off(uint32_t omax, uint32_t cz, float mz, float mxy)
{
    constexpr uint32_t PLANE_B = kHMax * kBoxW * sizeof(T);
    const uint32_t slot = (__float_as_uint(mz) + cz) & (uint32_t)(kRing - 1);
    const uint32_t o = slot * PLANE_B + (__float_as_uint(mxy) - (uint32_t)kMagicBits);
    return min(o, omax);
}

// cz of staged_off for the cell layer with frame origin Oz of a walk whose
// first plane (output plane z0 + a) has sequence seq0: the source plane
// Oz + iz has sequence seq0 + (Oz + iz) - (z0 + a), and the magic floor's
// bit pattern of iz is kMagicBits + iz (2^32 wrap arithmetic).
__device__ __forceinline__ uint32_t layer_cz(uint32_t seq0, int64_t Oz, int64_t z0, int a)
{
    return seq0 + (uint32_t)(Oz - z0) - (uint32_t)a - (uint32_t)kMagicBits;
}

// A voxel pair of an interior walk from the staged planes, in three steps
// so that a plane's address arithmetic can overlap the previous plane's
// loads: positions as (voxel 0, voxel 1) pairs per axis give the fractions
// and the two floor taps' addresses (prep), the eight taps of both voxels
// are loaded (taps), and the trilinear value is rounded and packed
// (finish).  No range tests: every tap is inside the staged window.  The
// same floors, fractions and trilinear arithmetic (trilerp2) as the gather
// kernel's samplers.
struct PairPrep {
    float2 fx, fy, fz;
    uint32_t a0, a1;  // shared-window addresses of the floor taps of voxel 0 / 1 in the ring
};

// ring: shared-window address of slot 0; kc = kMagic + the byte offset of
// frame (0, 0) in a plane slot.  The floors are integers below 2^22 in
// magnitude, so fly ROW_B + flx ES + kc is exact whenever the tap lies in
// the staged window.
template <typename T>
__device__ __forceinline__ PairPrep prep_pair(uint32_t ring, float kc, uint32_t omax, uint32_t cz, float2 px,
                                              float2 py, float2 pz)
{
    constexpr float ROW_B = (float)(kBoxW * sizeof(T)), ES = (float)sizeof(T);
    const float2 MM = f2(kMagic, kMagic);
    const float2 mx = __fadd2_rd(px, MM), my = __fadd2_rd(py, MM), mz = __fadd2_rd(pz, MM);
    const float2 flx = sub2(mx, MM), fly = sub2(my, MM);
    PairPrep q;
    q.fx = sub2(px, flx);
    q.fy = sub2(py, fly);
    q.fz = sub2(pz, sub2(mz, MM));
    const float2 mxy = fma2(fly, f2(ROW_B, ROW_B), fma2(flx, f2(ES, ES), f2(kc, kc)));
    q.a0 = ring + staged_off<T>(omax, cz, mz.x, mxy.x);
    q.a1 = ring + staged_off<T>(omax, cz, mz.y, mxy.y);
    return q;
}

// Magic float 2^23 + v of the staged voxel at shared-window address a + OFF:
// a 32-bit address with the constant offset folded into the load.  Volatile,
// so it stays after the wait for its plane.
template <typename T, int OFF>
__device__ __forceinline__ float lds_mag(uint32_t a)
{
    uint32_t v;
    if (sizeof(T) == 2) asm volatile("ld.shared.u16 %0, [%1+%2];" : "=r"(v) : "r"(a), "n"(OFF));
    else asm volatile("ld.shared.u8 %0, [%1+%2];" : "=r"(v) : "r"(a), "n"(OFF));
    return __int_as_float(0x4B000000 | (int)v);
}

// The eight taps of both voxels as magic floats: constant row, plane and
// element offsets from each voxel's floor tap.
template <typename T>
__device__ __forceinline__ void taps_pair(const PairPrep &q, float2 (&lo)[4], float2 (&hi)[4])
{
    constexpr int ES = sizeof(T), ROW_B = kBoxW * ES, PLANE_B = kHMax * ROW_B;
    lo[0] = f2(lds_mag<T, 0>(q.a0), lds_mag<T, 0>(q.a1));
    hi[0] = f2(lds_mag<T, ES>(q.a0), lds_mag<T, ES>(q.a1));
    lo[1] = f2(lds_mag<T, ROW_B>(q.a0), lds_mag<T, ROW_B>(q.a1));
    hi[1] = f2(lds_mag<T, ROW_B + ES>(q.a0), lds_mag<T, ROW_B + ES>(q.a1));
    lo[2] = f2(lds_mag<T, PLANE_B>(q.a0), lds_mag<T, PLANE_B>(q.a1));
    hi[2] = f2(lds_mag<T, PLANE_B + ES>(q.a0), lds_mag<T, PLANE_B + ES>(q.a1));
    lo[3] = f2(lds_mag<T, PLANE_B + ROW_B>(q.a0), lds_mag<T, PLANE_B + ROW_B>(q.a1));
    hi[3] = f2(lds_mag<T, PLANE_B + ROW_B + ES>(q.a0), lds_mag<T, PLANE_B + ROW_B + ES>(q.a1));
}

template <typename T>
__device__ __forceinline__ uint32_t finish_pair(const PairPrep &q, const float2 (&lo)[4], const float2 (&hi)[4])
{
    const float2 t = out_pair<T, true>(trilerp2(lo, hi, q.fx, q.fy, q.fz));
    return pack_pair<T>(__float_as_uint(t.x), __float_as_uint(t.y));
}

// Cell-layer set-up of row warp y of a staged walk: the y contraction of
// the row's nodes into Rw, then the lane's x contraction into position pairs
// per node layer c: PX[c] = (x of voxel 0, x of voxel 1), PY[c], PZ[c]
// likewise.  Same operations and order as row_layer (the gather kernel), so
// a voxel's position does not depend on which path sampled it.
template <typename T, int G>
__device__ __forceinline__ void layer_positions(const RJob &J, int64_t Ox, int64_t Oy, int64_t Oz, int y,
                                                const float4 *W, float4 *Rw, const float4 (&wx)[2], float2 (&PX)[4],
                                                float2 (&PY)[4], float2 (&PZ)[4])
{
    using Gm = TGeom<T, G>;
    const int lane = threadIdx.x & 31;
    // staged walks have int32 coordinates and node indices (the planning
    // kernel stages a walk only when its coordinates are below 2^30 and the
    // node grid below 2^31 nodes)
    const int ox0 = (int)Ox, oy0 = (int)Oy, oz0 = (int)Oz;
    const int c0[3] = {ox0 / G, oy0 / G, oz0 / G};
    const int gs0 = (int)J.gsz[0], gs1 = (int)J.gsz[1], gs2 = (int)J.gsz[2];
    const int yy = oy0 - c0[1] * G + y;
    const int cyb = yy / G;
    const float4 wy = W[yy % G];
    __syncwarp();  // every lane is done with the previous layer's Rw
    for (int i = lane; i < Gm::NRW; i += 32) {
        const int c = i / Gm::NX, nx = i % Gm::NX;
        const int gx = min(c0[0] + nx, gs0 - 1), gz = min(c0[2] + c, gs2 - 1);
        const float ox = (float)((gx - 1) * G - ox0), oz = (float)((gz - 1) * G - oz0);
        const float4 *np = J.nodes + ((uint32_t)gz * (uint32_t)gs1 * (uint32_t)gs0 + (uint32_t)gx);
        float4 v[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int gy = min(c0[1] + cyb + b, gs1 - 1);
            const float4 d = np[(uint32_t)gy * (uint32_t)gs0];
            v[b] = make_float4(d.x + ox, d.y + (float)((gy - 1) * G - oy0), d.z + oz, 0.f);
        }
        const float rx = fmaf(wy.x, v[0].x, fmaf(wy.y, v[1].x, fmaf(wy.z, v[2].x, wy.w * v[3].x)));
        const float ry = fmaf(wy.x, v[0].y, fmaf(wy.y, v[1].y, fmaf(wy.z, v[2].y, wy.w * v[3].y)));
        const float rz = fmaf(wy.x, v[0].z, fmaf(wy.y, v[1].z, fmaf(wy.z, v[2].z, wy.w * v[3].z)));
        // duplicated pairs: (x, x, y, y), (z, z, -, -) are FP32x2 operands as loaded
        Rw[2 * i] = make_float4(rx, rx, ry, ry);
        Rw[2 * i + 1] = make_float4(rz, rz, 0.f, 0.f);
    }
    __syncwarp();
    const int xn = (2 * lane) / G;
    float2 w[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) w[a] = f2((&wx[0].x)[a], (&wx[1].x)[a]);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float2 px = f2(0.f, 0.f), py = px, pz = px;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const float4 n = Rw[2 * (c * Gm::NX + xn + a)], m = Rw[2 * (c * Gm::NX + xn + a) + 1];
            px = fma2(w[a], f2(n.x, n.y), px);
            py = fma2(w[a], f2(n.z, n.w), py);
            pz = fma2(w[a], f2(m.x, m.y), pz);
        }
        PX[c] = px;
        PY[c] = py;
        PZ[c] = pz;
    }
}


// Global-memory sampling state of a row warp's layer (every path but the staged one).
template <typename T>
struct Gather {
    const T *base;   // source element at the frame origin (may lie outside the buffer)
    int py32, pz32;  // pitches as int (valid when the layer's offsets fit int32)
    int64_t py, pz;
    Rows<T> rows;
};

// A voxel pair gathered from global memory.
template <typename T, int INTERP>
__device__ __forceinline__ void gathered_pair(float2 p0, float2 p1, float2 pz2, const Frame &frame, const Clamp &cw,
                                              const Gather<T> &g, bool fast, int nv, bool pair_ok, T *dp)
{
    if constexpr (INTERP == 0) {
        uint32_t w;
        if (fast)
            pair_fast2<T, true>(p0, p1, pz2, g.rows, w);
        else if (cw.clamped)
            pair_clamped2<T, true>(p0, p1, pz2, g.rows, frame, cw.cl, cw.ch, nv, w);
        else if (cw.span32)
            pair_checked2<T, true, int>(p0, p1, pz2, g.base, g.py32, g.pz32, frame, cw.cl, cw.ch, nv, w);
        else
            pair_checked2<T, true, int64_t>(p0, p1, pz2, g.base, g.py, g.pz, frame, cw.cl, cw.ch, nv, w);
        store_packed<T>(dp, w, pair_ok, fast ? 2 : nv);
    } else {
        const float q[2][3] = {{p0.x, p0.y, pz2.x}, {p1.x, p1.y, pz2.y}};
        uint32_t outv[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            float v;
            if (fast) {
                v = sample_fast<T, INTERP>(g.base, g.py32, g.pz32, q[j][0], q[j][1], q[j][2]);
                outv[j] = (uint32_t)v;
            } else {
                const bool ok = j < nv && sample_checked<T, INTERP>(g.base, g.py, g.pz, frame, q[j][0], q[j][1],
                                                                   q[j][2], v);
                outv[j] = ok ? (uint32_t)v : 0u;
            }
        }
        store_pair<T>(dp, outv[0], outv[1], pair_ok, fast ? 2 : nv);
    }
}

// Positions of a voxel pair on a plane: sum over node layers c of the z
// weight pairs W2 times the layer's x/y-contracted position pairs (the
// order of row_layer's plane_positions, so both paths agree bit for bit).
__device__ __forceinline__ void pair_positions(const float2 (&w)[4], const float2 (&PX)[4], const float2 (&PY)[4],
                                               const float2 (&PZ)[4], float2 &px, float2 &py, float2 &pz)
{
    const float2 Z2 = f2(0.f, 0.f);
    px = fma2(w[0], PX[0], fma2(w[1], PX[1], fma2(w[2], PX[2], fma2(w[3], PX[3], Z2))));
    py = fma2(w[0], PY[0], fma2(w[1], PY[1], fma2(w[2], PY[2], fma2(w[3], PY[3], Z2))));
    pz = fma2(w[0], PZ[0], fma2(w[1], PZ[1], fma2(w[2], PZ[2], fma2(w[3], PZ[3], Z2))));
}

// Row warp y's part of a staged walk: rows y + k kRowWarps (k <
// kRowsPerWarp), whose voxel pairs are independent work for the lane.  Per
// output plane z it waits for the planes up to z + b, samples, stores, and
// releases plane z + a, which no later plane of the walk reads; the
// fractions and tap addresses of a plane are computed during the plane
// before it (they need no staged data), so that their arithmetic overlaps
// the previous plane's loads.
//
// An interior walk (BORDER false: every sample inside, whole rows, paired
// stores) runs no range test.  Any other staged walk (one that reaches the
// volume's or the source buffer's faces, or a partial unit) runs the same
// arithmetic, then the reference's range rule as a mask (a sample with any
// q outside [0, sz - 1] writes 0), and stores only inside the output
// region.  This gives the checked sample's bits for every voxel:
//  - the staged window holds the floor tap and the +1 tap of every sample of
//    the walk, zero-filled where it reaches past the source, and a tap
//    offset is clamped into the ring whatever the position, so no position
//    reads outside shared memory;
//  - a valid sample's taps are inside the volume and the source buffer, but
//    for q = sz - 1 exactly, whose +1 tap has weight 0 (lo + 0 (hi - lo) =
//    lo exactly, as the clamped floor sz - 2 with fraction 1 gives hi);
//  - an invalid sample (NaN included: every comparison fails) is masked.
// false if a wait gave up.
template <typename T, int G, bool BORDER>
__device__ bool walk_rows(const RJob &J, const Walk &w, const Plan &P, const TSmem &S, float4 *Rw,
                          const float4 (&wx)[2], RingPos &R)
{
    using Gm = TGeom<T, G>;
    constexpr int NR = kRowsPerWarp;
    constexpr uint32_t M0 = sizeof(T) == 2 ? 0xFFFFu : 0xFFu;
    constexpr uint32_t M1 = sizeof(T) == 2 ? 0xFFFF0000u : 0xFF00u;
    const int y = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x = 2 * lane;
    const uint32_t seq0 = R.rseq;   // sequence of the walk's first plane
    const uint32_t Wn = (uint32_t)(P.b - P.a + 1);  // planes of a window
    T *dp = static_cast<T *>(J.dst) +
            ((w.z0 - J.out_o[2]) * J.dst_pz + (w.Oy + y - J.out_o[1]) * J.dst_py + (w.Ox - J.out_o[0])) + x;
    const int64_t dpz = J.dst_pz, drow2 = kRowWarps * J.dst_py;
    // border walks: rows inside the output region (uniform across the warp),
    // the lane's valid voxels, whether a pair can be stored as one word
    bool rowv[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) rowv[k] = !BORDER || (int64_t)(y + k * kRowWarps) < J.out_o[1] + J.out_n[1] - w.Oy;
    const int xe = BORDER ? (int)min(J.out_o[0] + J.out_n[0] - w.Ox, (int64_t)kTBX) : kTBX;
    const bool pair_ok =
        !BORDER || ((((uintptr_t)J.dst) % (2 * sizeof(T))) == 0 && (J.dst_py % 2 == 0) && (J.dst_pz % 2 == 0));
    // kMagic + the byte offset of frame (0, 0) in a plane slot (an integer
    // below 2^14: exact)
    const float kc = kMagic + (float)(P.DY * Gm::ROW_B + P.DX * Gm::ES);
    const uint32_t omax = (uint32_t)(kRing * Gm::PLANE_B - Gm::ROW_B - 2 * Gm::ES);
    for (int64_t zf = w.z0; zf < w.z1;) {
        const int64_t ze = min(w.z1, (zf / G + 1) * G);
        const int64_t Oz = (zf / G) * G;
        const int zoff = (int)(zf - Oz), zend = (int)(ze - Oz);
        float2 PX[NR][4], PY[NR][4], PZ[NR][4];
#pragma unroll
        for (int k = 0; k < NR; ++k)
            if (rowv[k])
                layer_positions<T, G>(J, w.Ox, w.Oy, Oz, y + k * kRowWarps, S.W, Rw, wx, PX[k], PY[k], PZ[k]);
        Frame fr;  // valid samples: lo <= q <= hi per axis (frame coordinates)
        if (BORDER) {
            const int64_t O[3] = {w.Ox, w.Oy, Oz};
            fr = make_frame(J, O);
        }
        const uint32_t cz = layer_cz(seq0, Oz, w.z0, P.a);
        auto prep = [&](int p, PairPrep (&q)[NR], uint32_t (&keep)[NR]) {
            const float4 wa = S.W2[2 * p], wb = S.W2[2 * p + 1];
            const float2 wz[4] = {f2(wa.x, wa.y), f2(wa.z, wa.w), f2(wb.x, wb.y), f2(wb.z, wb.w)};
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                float2 px, py, pz;
                pair_positions(wz, PX[k], PY[k], PZ[k], px, py, pz);
                q[k] = prep_pair<T>(S.sring, kc, omax, cz, px, py, pz);
                if (BORDER) {
                    const bool ok0 = px.x >= fr.lo[0] && px.x <= fr.hi[0] && py.x >= fr.lo[1] && py.x <= fr.hi[1] &&
                                     pz.x >= fr.lo[2] && pz.x <= fr.hi[2];
                    const bool ok1 = px.y >= fr.lo[0] && px.y <= fr.hi[0] && py.y >= fr.lo[1] && py.y <= fr.hi[1] &&
                                     pz.y >= fr.lo[2] && pz.y <= fr.hi[2];
                    keep[k] = (ok0 ? M0 : 0u) | (ok1 ? M1 : 0u);
                }
            }
        };
        PairPrep q[NR];
        uint32_t keep[NR];
        prep(zoff, q, keep);
        // sequence past the last plane output plane Oz + pz reads
        uint32_t need = seq0 + (uint32_t)(zf - w.z0) + Wn;
        // one output plane, its planes already waited for
        auto plane = [&](int pz) {
            float2 lo[NR][4], hi[NR][4];
#pragma unroll
            for (int k = 0; k < NR; ++k) taps_pair<T>(q[k], lo[k], hi[k]);
            PairPrep nq[NR];
            uint32_t nkeep[NR];
            prep(min(pz + 1, G - 1), nq, nkeep);  // (the last plane's is not used)
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                const uint32_t v = finish_pair<T>(q[k], lo[k], hi[k]);
                if (!BORDER) {
                    if (sizeof(T) == 2) *reinterpret_cast<uint32_t *>(dp + k * drow2) = v;
                    else *reinterpret_cast<uint16_t *>(dp + k * drow2) = (uint16_t)v;
                } else if (rowv[k] && x < xe) {
                    store_packed<T>(dp + k * drow2, v & keep[k], pair_ok, xe - x);
                }
                q[k] = nq[k];
                if (BORDER) keep[k] = nkeep[k];
            }
            dp += dpz;
        };
        // interior walks take two output planes a step: one wait (the second
        // plane's window reaches one plane further) and one release of both
        // planes' oldest planes (border walks, one plane a step, keep their
        // masks in registers that way)
        int pz = zoff;
        if constexpr (!BORDER) {
            for (; pz + 1 < zend; pz += 2, need += 2) {
                if (!wait_planes(S, R, need + 1)) return false;
                plane(pz);
                plane(pz + 1);
                release_two_planes(S, R);
            }
        }
        for (; pz < zend; ++pz, ++need) {
            if (!wait_planes(S, R, need)) return false;
            plane(pz);
            release_plane(S, R);
        }
        zf = ze;
    }
    for (uint32_t i = 1; i < Wn; ++i) release_plane(S, R);  // the rest of the last window
    return true;
}

// One unit gathered from global memory (gather kernel): warp y computes
// output row y of the unit at flattened index u.
template <typename T, int G, int INTERP>
__device__ void rows_gather(const RJob *__restrict__ jobs, int njobs, int64_t u, const float4 *W, float4 *Rw,
                            const float4 (&wx)[2])
{
    const int y = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x = 2 * lane;
    const Walk w = walk_of(jobs, njobs, u);
    const RJob &J = jobs[w.j];
    const int xe = (int)min(J.out_o[0] + J.out_n[0] - w.Ox, (int64_t)kTBX);
    if ((int64_t)y >= J.out_o[1] + J.out_n[1] - w.Oy) return;
    const T *src = static_cast<const T *>(J.src);
    const bool pair_ok = (((uintptr_t)J.dst) % (2 * sizeof(T))) == 0 && (J.dst_py % 2 == 0) && (J.dst_pz % 2 == 0);
    T *drow = static_cast<T *>(J.dst) +
              ((w.z0 - J.out_o[2]) * J.dst_pz + (w.Oy + y - J.out_o[1]) * J.dst_py + (w.Ox - J.out_o[0]));
    for (int64_t zf = w.z0; zf < w.z1;) {
        const int64_t ze = min(w.z1, (zf / G + 1) * G);
        const int64_t Oz = (zf / G) * G;
        const int zoff = (int)(zf - Oz), zn = (int)(ze - zf);
        RowLayer L;
        row_layer<T, G>(J, w.Ox, w.Oy, Oz, zoff, zn, y, xe, W, Rw, wx, L);
        const int64_t O[3] = {w.Ox, w.Oy, Oz};
        const Frame frame = make_frame(J, O);
        const Clamp cw = make_clamp(J, frame, L.mn, L.mx);
        Gather<T> g;
        g.base = src + ((Oz - J.src_o[2]) * J.src_pz + (w.Oy - J.src_o[1]) * J.src_py + (w.Ox - J.src_o[0]));
        g.py32 = (int)J.src_py;
        g.pz32 = (int)J.src_pz;
        g.py = J.src_py;
        g.pz = J.src_pz;
        g.rows = make_rows(g.base, g.py32, g.pz32, cw.cl, cw.span32);
        for (int pz = zoff; pz < zoff + zn; ++pz) {
            float2 p0, p1, pz2;
            plane_positions(L, W[pz], p0, p1, pz2);
            const float fz = (float)pz;
            const bool fast = L.row_fast && fz >= L.zlo && fz < L.zhi;
            if (fast || x < xe) gathered_pair<T, INTERP>(p0, p1, pz2, frame, cw, g, fast, xe - x, pair_ok, drow + x);
            drow += J.dst_pz;
        }
        zf = ze;
    }
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

// Plans every unit (one warp each, 8 per CTA): plans[u], and the units that
// cannot be staged appended to fb ([0] count, then unit indices).
template <typename T, int G>
__global__ void __launch_bounds__(256) k_tps_plan(const RJob *__restrict__ jobs, int njobs, int64_t total_units,
                                                  Plan *__restrict__ plans, int64_t *fb)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = (int64_t)gridDim.x * 8;
    for (int64_t u = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); u < total_units; u += nw) {
        const Walk w = walk_of(jobs, njobs, u);
        const RJob &J = jobs[w.j];
        Plan P = {};
        if (J.tma_ok) P = plan_walk<T, G>(J, w);
        if (lane == 0) {
            plans[u] = P;
            if (!P.staged) {
                const unsigned long long n = atomicAdd(reinterpret_cast<unsigned long long *>(fb), 1ull);
                fb[1 + n] = u;
            }
        }
    }
}

// The staged walks as two lists in unit order (one CTA of 32 warps): l0 the
// interior walks, l1 the others; each list's count at [0], the unit indices
// after it.  Warp w compacts a contiguous range of units with ballots; the
// ranges' offsets come from the warps' counts.
__global__ void __launch_bounds__(1024) k_tps_lists(const Plan *__restrict__ plans, int64_t total, int *l0, int *l1)
{
    __shared__ int wc[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t per = (((total + 31) / 32) + 31) / 32 * 32;  // units per warp, a multiple of 32
    const int64_t b = (int64_t)warp * per, e = min(total, b + per);
    int c0 = 0, c1 = 0;
    for (int64_t u0 = b; u0 < e; u0 += 32) {
        const int64_t u = u0 + lane;
        const bool st = u < e && plans[u].staged, in = st && plans[u].interior;
        c0 += __popc(__ballot_sync(0xffffffffu, st && in));
        c1 += __popc(__ballot_sync(0xffffffffu, st && !in));
    }
    if (lane == 0) {
        wc[0][warp] = c0;
        wc[1][warp] = c1;
    }
    __syncthreads();
    int o0 = 0, o1 = 0;
    for (int i = 0; i < warp; ++i) {
        o0 += wc[0][i];
        o1 += wc[1][i];
    }
    const unsigned below = (1u << lane) - 1u;
    for (int64_t u0 = b; u0 < e; u0 += 32) {
        const int64_t u = u0 + lane;
        const bool st = u < e && plans[u].staged, in = st && plans[u].interior;
        const unsigned m0 = __ballot_sync(0xffffffffu, st && in), m1 = __ballot_sync(0xffffffffu, st && !in);
        if (st && in) l0[1 + o0 + __popc(m0 & below)] = (int)u;
        if (st && !in) l1[1 + o1 + __popc(m1 & below)] = (int)u;
        o0 += __popc(m0);
        o1 += __popc(m1);
    }
    if (warp == 31 && lane == 0) {  // the last warp's end offsets are the totals
        l0[0] = o0;
        l1[0] = o1;
    }
}

// TPS units whose source footprint is staged by TMA (trilinear), with the
// plans of k_tps_plan; units without a staged plan are left to k_tps_gather.
template <typename T, int G, int MODE>
__global__ void __launch_bounds__(kStagedThreads, 1) k_tps_staged(const RJob *__restrict__ jobs,
                                                                   const int *__restrict__ list,
                                                                   const Plan *__restrict__ plans, int *err)
{
    using Gm = TGeom<T, G>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int abort_sh;
    // ring slots first, on a 128-byte boundary (TMA destinations), then the
    // mbarriers, the weight tables and the row warps' node rows
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = (128u - (raw & 127u)) & 127u;
    TSmem S;
    S.base = smem_raw + pad;
    S.sring = raw + pad;
    S.sfull = S.sring + (uint32_t)Gm::RING_B;
    S.W = reinterpret_cast<float4 *>(S.base + Gm::RING_B + 8 * Gm::NBAR);
    S.W2 = S.W + G;
    S.Rw = S.W2 + 2 * G;
    S.abort = &abort_sh;
    const int tid = threadIdx.x;
    if (tid < G) {
        const float4 w = bspline_w(tid, G);
        S.W[tid] = w;
        S.W2[2 * tid] = make_float4(w.x, w.x, w.y, w.y);
        S.W2[2 * tid + 1] = make_float4(w.z, w.z, w.w, w.w);
    }
    if (tid < kPairs) {
        mbar_init(full_bar(S, tid), 2);                       // one arrival per plane of the pair
        mbar_init(empty_bar(S, tid), 32 * kRowWarps);         // every lane of every row warp
    }
    if (tid == 0) {
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    if (warp == kRowWarps) {  // the producer warp: lane 0 issues every copy
        if (lane == 0) {
            uint32_t seq = 0;
            if (!produce<T, G>(jobs, list, plans, S, seq)) {
                *reinterpret_cast<volatile int *>(&abort_sh) = 1;  // the row warps see it in their waits
                if (err) atomicOr(err, kKernErrTimeout);
            }
            drain_copies(S, seq);
        }
        return;
    }
    float4 *Rw = S.Rw + warp * 2 * Gm::NRW;
    const int x = 2 * lane;
    const float4 wx[2] = {S.W[x % G], S.W[(x + 1) % G]};
    RingPos R = {0u, 0u};
    const int n = list_count(list);
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const Plan P = plans[list[1 + i]];
        Walk w;
        w.j = P.j;
        w.Ox = P.ox;
        w.Oy = P.oy;
        w.z0 = P.z0;
        w.z1 = P.z1;
        const RJob &J = jobs[w.j];
        const bool ok = walk_rows<T, G, MODE == 1>(J, w, P, S, Rw, wx, R);
        if (!ok) {
            // the other warps see the flag in their waits and return
            *reinterpret_cast<volatile int *>(&abort_sh) = 1;
            if (lane == 0 && err) atomicOr(err, kKernErrTimeout);
            return;
        }
    }
}

// TPS units gathered from global memory: the units of fb when it is given
// (the staged kernel's fallback list), else units [0, total_units).
template <typename T, int G, int INTERP>
__global__ void __launch_bounds__(kTpsThreads, 1) k_tps_gather(const RJob *__restrict__ jobs, int njobs,
                                                                int64_t total_units, const int64_t *fb)
{
    using Gm = TGeom<T, G>;
    __shared__ float4 W[G];
    __shared__ float4 Rw[kTBY * Gm::NRW];
    const int tid = threadIdx.x;
    if (tid < G) W[tid] = bspline_w(tid, G);
    __syncthreads();
    const int x = 2 * (tid & 31);
    const float4 wx[2] = {W[x % G], W[(x + 1) % G]};
    float4 *rw = Rw + (tid >> 5) * Gm::NRW;
    const int64_t n = fb ? fb[0] : total_units;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x)
        rows_gather<T, G, INTERP>(jobs, njobs, fb ? fb[1 + i] : i, W, rw, wx);
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

// TPS launches: trilinear jobs run the planning kernel, the staged kernel
// and the gather kernel over the planning kernel's fallback list (ws: the
// list, 1 + total int64 with the count zeroed by the caller, then the plans
// on a 16-byte boundary); nearest-neighbour jobs, or a launch without ws, run
// the gather kernel over every unit.
template <typename T, int G, int INTERP>
cudaError_t launch_tps_t(const RJob *jobs, int njobs, int64_t total, cudaStream_t st, int sms, int *err, void *ws)
{
    using Gm = TGeom<T, G>;
    int64_t *fb = static_cast<int64_t *>(ws);
    if (INTERP == 0 && fb) {
        Plan *plans = reinterpret_cast<Plan *>(fb + ((1 + total + 1) & ~(int64_t)1));
        int64_t pgrid = (total + 7) / 8;
        if (pgrid > (int64_t)sms * 8) pgrid = (int64_t)sms * 8;
        k_tps_plan<T, G><<<(unsigned)pgrid, 256, 0, st>>>(jobs, njobs, total, plans, fb);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        // the two walk lists after the plans: [count, units...] each
        int *l0 = reinterpret_cast<int *>(plans + total);
        int *l1 = l0 + 1 + total;
        k_tps_lists<<<1, 1024, 0, st>>>(plans, total, l0, l1);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        const auto k0 = k_tps_staged<T, G, 0>, k1 = k_tps_staged<T, G, 1>;
        for (int mode = 0; mode < 2; ++mode) {  // interior walks, then the others
            const auto k = mode == 0 ? k0 : k1;
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Gm::smem_bytes);
            if (e != cudaSuccess) return e;
            int per_sm = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kStagedThreads, Gm::smem_bytes);
            if (e != cudaSuccess) return e;
            if (per_sm < 1) return cudaErrorInvalidConfiguration;
            int64_t grid = (int64_t)sms * per_sm;
            if (grid > total) grid = total;
            if (grid < 1) grid = 1;
            k<<<(unsigned)grid, kStagedThreads, Gm::smem_bytes, st>>>(jobs, mode == 0 ? l0 : l1, plans, err);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    auto kg = k_tps_gather<T, G, INTERP>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kg, kTpsThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t grid = (int64_t)sms * per_sm;
    const bool listed = INTERP == 0 && fb;
    if (!listed && grid > total) grid = total;
    if (grid < 1) grid = 1;
    kg<<<(unsigned)grid, kTpsThreads, 0, st>>>(jobs, njobs, total, listed ? fb : nullptr);
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
cudaError_t dispatch_g(const RJob *jobs, int njobs, int64_t total, int g, cudaStream_t st, int sms, int *err,
                       void *fb)
{
    switch (g) {
    case 4: return launch_tps_t<T, 4, INTERP>(jobs, njobs, total, st, sms, err, fb);
    case 8: return launch_tps_t<T, 8, INTERP>(jobs, njobs, total, st, sms, err, fb);
    case 16: return launch_tps_t<T, 16, INTERP>(jobs, njobs, total, st, sms, err, fb);
    case 32: return launch_tps_t<T, 32, INTERP>(jobs, njobs, total, st, sms, err, fb);
    case 64: return launch_tps_t<T, 64, INTERP>(jobs, njobs, total, st, sms, err, fb);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

size_t tps_stage_ws_bytes(int64_t total_bricks)
{
    // fallback list, plans, the two staged-walk lists
    return sizeof(int64_t) * (size_t)((1 + total_bricks + 1) & ~(int64_t)1) + sizeof(Plan) * (size_t)total_bricks +
           sizeof(int) * (size_t)(2 * (1 + total_bricks));
}

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
                            int interp, cudaStream_t st, int sm_count, int *err, void *stage_ws)
{
    if (total_bricks <= 0) return cudaSuccess;
    if (kind == 0) {
        if (dtype == 1) return interp ? launch_affine_t<uint8_t, 1>(jobs_dev, njobs, total_bricks, st, sm_count)
                                      : launch_affine_t<uint8_t, 0>(jobs_dev, njobs, total_bricks, st, sm_count);
        return interp ? launch_affine_t<uint16_t, 1>(jobs_dev, njobs, total_bricks, st, sm_count)
                      : launch_affine_t<uint16_t, 0>(jobs_dev, njobs, total_bricks, st, sm_count);
    }
    if (dtype == 1)
        return interp ? dispatch_g<uint8_t, 1>(jobs_dev, njobs, total_bricks, g, st, sm_count, err, nullptr)
                      : dispatch_g<uint8_t, 0>(jobs_dev, njobs, total_bricks, g, st, sm_count, err, stage_ws);
    return interp ? dispatch_g<uint16_t, 1>(jobs_dev, njobs, total_bricks, g, st, sm_count, err, nullptr)
                  : dispatch_g<uint16_t, 0>(jobs_dev, njobs, total_bricks, g, st, sm_count, err, stage_ws);
}

}  // namespace tw
