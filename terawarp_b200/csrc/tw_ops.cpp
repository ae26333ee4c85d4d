// tw_ops.cpp -- the reference's operator-level entry points (whole-image TPS
// and affine warps) and the TeraWarp command's parameter surface, built on
// the device kernels and the slab pipeline.
#include "tw_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

using namespace tw;

namespace {

struct DevGuard {
    tw_ctx *ctx;
    void *p = nullptr;
    size_t bytes = 0;
    ~DevGuard() { if (p) dfree(ctx, p, bytes); }
};

struct TpsGuard {
    tw_tps *t = nullptr;
    ~TpsGuard() { destroy_tps(t); }
};

size_t elem_size(int dtype) { return dtype == TW_U8 ? 1 : 2; }

// Output planes per slab: ~256 MiB of output, a multiple of `align`.
int64_t pick_slab(size_t plane_bytes, int64_t planes, int64_t align)
{
    int64_t s = (int64_t)((256ull << 20) / std::max<size_t>(plane_bytes, 1));
    s = std::max<int64_t>(align, (s / align) * align);
    return std::min<int64_t>(s, ((planes + align - 1) / align) * align);
}

// TPS warp of a (possibly host-resident) volume with a device node grid;
// output dims dst_sz (the node grid covers the output), one channel.
tw_status tps_warp_volume(tw_ctx *ctx, const float4 *nodes, int g, int dtype, int interp, const void *src,
                          const int64_t src_sz[3], void *dst, const int64_t dst_sz[3])
{
    const int64_t gsz[3] = {grid_size(dst_sz[0], g), grid_size(dst_sz[1], g), grid_size(dst_sz[2], g)};
    std::vector<float> zmin, zmax;
    TW_TRY(tps_layer_zhull(ctx, nodes, gsz, g, ctx->stream, zmin, zmax));
    const size_t es = elem_size(dtype);
    SlabIO io;
    io.src = src;
    io.dst = dst;
    io.src_plane_bytes = es * (size_t)src_sz[0] * (size_t)src_sz[1];
    io.dst_plane_bytes = es * (size_t)dst_sz[0] * (size_t)dst_sz[1];
    io.src_planes = src_sz[2];
    io.dst_planes = dst_sz[2];
    io.slab = pick_slab(io.dst_plane_bytes, dst_sz[2], g);
    auto need = [&](int64_t z0, int64_t z1, int64_t &lo, int64_t &hi) {
        float mn = 3.4e38f, mx = -3.4e38f;
        for (int64_t cz = z0 / g; cz <= (z1 - 1) / g && cz < (int64_t)zmin.size(); ++cz) {
            mn = std::min(mn, zmin[cz]);
            mx = std::max(mx, zmax[cz]);
        }
        lo = (int64_t)std::floor((double)mn) - 1;
        hi = (int64_t)std::floor((double)mx) + 2;
    };
    auto compute = [&](int64_t z0, int64_t z1, const void *d_src, void *d_dst, cudaStream_t st) -> tw_status {
        RJob j = tps_job(d_src, src_sz, d_dst, dst_sz, nodes, g, dtype, interp);
        j.out_o[2] = z0;
        j.out_n[2] = z1 - z0;
        j.dst = static_cast<char *>(d_dst) + (size_t)z0 * io.dst_plane_bytes;
        return run_jobs(ctx, &j, 1, st);
    };
    return stream_slabs(ctx, io, need, compute);
}

tw_status affine_warp_volume(tw_ctx *ctx, const double M[16], int dtype, int interp, const void *src,
                             const int64_t src_sz[3], void *dst, const int64_t dst_sz[3])
{
    const size_t es = elem_size(dtype);
    SlabIO io;
    io.src = src;
    io.dst = dst;
    io.src_plane_bytes = es * (size_t)src_sz[0] * (size_t)src_sz[1];
    io.dst_plane_bytes = es * (size_t)dst_sz[0] * (size_t)dst_sz[1];
    io.src_planes = src_sz[2];
    io.dst_planes = dst_sz[2];
    io.slab = pick_slab(io.dst_plane_bytes, dst_sz[2], 8);
    auto need = [&](int64_t z0, int64_t z1, int64_t &lo, int64_t &hi) {
        // q_z over the box corners of output planes [z0, z1) (affine: extremes at corners)
        double mn = 1e300, mx = -1e300;
        for (int c = 0; c < 8; ++c) {
            double x = (c & 1) ? (double)(dst_sz[0] - 1) : 0.0;
            double y = (c & 2) ? (double)(dst_sz[1] - 1) : 0.0;
            double z = (c & 4) ? (double)(z1 - 1) : (double)z0;
            double q = M[8] * x + M[9] * y + M[10] * z + M[11];
            mn = std::min(mn, q);
            mx = std::max(mx, q);
        }
        lo = (int64_t)std::floor(mn) - 1;
        hi = (int64_t)std::floor(mx) + 2;
    };
    auto compute = [&](int64_t z0, int64_t z1, const void *d_src, void *d_dst, cudaStream_t st) -> tw_status {
        RJob j = affine_job(d_src, src_sz, d_dst, dst_sz, M, dtype, interp);
        j.out_o[2] = z0;
        j.out_n[2] = z1 - z0;
        j.dst = static_cast<char *>(d_dst) + (size_t)z0 * io.dst_plane_bytes;
        return run_jobs(ctx, &j, 1, st);
    };
    return stream_slabs(ctx, io, need, compute);
}

// Solve + node grid for a TPS job whose output canvas is dst_sz.
tw_status build_tps_field(tw_ctx *ctx, const tw_marker *centres, const tw_marker *values, int n, double lambda,
                          double scale, int g, const int64_t dst_sz[3], TpsGuard &tg, DevGuard &nodes)
{
    TW_TRY(make_tps(ctx, centres, values, n, lambda, scale, ctx->stream, &tg.t));
    const int64_t gsz[3] = {grid_size(dst_sz[0], g), grid_size(dst_sz[1], g), grid_size(dst_sz[2], g)};
    nodes.bytes = sizeof(float4) * (size_t)(gsz[0] * gsz[1] * gsz[2]);
    TW_TRY(dmalloc(ctx, &nodes.p, nodes.bytes));
    const int64_t off[3] = {0, 0, 0};
    return eval_grid(ctx, tg.t, gsz, g, off, static_cast<float4 *>(nodes.p), ctx->stream);
}

}  // namespace

extern "C" {

tw_status tw_imgwarp_smallmemory_image(tw_ctx *ctx, const tw_marker *ql_marker_tar, const tw_marker *ql_marker_sub,
                                       int n, int64_t szBlock_x, int64_t szBlock_y, int64_t szBlock_z, int interp_df,
                                       int interp_img, int dtype, const void *img_sub, const int64_t sz_img_sub[4],
                                       void *img_warp)
{
    if (!ctx) return TW_ERR_ARG;
    // argument checks of q_imgwarp_tps_quicksmallmemory.cpp:2001-2034
    if (!img_sub || !sz_img_sub || !img_warp) return fail(ctx, TW_ERR_ARG, "p_img_sub or sz_img_sub is invalid");
    if (!ql_marker_tar || !ql_marker_sub || n <= 0) return fail(ctx, TW_ERR_ARG, "target or subject control points is invalid");
    if (szBlock_x <= 0 || szBlock_y <= 0 || szBlock_z <= 0) return fail(ctx, TW_ERR_ARG, "block size is invalid");
    for (int a = 0; a < 4; ++a)
        if (sz_img_sub[a] <= 0) return fail(ctx, TW_ERR_ARG, "image size is invalid");
    if (szBlock_x >= sz_img_sub[0] || szBlock_y >= sz_img_sub[1] || szBlock_z >= sz_img_sub[2])
        return fail(ctx, TW_ERR_ARG, "block size should smaller than the image size");
    if (interp_df != 0 && interp_df != 1) return fail(ctx, TW_ERR_ARG, "DF_interp_method should be 0(linear) or 1(bspline)");
    if (interp_img != 0 && interp_img != 1) return fail(ctx, TW_ERR_ARG, "img_interp_method should be 0(linear) or 1(nn)");
    if (szBlock_x != szBlock_y || szBlock_x != szBlock_z)
        return fail(ctx, TW_ERR_ARG, "df_interp_method=bspline need szBlock_x=szBlock_y=szBlock_z");
    if (dtype != TW_U8 && dtype != TW_U16) return fail(ctx, TW_ERR_ARG, "dtype must be TW_U8 or TW_U16");
    const int g = (int)szBlock_x;
    if (!g_supported(g)) return fail(ctx, TW_ERR_UNSUPPORTED, "grid spacing must be 4, 8, 16, 32 or 64");
    if (n < 4) return fail(ctx, TW_ERR_SINGULAR, "TPS needs at least 4 landmark pairs");
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    const int64_t sz[3] = {sz_img_sub[0], sz_img_sub[1], sz_img_sub[2]};
    TpsGuard tg;
    DevGuard nodes{ctx};
    // matchTargetPos = ql_marker_tar are the TPS values, matchSubjectPos =
    // ql_marker_sub the centres (q_imgwarp_tps_quicksmallmemory.cpp:2039-2046, :416-464)
    TW_TRY(build_tps_field(ctx, ql_marker_sub, ql_marker_tar, n, 0.2, 1.0, g, sz, tg, nodes));
    const size_t vol = elem_size(dtype) * (size_t)(sz[0] * sz[1] * sz[2]);
    for (int64_t c = 0; c < sz_img_sub[3]; ++c) {
        TW_TRY(tps_warp_volume(ctx, static_cast<const float4 *>(nodes.p), g, dtype, interp_img,
                               static_cast<const char *>(img_sub) + c * vol, sz, static_cast<char *>(img_warp) + c * vol,
                               sz));
    }
    return TW_OK;
}

tw_status tw_q_imagewarp_affine_image(tw_ctx *ctx, const tw_marker *ql_marker_tar, const tw_marker *ql_marker_sub,
                                      int n, int dtype, const void *img_sub, const int64_t sz_img_sub[4], void *img_out)
{
    if (!ctx) return TW_ERR_ARG;
    // q_warp_affine_tps.cpp:1334-1338
    if (!ql_marker_tar || !ql_marker_sub || n <= 0) return fail(ctx, TW_ERR_ARG, "target or subject control points is invalid");
    if (!img_sub || !img_out || !sz_img_sub) return fail(ctx, TW_ERR_ARG, "image is invalid");
    if (dtype != TW_U8 && dtype != TW_U16) return fail(ctx, TW_ERR_ARG, "dtype must be TW_U8 or TW_U16");
    for (int a = 0; a < 4; ++a)
        if (sz_img_sub[a] <= 0) return fail(ctx, TW_ERR_ARG, "image size is invalid");
    double M[16];
    TW_TRY(tw_fit_affine(ctx, ql_marker_tar, ql_marker_sub, n, M));  // B = T A: sub = T tar
    const int64_t sz[3] = {sz_img_sub[0], sz_img_sub[1], sz_img_sub[2]};
    const size_t vol = elem_size(dtype) * (size_t)(sz[0] * sz[1] * sz[2]);
    for (int64_t c = 0; c < sz_img_sub[3]; ++c)
        TW_TRY(affine_warp_volume(ctx, M, dtype, 0, static_cast<const char *>(img_sub) + c * vol, sz,
                                  static_cast<char *>(img_out) + c * vol, sz));
    return TW_OK;
}

void tw_params_default(tw_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->warp_mode = 0;
    p->device_mode = 1;
    p->resize_mode = 0;
    p->deformation_mode = 1;
    p->para_x = p->para_y = p->para_z = 1.0;
    p->grid_spacing = 4;
    p->marker_scale = 1.0;
    p->lambda = 0.2;
    p->interp = 0;
}

tw_status tw_output_size(const tw_params *p, const int64_t in_sz[3], int64_t out_sz[3])
{
    if (!p || !in_sz || !out_sz) return TW_ERR_ARG;
    if (p->resize_mode == 1) {
        out_sz[0] = p->newsize_x;
        out_sz[1] = p->newsize_y;
        out_sz[2] = p->newsize_z;
        if (out_sz[0] < 1 || out_sz[1] < 1 || out_sz[2] < 1) return TW_ERR_ARG;
    } else if (p->resize_mode == 0) {
        for (int a = 0; a < 3; ++a) out_sz[a] = in_sz[a];
    } else {
        return TW_ERR_ARG;
    }
    return TW_OK;
}

tw_status tw_bigimagewarp(tw_ctx *ctx, const tw_params *p, const tw_marker *marker_sub, const tw_marker *marker_tar,
                          int n, int dtype, const void *img_sub, const int64_t sz[4], void *img_out)
{
    if (!ctx || !p || !img_sub || !sz || !img_out) return TW_ERR_ARG;
    if (p->device_mode != 1)
        return fail(ctx, TW_ERR_UNSUPPORTED, "device_mode must be 1: this build has no CPU warp path");
    if (dtype != TW_U8 && dtype != TW_U16) return fail(ctx, TW_ERR_ARG, "dtype must be TW_U8 or TW_U16");
    for (int a = 0; a < 4; ++a)
        if (sz[a] <= 0) return fail(ctx, TW_ERR_ARG, "image size is invalid");
    const int64_t in_sz[3] = {sz[0], sz[1], sz[2]};
    int64_t out_sz[3];
    if (tw_output_size(p, in_sz, out_sz) != TW_OK) return fail(ctx, TW_ERR_ARG, "invalid resize_mode / newsize");
    const int interp = p->interp;
    if (interp != 0 && interp != 1) return fail(ctx, TW_ERR_ARG, "interp must be 0 or 1");
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t es = elem_size(dtype);
    const size_t in_vol = es * (size_t)(in_sz[0] * in_sz[1] * in_sz[2]);
    const size_t out_vol = es * (size_t)(out_sz[0] * out_sz[1] * out_sz[2]);
    const double scale = p->marker_scale > 0 ? p->marker_scale : 1.0;
    const double lambda = p->lambda > 0 ? p->lambda : 0.2;

    if (p->warp_mode == 0 && p->deformation_mode == 1) {
        const int g = p->grid_spacing > 0 ? p->grid_spacing : 4;
        if (!g_supported(g)) return fail(ctx, TW_ERR_UNSUPPORTED, "grid spacing must be 4, 8, 16, 32 or 64");
        if (!marker_sub || !marker_tar || n < 4) return fail(ctx, TW_ERR_ARG, "TPS needs n >= 4 landmark pairs");
        TpsGuard tg;
        DevGuard nodes{ctx};
        // the plugin passes (sub, tar) into (ql_marker_tar, ql_marker_sub)
        // (plugin_Bigimagewarp.cpp:197): centres = target markers,
        // values = subject markers
        TW_TRY(build_tps_field(ctx, marker_tar, marker_sub, n, lambda, scale, g, out_sz, tg, nodes));
        for (int64_t c = 0; c < sz[3]; ++c)
            TW_TRY(tps_warp_volume(ctx, static_cast<const float4 *>(nodes.p), g, dtype, interp,
                                   static_cast<const char *>(img_sub) + c * in_vol, in_sz,
                                   static_cast<char *>(img_out) + c * out_vol, out_sz));
        return TW_OK;
    }
    double M[16];
    if (p->warp_mode == 0 && p->deformation_mode == 0) {
        if (!marker_sub || !marker_tar || n < 4) return fail(ctx, TW_ERR_ARG, "affine needs n >= 4 landmark pairs");
        std::vector<tw_marker> ts(n), ss(n);
        for (int i = 0; i < n; ++i) {
            ts[i] = {(float)(scale * marker_tar[i].x), (float)(scale * marker_tar[i].y), (float)(scale * marker_tar[i].z)};
            ss[i] = {(float)(scale * marker_sub[i].x), (float)(scale * marker_sub[i].y), (float)(scale * marker_sub[i].z)};
        }
        TW_TRY(tw_fit_affine(ctx, ts.data(), ss.data(), n, M));
    } else {
        const double para[3] = {p->para_x, p->para_y, p->para_z};
        if (make_param_affine(p->warp_mode, p->deformation_mode, para, in_sz, out_sz, M) != TW_OK)
            return fail(ctx, TW_ERR_ARG, "invalid warp_mode / deformation_mode / para_*");
    }
    for (int64_t c = 0; c < sz[3]; ++c)
        TW_TRY(affine_warp_volume(ctx, M, dtype, interp, static_cast<const char *>(img_sub) + c * in_vol, in_sz,
                                  static_cast<char *>(img_out) + c * out_vol, out_sz));
    return TW_OK;
}

int tw_downsample_factor(const int64_t sz[3])
{
    if (!sz) return 1;
    int64_t f = std::max(sz[0], std::max(sz[1], sz[2]));
    int64_t d = f / 600 + (f % 600 >= 300 ? 1 : 0);
    return (int)std::max<int64_t>(1, d);
}

tw_status tw_downsample_image(tw_ctx *ctx, int dtype, const void *img, const int64_t sz[4], void *img_out,
                              int64_t out_sz[3])
{
    if (!ctx || !img || !sz || !img_out || !out_sz) return TW_ERR_ARG;
    if (dtype != TW_U8 && dtype != TW_U16) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    const int64_t in_sz[3] = {sz[0], sz[1], sz[2]};
    const int f = tw_downsample_factor(in_sz);
    for (int a = 0; a < 3; ++a) {
        out_sz[a] = in_sz[a] / f;
        if (out_sz[a] < 1) return fail(ctx, TW_ERR_ARG, "volume too small to downsample");
    }
    // the reference fits the matrix from (tar, tar * factor)
    // (q_warp_affine_tps.cpp:1494-1501), i.e. a pure scaling by the factor
    double M[16] = {0};
    M[0] = M[5] = M[10] = (double)f;
    M[15] = 1.0;
    const size_t es = elem_size(dtype);
    const size_t in_vol = es * (size_t)(in_sz[0] * in_sz[1] * in_sz[2]);
    const size_t out_vol = es * (size_t)(out_sz[0] * out_sz[1] * out_sz[2]);
    for (int64_t c = 0; c < sz[3]; ++c)
        TW_TRY(affine_warp_volume(ctx, M, dtype, 0, static_cast<const char *>(img) + c * in_vol, in_sz,
                                  static_cast<char *>(img_out) + c * out_vol, out_sz));
    return TW_OK;
}

}  // extern "C"
