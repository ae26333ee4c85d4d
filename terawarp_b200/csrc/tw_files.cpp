// tw_files.cpp -- the plugin's whole command on files: marker files in, a
// .v3draw volume or a directory of slices in, the warped volume (and its
// downsampled preview) out, as bigimagewarp does (plugin_Bigimagewarp.cpp:
// 123-336) with its whole-image branch (:158-209) and its slice-directory
// branch (:210-330).
#include "tw_host.h"

#include <sys/stat.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace tw;

namespace {

std::string base_name(const std::string &path, bool strip_ext)
{
    std::string p = path;
    while (p.size() > 1 && p.back() == '/') p.pop_back();
    const size_t slash = p.find_last_of('/');
    std::string b = slash == std::string::npos ? p : p.substr(slash + 1);
    if (strip_ext) {
        const size_t dot = b.find_last_of('.');
        if (dot != std::string::npos && dot > 0) b = b.substr(0, dot);
    }
    return b;
}

// Output name suffix of a mode (the reference has _affine and _stps).
const char *mode_suffix(const tw_params *p)
{
    if (p->warp_mode == 0) return p->deformation_mode == 0 ? "_affine" : (p->deformation_mode == 1 ? "_stps" : "_scaling");
    return p->deformation_mode == 0 ? "_rotation" : "_translation";
}

bool read_markers(const char *path, std::vector<tw_marker> &m)
{
    int n = 0;
    if (tw_marker_file_read(path, nullptr, 0, &n) != TW_OK) return false;
    m.resize((size_t)n);
    return tw_marker_file_read(path, m.data(), n, &n) == TW_OK;
}

struct SliceDir {
    tw_slice_dir *d = nullptr;
    ~SliceDir() { tw_slice_dir_close(d); }
};
struct SliceWriter {
    tw_slice_writer *w = nullptr;
    ~SliceWriter() { tw_slice_writer_close(w); }
};

// Tiled warp of a slice directory into another: TPS from landmarks, or the
// 4x4 matrix M (pull-back).
tw_status warp_slices(tw_ctx *ctx, const tw_params *p, const tw_marker *sub, const tw_marker *tar, int n,
                      const double *M, const std::string &src_dir, const std::string &dst_dir, int64_t out_sz_req[3],
                      bool tps)
{
    SliceDir in;
    TW_TRY(tw_slice_dir_open(src_dir.c_str(), 0, &in.d) == TW_OK ? TW_OK
                                                                   : fail(ctx, TW_ERR_IO, "cannot open slices in " + src_dir));
    int64_t sz[3];
    int dtype = 0;
    tw_slice_dir_info(in.d, sz, &dtype);
    if (dtype != TW_U8 && dtype != TW_U16) return fail(ctx, TW_ERR_UNSUPPORTED, "slices must be uint8 or uint16");
    int64_t out_sz[3] = {sz[0], sz[1], sz[2]};
    if (out_sz_req)
        for (int a = 0; a < 3; ++a) out_sz[a] = out_sz_req[a] > 0 ? out_sz_req[a] : sz[a];
    SliceWriter out;
    if (tw_slice_writer_create(dst_dir.c_str(), out_sz, dtype, 0, &out.w) != TW_OK)
        return fail(ctx, TW_ERR_IO, "cannot create the output slices in " + dst_dir);
    tw_tile_opts opts;
    std::memset(&opts, 0, sizeof(opts));
    opts.interp = p->interp;
    if (tps) {
        const int g = p->grid_spacing > 0 ? p->grid_spacing : 4;
        const double scale = p->marker_scale > 0 ? p->marker_scale : 4.0;
        // the plugin passes (subject, target) into (ql_marker_tar, ql_marker_sub)
        // (plugin_Bigimagewarp.cpp:294)
        return tw_imgwarp_smallmemory_tiled(ctx, sub, tar, n, scale, g, dtype, sz, tw_box_reader_slices, in.d,
                                            tw_box_writer_slices, out.w, &opts);
    }
    return tw_warp_affine_tiled(ctx, M, dtype, sz, out_sz, tw_box_reader_slices, in.d, tw_box_writer_slices, out.w,
                                &opts);
}

}  // namespace

extern "C" {

tw_status tw_bigimagewarp_files(tw_ctx *ctx, const tw_params *p, const char *img_sub, const char *marker_sub,
                                const char *marker_tar, const char *out_dir)
{
    if (!ctx || !p || !img_sub || !out_dir) return TW_ERR_ARG;
    if (p->device_mode != 1)
        return fail(ctx, TW_ERR_UNSUPPORTED, "device_mode must be 1: this build has no CPU warp path");
    const bool needs_markers = p->warp_mode == 0 && (p->deformation_mode == 0 || p->deformation_mode == 1);
    std::vector<tw_marker> sub, tar;
    if (needs_markers) {
        if (!marker_sub || !marker_tar || !read_markers(marker_sub, sub) || !read_markers(marker_tar, tar))
            return fail(ctx, TW_ERR_IO, "at least one marker file is invalid");
        if (sub.size() != tar.size() || sub.empty())
            return fail(ctx, TW_ERR_ARG, "target or subject control points is invalid");
    }
    const int n = (int)sub.size();
    struct stat st;
    if (::stat(img_sub, &st) != 0) return fail(ctx, TW_ERR_IO, std::string("cannot read ") + img_sub);
    const std::string suffix = mode_suffix(p);
    const std::string out = out_dir;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));

    if (!S_ISDIR(st.st_mode)) {
        // whole image (.v3draw)
        int64_t sz[4];
        int dtype = 0;
        if (tw_v3draw_read_header(img_sub, sz, &dtype, nullptr) != TW_OK)
            return fail(ctx, TW_ERR_IO, std::string("not a raw stack: ") + img_sub);
        if (dtype != TW_U8 && dtype != TW_U16) return fail(ctx, TW_ERR_UNSUPPORTED, "image must be uint8 or uint16");
        const size_t es = dtype == TW_U8 ? 1 : 2;
        std::vector<unsigned char> img(es * (size_t)(sz[0] * sz[1] * sz[2] * sz[3]));
        if (tw_v3draw_read(img_sub, img.data(), img.size()) != TW_OK)
            return fail(ctx, TW_ERR_IO, std::string("cannot read ") + img_sub);
        const int64_t in3[3] = {sz[0], sz[1], sz[2]};
        int64_t out3[3];
        if (tw_output_size(p, in3, out3) != TW_OK) return fail(ctx, TW_ERR_ARG, "invalid resize_mode / newsize");
        std::vector<unsigned char> res(es * (size_t)(out3[0] * out3[1] * out3[2] * sz[3]));
        TW_TRY(tw_bigimagewarp(ctx, p, sub.data(), tar.data(), n, dtype, img.data(), sz, res.data()));
        const std::string name = out + "/" + base_name(img_sub, true) + suffix;
        const int64_t osz[4] = {out3[0], out3[1], out3[2], sz[3]};
        if (tw_v3draw_write((name + ".v3draw").c_str(), res.data(), osz, dtype) != TW_OK)
            return fail(ctx, TW_ERR_IO, "cannot write " + name + ".v3draw");
        if (p->downsample_mode) {
            const int f = tw_downsample_factor(out3);
            std::vector<unsigned char> ds(es * (size_t)((out3[0] / f) * (out3[1] / f) * (out3[2] / f) * sz[3]));
            int64_t dsz[3];
            TW_TRY(tw_downsample_image(ctx, dtype, res.data(), osz, ds.data(), dsz));
            const int64_t d4[4] = {dsz[0], dsz[1], dsz[2], sz[3]};
            if (tw_v3draw_write((name + "_downsample.v3draw").c_str(), ds.data(), d4, dtype) != TW_OK)
                return fail(ctx, TW_ERR_IO, "cannot write " + name + "_downsample.v3draw");
        }
        return TW_OK;
    }

    // directory of per-Z slices: tiled, tiles written into the output slices
    const std::string name = out + "/" + base_name(img_sub, false) + suffix;
    const std::string warped = name + "_slice";
    int64_t in_sz[3];
    {
        SliceDir probe;
        if (tw_slice_dir_open(img_sub, 1, &probe.d) != TW_OK)
            return fail(ctx, TW_ERR_IO, std::string("cannot open slices in ") + img_sub);
        tw_slice_dir_info(probe.d, in_sz, nullptr);
    }
    int64_t out_sz[3];
    if (tw_output_size(p, in_sz, out_sz) != TW_OK) return fail(ctx, TW_ERR_ARG, "invalid resize_mode / newsize");
    if (p->warp_mode == 0 && p->deformation_mode == 1) {
        if (out_sz[0] != in_sz[0] || out_sz[1] != in_sz[1] || out_sz[2] != in_sz[2])
            return fail(ctx, TW_ERR_UNSUPPORTED, "the tiled TPS warp keeps the input size");
        TW_TRY(warp_slices(ctx, p, sub.data(), tar.data(), n, nullptr, img_sub, warped, nullptr, true));
    } else {
        double M[16];
        if (p->warp_mode == 0 && p->deformation_mode == 0) {
            // q_imagewarp_affine_cyf scales both marker sets (q_warp_affine_tps.cpp:866-874)
            const double s = p->marker_scale > 0 ? p->marker_scale : 4.0;
            std::vector<tw_marker> ts(n), ss(n);
            for (int i = 0; i < n; ++i) {
                ts[i] = {(float)(s * tar[i].x), (float)(s * tar[i].y), (float)(s * tar[i].z)};
                ss[i] = {(float)(s * sub[i].x), (float)(s * sub[i].y), (float)(s * sub[i].z)};
            }
            TW_TRY(tw_fit_affine(ctx, ts.data(), ss.data(), n, M));
        } else {
            const double para[3] = {p->para_x, p->para_y, p->para_z};
            if (tw_make_affine(p->warp_mode, p->deformation_mode, para, in_sz, out_sz, M) != TW_OK)
                return fail(ctx, TW_ERR_ARG, "invalid warp_mode / deformation_mode / para_*");
        }
        TW_TRY(warp_slices(ctx, p, nullptr, nullptr, 0, M, img_sub, warped, out_sz, false));
    }
    if (p->downsample_mode) {
        // q_imagewarp_affine_cyf_downsample (q_warp_affine_tps.cpp:1474-1519): a
        // pure scaling by the factor, from the warped slices
        const int f = tw_downsample_factor(out_sz);
        double M[16] = {0};
        M[0] = M[5] = M[10] = (double)f;
        M[15] = 1.0;
        int64_t dsz[3];
        for (int a = 0; a < 3; ++a) {
            dsz[a] = out_sz[a] / f;
            if (dsz[a] < 1) return fail(ctx, TW_ERR_ARG, "volume too small to downsample");
        }
        tw_params q = *p;
        q.interp = 0;
        TW_TRY(warp_slices(ctx, &q, nullptr, nullptr, 0, M, warped, name + "_downsample_slice", dsz, false));
    }
    return TW_OK;
}

}  // extern "C"
