// tw_tiled.cpp -- out-of-core tiled warps: the output volume is cut into
// tiles; each tile's source box (the exact footprint of its samples) is read
// by a tile source, streamed host -> HBM, warped, and streamed back to a tile
// sink, with reads, H2D copies, kernels and D2H copies of consecutive tiles
// overlapped on three streams through a ring of pinned and device slots.
//
// Reference: imgwarp_smallmemory_CYF (q_imgwarp_tps_quicksmallmemory.cpp:
// 1161-1994) and q_imagewarp_affine_cyf (q_warp_affine_tps.cpp:851-1329) loop
// over 1000^3 tiles synchronously (read, warp, save), estimate each tile's
// source box from 14 (TPS) or 8 (affine) probe points plus a 60 / 10 voxel
// halo, and write 0 where a sample falls outside that box.  Here the box is
// the convex-hull bound of the B-spline over the tile's nodes (or the affine
// image of the tile's corners), so the tiled output equals the whole-volume
// output voxel for voxel.
#include "tw_host.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

using namespace tw;

namespace {

size_t esize(int dtype) { return dtype == TW_U8 ? 1 : 2; }

struct Box {
    int64_t o[3];   // origin
    int64_t n[3];   // extent (0 on any axis = empty)
    int64_t count() const { return n[0] * n[1] * n[2]; }
};

struct TileIO {
    tw_read_box_fn read;
    void *read_user;
    tw_write_box_fn write;
    void *write_user;
};

struct Slot {
    void *d_src = nullptr, *d_dst = nullptr;
    void *h_src = nullptr, *h_dst = nullptr;
    cudaEvent_t e_in = nullptr, e_comp = nullptr, e_out = nullptr;
    int64_t batch = -1;      // batch whose result is in flight in this slot
};

// Tiles warped by one resample launch: a full tile goes alone; the smaller
// ones (the volume's uneven edge tiles) are grouped, in tile order, until a
// group holds as many output voxels as a full tile (at most 64 tiles).  Each
// tile's source box and output sit in the slot's buffers at 256-byte aligned
// element offsets.
struct Batch {
    std::vector<int64_t> tiles;
    std::vector<int64_t> src_off, out_off;
    int64_t src_total = 0, out_total = 0;
};

// Source-box bound for a tile from the hull of its sample positions.  With
// align > 1 the box's x extent is widened (inside the volume) to a multiple of
// `align` elements and to at least min_x, and its y extent to at least min_y,
// so that it meets the TMA rules of the staged resample (16-byte pitches, no
// narrower or lower than one staged plane).
Box box_from_hull(const float lo[3], const float hi[3], const int64_t sz[3], int64_t align = 1, int64_t min_x = 0,
                  int64_t min_y = 0)
{
    Box b;
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(lo[a]) || !std::isfinite(hi[a])) {  // degenerate field: read everything
            b.o[a] = 0;
            b.n[a] = sz[a];
            continue;
        }
        int64_t l = (int64_t)std::floor((double)lo[a]) - 1;
        int64_t h = (int64_t)std::floor((double)hi[a]) + 2;
        l = std::max<int64_t>(l, 0);
        h = std::min<int64_t>(h, sz[a] - 1);
        b.o[a] = l;
        b.n[a] = h >= l ? h - l + 1 : 0;
    }
    if (align > 1 && b.n[0] > 0 && b.n[1] > 0 && b.n[2] > 0) {
        int64_t w = std::max(b.n[0], std::min(min_x, sz[0]));
        w = std::min(sz[0], ((w + align - 1) / align) * align);
        const int64_t o = std::max<int64_t>(0, std::min(b.o[0], sz[0] - w));
        b.o[0] = o;
        b.n[0] = w;
        const int64_t hgt = std::min(sz[1], std::max(b.n[1], min_y));
        b.o[1] = std::max<int64_t>(0, std::min(b.o[1], sz[1] - hgt));
        b.n[1] = hgt;
    }
    return b;
}

// Copies a box between a host volume and a device buffer with the DMA
// engine (strided 3-D copy, no host CPU work).
cudaError_t copy_box(void *dst, const void *src, int64_t dst_x, int64_t dst_y, const int64_t dst_off[3],
                     int64_t src_x, int64_t src_y, const int64_t src_off[3], const int64_t n[3], size_t es,
                     cudaMemcpyKind kind, cudaStream_t st)
{
    cudaMemcpy3DParms p;
    std::memset(&p, 0, sizeof(p));
    p.srcPtr = make_cudaPitchedPtr(const_cast<void *>(src), (size_t)src_x * es, (size_t)src_x, (size_t)src_y);
    p.dstPtr = make_cudaPitchedPtr(dst, (size_t)dst_x * es, (size_t)dst_x, (size_t)dst_y);
    p.srcPos = make_cudaPos((size_t)src_off[0] * es, (size_t)src_off[1], (size_t)src_off[2]);
    p.dstPos = make_cudaPos((size_t)dst_off[0] * es, (size_t)dst_off[1], (size_t)dst_off[2]);
    p.extent = make_cudaExtent((size_t)n[0] * es, (size_t)n[1], (size_t)n[2]);
    p.kind = kind;
    return cudaMemcpy3DAsync(&p, st);
}

tw_status run_tiled(tw_ctx *ctx, int kind, const float4 *nodes, int g, const double *M, int dtype, int interp,
                    const int64_t src_sz[3], const int64_t out_sz[3], const TileIO &io, const tw_tile_opts *opts)
{
    const size_t es = esize(dtype);
    int64_t T[3] = {512, 512, 512};
    int depth = 2;
    if (opts) {
        for (int a = 0; a < 3; ++a)
            if (opts->tile[a] > 0) T[a] = opts->tile[a];
        if (opts->staging_depth > 0) depth = std::min(4, std::max(2, opts->staging_depth));
    }
    if (kind == 1) {
        // TPS tiles start on resample-unit boundaries of the whole volume
        // (64 in x, 16 in y, a control cell layer in z): every unit then has
        // the frame it has in a whole-volume warp, so the tiled output equals
        // the whole-volume output voxel for voxel
        int64_t bd[3];
        brick_dims(1, g, bd);
        for (int a = 0; a < 3; ++a) T[a] = std::max<int64_t>(bd[a], (T[a] / bd[a]) * bd[a]);
    }
    for (int a = 0; a < 3; ++a) T[a] = std::min(T[a], out_sz[a]);
    // output region (the whole output unless the options name one); a TPS
    // region grows to whole resample units so that every unit keeps its
    // whole-volume frame
    int64_t r0[3] = {0, 0, 0}, r1[3] = {out_sz[0], out_sz[1], out_sz[2]};
    if (opts && (opts->region_n[0] > 0 || opts->region_n[1] > 0 || opts->region_n[2] > 0)) {
        int64_t bd[3] = {1, 1, 1};
        if (kind == 1) brick_dims(1, g, bd);
        for (int a = 0; a < 3; ++a) {
            if (opts->region_n[a] <= 0 || opts->region_o[a] < 0 || opts->region_o[a] >= out_sz[a])
                return fail(ctx, TW_ERR_ARG, "tile region outside the output volume");
            r0[a] = (opts->region_o[a] / bd[a]) * bd[a];
            r1[a] = std::min(out_sz[a], ((opts->region_o[a] + opts->region_n[a] + bd[a] - 1) / bd[a]) * bd[a]);
        }
    }
    int64_t nt[3], t0[3];
    for (int a = 0; a < 3; ++a) {
        t0[a] = r0[a] / T[a];
        nt[a] = (r1[a] + T[a] - 1) / T[a] - t0[a];
    }
    const int64_t ntiles = nt[0] * nt[1] * nt[2];

    // tile boxes (clipped to the region) and their source footprints
    std::vector<Box> tiles(ntiles), srcs(ntiles);
    for (int64_t t = 0; t < ntiles; ++t) {
        int64_t ix = t % nt[0], iy = (t / nt[0]) % nt[1], iz = t / (nt[0] * nt[1]);
        const int64_t idx[3] = {ix + t0[0], iy + t0[1], iz + t0[2]};
        for (int a = 0; a < 3; ++a) {
            const int64_t lo = std::max(idx[a] * T[a], r0[a]);
            const int64_t hi = std::min((idx[a] + 1) * T[a], r1[a]);
            tiles[t].o[a] = lo;
            tiles[t].n[a] = hi - lo;
        }
    }
    if (kind == 1) {
        std::vector<CellBox> cb(ntiles);
        for (int64_t t = 0; t < ntiles; ++t)
            for (int a = 0; a < 3; ++a) {
                cb[t].c0[a] = tiles[t].o[a] / g;
                cb[t].c1[a] = (tiles[t].o[a] + tiles[t].n[a] + g - 1) / g;
            }
        const int64_t gsz[3] = {grid_size(out_sz[0], g), grid_size(out_sz[1], g), grid_size(out_sz[2], g)};
        std::vector<float> lo, hi;
        TW_TRY(tps_box_hull(ctx, nodes, gsz, g, cb, ctx->stream, lo, hi));
        for (int64_t t = 0; t < ntiles; ++t)
            srcs[t] = box_from_hull(&lo[3 * t], &hi[3 * t], src_sz, 16 / (int64_t)es, kStageBoxW, kStageBoxH);
    } else {
        for (int64_t t = 0; t < ntiles; ++t) {
            float lo[3], hi[3];
            for (int r = 0; r < 3; ++r) {
                double mn = 1e300, mxv = -1e300;
                for (int c = 0; c < 8; ++c) {
                    double p[3];
                    for (int a = 0; a < 3; ++a)
                        p[a] = (double)tiles[t].o[a] + (((c >> a) & 1) ? (double)(tiles[t].n[a] - 1) : 0.0);
                    double q = M[r * 4] * p[0] + M[r * 4 + 1] * p[1] + M[r * 4 + 2] * p[2] + M[r * 4 + 3];
                    mn = std::min(mn, q);
                    mxv = std::max(mxv, q);
                }
                lo[r] = (float)mn;
                hi[r] = (float)mxv;
            }
            srcs[t] = box_from_hull(lo, hi, src_sz);
        }
    }
    // batches: every full tile alone, then the edge tiles in groups
    const int64_t full = T[0] * T[1] * T[2];
    std::vector<Batch> batches;
    auto align_up = [&](int64_t v) {
        const int64_t q = 256 / (int64_t)es;
        return (v + q - 1) / q * q;
    };
    auto add = [&](Batch &b, int64_t t) {
        b.tiles.push_back(t);
        b.src_off.push_back(b.src_total);
        b.out_off.push_back(b.out_total);
        b.src_total += align_up(srcs[t].count());
        b.out_total += align_up(tiles[t].count());
    };
    for (int64_t t = 0; t < ntiles; ++t)
        if (tiles[t].count() == full) {
            batches.emplace_back();
            add(batches.back(), t);
        }
    {
        Batch b;
        int64_t out = 0;
        for (int64_t t = 0; t < ntiles; ++t) {
            if (tiles[t].count() == full) continue;
            if (!b.tiles.empty() && (out + tiles[t].count() > full || (int64_t)b.tiles.size() >= tw_ctx::kJobsPerSlot)) {
                batches.push_back(std::move(b));
                b = Batch();
                out = 0;
            }
            add(b, t);
            out += tiles[t].count();
        }
        if (!b.tiles.empty()) batches.push_back(std::move(b));
    }
    int64_t max_src = 1, max_out = 1;
    for (const Batch &b : batches) {
        max_src = std::max(max_src, b.src_total);
        max_out = std::max(max_out, b.out_total);
    }

    // the built-in host-volume reader/writer on pinned memory become DMA copies
    const tw_host_volume *hv_in = io.read == tw_box_reader_host ? static_cast<const tw_host_volume *>(io.read_user)
                                                                  : nullptr;
    const tw_host_volume *hv_out = io.write == tw_box_writer_host ? static_cast<const tw_host_volume *>(io.write_user)
                                                                    : nullptr;
    const bool dma_in = hv_in && is_pinned_ptr(hv_in->data);
    const bool dma_out = hv_out && is_pinned_ptr(hv_out->data);
    for (int a = 0; a < 3; ++a) {
        if (hv_in && (hv_in->sz[a] != src_sz[a] || hv_in->dtype != dtype))
            return fail(ctx, TW_ERR_ARG, "tile source volume does not match the source dims / dtype");
        if (hv_out && (hv_out->sz[a] != out_sz[a] || hv_out->dtype != dtype))
            return fail(ctx, TW_ERR_ARG, "tile sink volume does not match the output dims / dtype");
    }

    std::vector<Slot> slots(depth);
    struct Cleanup {
        tw_ctx *ctx;
        std::vector<Slot> &s;
        size_t sb, ob;
        ~Cleanup()
        {
            for (auto &x : s) {
                if (x.d_src) dfree(ctx, x.d_src, sb);
                if (x.d_dst) dfree(ctx, x.d_dst, ob);
                if (x.h_src) cudaFreeHost(x.h_src);
                if (x.h_dst) cudaFreeHost(x.h_dst);
                if (x.e_in) cudaEventDestroy(x.e_in);
                if (x.e_comp) cudaEventDestroy(x.e_comp);
                if (x.e_out) cudaEventDestroy(x.e_out);
            }
        }
    } cleanup{ctx, slots, (size_t)max_src * es, (size_t)max_out * es};
    for (auto &s : slots) {
        TW_TRY(dmalloc(ctx, &s.d_src, (size_t)max_src * es));
        TW_TRY(dmalloc(ctx, &s.d_dst, (size_t)max_out * es));
        if (!dma_in) TW_CUDA_TRY(cudaHostAlloc(&s.h_src, (size_t)max_src * es, cudaHostAllocDefault));
        if (!dma_out) TW_CUDA_TRY(cudaHostAlloc(&s.h_dst, (size_t)max_out * es, cudaHostAllocDefault));
        TW_CUDA_TRY(cudaEventCreateWithFlags(&s.e_in, cudaEventDisableTiming));
        TW_CUDA_TRY(cudaEventCreateWithFlags(&s.e_comp, cudaEventDisableTiming));
        TW_CUDA_TRY(cudaEventCreateWithFlags(&s.e_out, cudaEventDisableTiming));
    }

    // hands a finished batch's tiles to the sink (after their D2H completed)
    auto retire = [&](Slot &s) -> tw_status {
        if (s.batch < 0) return TW_OK;
        TW_CUDA_TRY(cudaEventSynchronize(s.e_out));
        const Batch &bt = batches[s.batch];
        if (!dma_out && io.write) {
            for (size_t i = 0; i < bt.tiles.size(); ++i) {
                const int64_t t = bt.tiles[i];
                const Box &b = tiles[t];
                const char *h = static_cast<const char *>(s.h_dst) + (size_t)bt.out_off[i] * es;
                if (io.write(io.write_user, b.o[0], b.o[1], b.o[2], b.n[0], b.n[1], b.n[2], h) != 0)
                    return fail(ctx, TW_ERR_IO, "tile sink failed at tile " + std::to_string(t));
            }
        }
        s.batch = -1;
        return TW_OK;
    };

    std::vector<RJob> jobs;
    for (int64_t bi = 0; bi < (int64_t)batches.size(); ++bi) {
        Slot &s = slots[bi % depth];
        TW_TRY(retire(s));  // frees the slot's pinned output and, transitively, its device buffers
        const Batch &bt = batches[bi];
        // 1. source boxes -> device slot
        for (size_t i = 0; i < bt.tiles.size(); ++i) {
            const int64_t t = bt.tiles[i];
            const Box &sb = srcs[t];
            if (sb.count() == 0) continue;
            char *d = static_cast<char *>(s.d_src) + (size_t)bt.src_off[i] * es;
            const int64_t zero[3] = {0, 0, 0};
            if (dma_in) {
                TW_CUDA_TRY(copy_box(d, hv_in->data, sb.n[0], sb.n[1], zero, hv_in->sz[0], hv_in->sz[1], sb.o, sb.n,
                                     es, cudaMemcpyHostToDevice, ctx->h2d));
            } else {
                if (!io.read) return fail(ctx, TW_ERR_ARG, "no tile source");
                char *h = static_cast<char *>(s.h_src) + (size_t)bt.src_off[i] * es;
                if (io.read(io.read_user, sb.o[0], sb.o[1], sb.o[2], sb.n[0], sb.n[1], sb.n[2], h) != 0)
                    return fail(ctx, TW_ERR_IO, "tile source failed at tile " + std::to_string(t));
                TW_CUDA_TRY(cudaMemcpyAsync(d, h, (size_t)sb.count() * es, cudaMemcpyHostToDevice, ctx->h2d));
            }
        }
        for (int64_t t : bt.tiles) ctx->h2d_bytes += (uint64_t)srcs[t].count() * es;
        TW_CUDA_TRY(cudaEventRecord(s.e_in, ctx->h2d));
        // 2. warp the batch's tiles in one launch (tiles no sample of which
        // lands in the volume are zeroed instead)
        TW_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, s.e_in, 0));
        jobs.clear();
        for (size_t i = 0; i < bt.tiles.size(); ++i) {
            const int64_t t = bt.tiles[i];
            const Box &tb = tiles[t];
            const Box &sb = srcs[t];
            char *dd = static_cast<char *>(s.d_dst) + (size_t)bt.out_off[i] * es;
            if (sb.count() == 0) {
                TW_CUDA_TRY(cudaMemsetAsync(dd, 0, (size_t)tb.count() * es, ctx->stream));
                continue;
            }
            const char *ds = static_cast<const char *>(s.d_src) + (size_t)bt.src_off[i] * es;
            RJob j = kind == 1 ? tps_job(ds, src_sz, dd, out_sz, nodes, g, dtype, interp)
                               : affine_job(ds, src_sz, dd, out_sz, M, dtype, interp);
            for (int a = 0; a < 3; ++a) {
                j.src_o[a] = sb.o[a];
                j.src_n[a] = sb.n[a];
                j.out_o[a] = tb.o[a];
                j.out_n[a] = tb.n[a];
            }
            j.src_py = sb.n[0];
            j.src_pz = sb.n[0] * sb.n[1];
            j.dst_py = tb.n[0];
            j.dst_pz = tb.n[0] * tb.n[1];
            jobs.push_back(j);
        }
        if (!jobs.empty()) TW_TRY(run_jobs(ctx, jobs.data(), (int)jobs.size(), ctx->stream));
        TW_CUDA_TRY(cudaEventRecord(s.e_comp, ctx->stream));
        // 3. tiles -> host (retire() has already waited for this slot's
        // previous batch, so its buffers are free for the next use)
        TW_CUDA_TRY(cudaStreamWaitEvent(ctx->d2h, s.e_comp, 0));
        const int64_t zero[3] = {0, 0, 0};
        for (size_t i = 0; i < bt.tiles.size(); ++i) {
            const int64_t t = bt.tiles[i];
            const Box &tb = tiles[t];
            const char *dd = static_cast<const char *>(s.d_dst) + (size_t)bt.out_off[i] * es;
            if (dma_out) {
                TW_CUDA_TRY(copy_box(hv_out->data, dd, hv_out->sz[0], hv_out->sz[1], tb.o, tb.n[0], tb.n[1], zero,
                                     tb.n, es, cudaMemcpyDeviceToHost, ctx->d2h));
            } else {
                char *h = static_cast<char *>(s.h_dst) + (size_t)bt.out_off[i] * es;
                TW_CUDA_TRY(cudaMemcpyAsync(h, dd, (size_t)tb.count() * es, cudaMemcpyDeviceToHost, ctx->d2h));
            }
        }
        for (int64_t t : bt.tiles) ctx->d2h_bytes += (uint64_t)tiles[t].count() * es;
        TW_CUDA_TRY(cudaEventRecord(s.e_out, ctx->d2h));
        s.batch = bi;
    }
    const int64_t nb = (int64_t)batches.size();
    for (int64_t bi = std::max<int64_t>(0, nb - depth); bi < nb; ++bi) TW_TRY(retire(slots[bi % depth]));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->h2d));
    TW_CUDA_TRY(cudaStreamSynchronize(ctx->d2h));
    return check_kernel_errors(ctx);
}

void copy_rows(char *dst, const char *src, int64_t nrows, size_t row_bytes, int64_t dst_pitch, int64_t src_pitch,
               int threads)
{
    auto work = [&](int64_t r0, int64_t r1) {
        for (int64_t r = r0; r < r1; ++r) std::memcpy(dst + r * dst_pitch, src + r * src_pitch, row_bytes);
    };
    if (threads <= 1 || nrows < 64) {
        work(0, nrows);
        return;
    }
    std::vector<std::thread> th;
    const int64_t per = (nrows + threads - 1) / threads;
    for (int i = 0; i < threads; ++i) {
        const int64_t r0 = i * per, r1 = std::min(nrows, r0 + per);
        if (r0 < r1) th.emplace_back(work, r0, r1);
    }
    for (auto &x : th) x.join();
}

// ------------------------------------------------------------- autotuner

std::mutex g_tune_mu;
std::map<std::string, tw_tile_candidate> g_tune_cache;  // choices made in this process

std::string tune_key(const int64_t sz[3], int dtype, int g, int n, const std::string &device)
{
    int64_t bucket = 0;
    if (n > 0)
        for (bucket = 1; bucket < n; bucket <<= 1) {
        }
    std::ostringstream k;
    k << "tps:" << sz[0] << "x" << sz[1] << "x" << sz[2] << ":" << (dtype == TW_U8 ? "u8" : "u16") << ":g" << g
      << ":n" << bucket << ":" << device;
    return k.str();
}

bool cache_file_lookup(const char *path, const std::string &key, tw_tile_candidate &out)
{
    std::ifstream f(path);
    if (!f) return false;
    bool found = false;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        std::string k;
        tw_tile_candidate c{};
        if (in >> k >> c.tile[0] >> c.tile[1] >> c.tile[2] >> c.staging_depth >> c.seconds && k == key) {
            out = c;
            found = true;  // the last line of a key wins
        }
    }
    return found;
}

void cache_file_store(const char *path, const std::string &key, const tw_tile_candidate &c)
{
    std::ofstream f(path, std::ios::app);
    if (f) f << key << " " << c.tile[0] << " " << c.tile[1] << " " << c.tile[2] << " " << c.staging_depth << " "
             << c.seconds << "\n";
}

// A sink that discards the tiles (the tuner times the pipeline, not a sink).
int discard_box(void *, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, const void *) { return 0; }

}  // namespace

extern "C" {

tw_status tw_tune_tiled_tps(tw_ctx *ctx, const tw_marker *ql_marker_tar, const tw_marker *ql_marker_sub, int n,
                            double marker_scale, int g, int dtype, const int64_t sz[3], tw_read_box_fn read_box,
                            void *read_user, tw_tile_candidate *cands, int ncands, const int64_t sample[3],
                            const char *cache_path, tw_tile_opts *best)
{
    if (!sz || !best || (dtype != TW_U8 && dtype != TW_U16) || !g_supported(g)) return TW_ERR_ARG;
    std::string device;
    if (ctx) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) return fail(ctx, TW_ERR_CUDA, "device query");
        device = prop.name;
        for (char &ch : device)
            if (ch == ' ') ch = '_';
    }
    const std::string key = tune_key(sz, dtype, g, n, device);
    auto give = [&](const tw_tile_candidate &c) {
        std::memset(best, 0, sizeof(*best));
        for (int a = 0; a < 3; ++a) best->tile[a] = c.tile[a];
        best->staging_depth = c.staging_depth;
        return TW_OK;
    };
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return give(it->second);
    }
    tw_tile_candidate hit{};
    if (cache_path && cache_file_lookup(cache_path, key, hit)) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = hit;
        return give(hit);
    }
    if (!ctx) return TW_ERR_NOT_READY;
    if (!ql_marker_tar || !ql_marker_sub || n < 4 || !read_box) return fail(ctx, TW_ERR_ARG, "tuning needs the job's landmarks and source");
    static const tw_tile_candidate kDefault[] = {
        {{512, 512, 512}, 2, 0}, {{512, 512, 512}, 3, 0}, {{1024, 1024, 256}, 2, 0},
        {{1024, 1024, 256}, 3, 0}, {{2048, 1024, 128}, 3, 0}, {{256, 256, 256}, 4, 0}};
    std::vector<tw_tile_candidate> list;
    if (cands && ncands > 0) list.assign(cands, cands + ncands);
    else list.assign(kDefault, kDefault + sizeof(kDefault) / sizeof(kDefault[0]));
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    // the job's field, once: solve + node grid of the whole volume
    tw_tps *tp = nullptr;
    TW_TRY(make_tps(ctx, ql_marker_sub, ql_marker_tar, n, 0.2, marker_scale > 0 ? marker_scale : 1.0, ctx->stream, &tp));
    std::unique_ptr<tw_tps, void (*)(tw_tps *)> guard(tp, destroy_tps);
    const int64_t gsz[3] = {grid_size(sz[0], g), grid_size(sz[1], g), grid_size(sz[2], g)};
    void *nodes = nullptr;
    const size_t nbytes = sizeof(float4) * (size_t)(gsz[0] * gsz[1] * gsz[2]);
    TW_TRY(dmalloc(ctx, &nodes, nbytes));
    struct NodeGuard {
        tw_ctx *c; void *p; size_t b;
        ~NodeGuard() { cudaStreamSynchronize(c->stream); dfree(c, p, b); }
    } ng{ctx, nodes, nbytes};
    const int64_t off[3] = {0, 0, 0};
    TW_TRY(eval_grid(ctx, tp, gsz, g, off, static_cast<float4 *>(nodes), ctx->stream));
    const int64_t sdef[3] = {1024, 1024, 512};
    TileIO io{read_box, read_user, discard_box, nullptr};
    auto time_one = [&](const tw_tile_candidate &c, double &secs) -> tw_status {
        tw_tile_opts o;
        std::memset(&o, 0, sizeof(o));
        for (int a = 0; a < 3; ++a) {
            o.tile[a] = c.tile[a];
            o.region_o[a] = 0;
            o.region_n[a] = std::min(sz[a], sample && sample[a] > 0 ? sample[a] : sdef[a]);
        }
        o.staging_depth = c.staging_depth;
        const auto t0 = std::chrono::steady_clock::now();
        TW_TRY(run_tiled(ctx, 1, static_cast<const float4 *>(nodes), g, nullptr, dtype, 0, sz, sz, io, &o));
        secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return TW_OK;
    };
    double warm = 0;
    TW_TRY(time_one(list[0], warm));  // the first run pays one-time set-up
    size_t bi = 0;
    for (size_t i = 0; i < list.size(); ++i) {
        TW_TRY(time_one(list[i], list[i].seconds));
        if (list[i].seconds < list[bi].seconds) bi = i;
    }
    if (cands && ncands > 0)
        for (int i = 0; i < ncands; ++i) cands[i].seconds = list[(size_t)i].seconds;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = list[bi];
    }
    if (cache_path) cache_file_store(cache_path, key, list[bi]);
    return give(list[bi]);
}

int tw_box_reader_host(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz, void *dst)
{
    const tw_host_volume *v = static_cast<const tw_host_volume *>(user);
    if (!v || !v->data || !dst) return 1;
    const size_t es = esize(v->dtype);
    if (x0 < 0 || y0 < 0 || z0 < 0 || x0 + nx > v->sz[0] || y0 + ny > v->sz[1] || z0 + nz > v->sz[2]) return 2;
    // row r of the box = (y, z) = (r % ny, r / ny)
    const int threads = v->threads > 0 ? v->threads : (int)std::max(1u, std::thread::hardware_concurrency() / 2);
    auto work = [&](int64_t r0, int64_t r1) {
        for (int64_t r = r0; r < r1; ++r) {
            const int64_t y = r % ny, z = r / ny;
            std::memcpy(static_cast<char *>(dst) + (size_t)r * nx * es,
                        static_cast<const char *>(v->data) + (((z0 + z) * v->sz[1] + (y0 + y)) * v->sz[0] + x0) * es,
                        (size_t)nx * es);
        }
    };
    const int64_t rows = ny * nz;
    if (threads <= 1 || rows < 64) {
        work(0, rows);
        return 0;
    }
    std::vector<std::thread> th;
    const int64_t per = (rows + threads - 1) / threads;
    for (int i = 0; i < threads; ++i) {
        const int64_t r0 = i * per, r1 = std::min(rows, r0 + per);
        if (r0 < r1) th.emplace_back(work, r0, r1);
    }
    for (auto &x : th) x.join();
    return 0;
}

int tw_box_writer_host(void *user, int64_t x0, int64_t y0, int64_t z0, int64_t nx, int64_t ny, int64_t nz,
                       const void *src)
{
    const tw_host_volume *v = static_cast<const tw_host_volume *>(user);
    if (!v || !v->data || !src) return 1;
    const size_t es = esize(v->dtype);
    if (x0 < 0 || y0 < 0 || z0 < 0 || x0 + nx > v->sz[0] || y0 + ny > v->sz[1] || z0 + nz > v->sz[2]) return 2;
    const int threads = v->threads > 0 ? v->threads : (int)std::max(1u, std::thread::hardware_concurrency() / 2);
    for (int64_t z = 0; z < nz; ++z)
        copy_rows(static_cast<char *>(v->data) + (((z0 + z) * v->sz[1] + y0) * v->sz[0] + x0) * es,
                  static_cast<const char *>(src) + (size_t)z * nx * ny * es, ny, (size_t)nx * es,
                  (int64_t)(v->sz[0] * es), (int64_t)(nx * es), nz > 1 ? 1 : threads);
    return 0;
}

tw_status tw_imgwarp_smallmemory_tiled(tw_ctx *ctx, const tw_marker *ql_marker_tar, const tw_marker *ql_marker_sub,
                                       int n, double marker_scale, int g, int dtype, const int64_t sz[3],
                                       tw_read_box_fn read_box, void *read_user, tw_write_box_fn write_box,
                                       void *write_user, const tw_tile_opts *opts)
{
    if (!ctx || !sz) return TW_ERR_ARG;
    if (!ql_marker_tar || !ql_marker_sub || n <= 0) return fail(ctx, TW_ERR_ARG, "target or subject control points is invalid");
    if (!g_supported(g)) return fail(ctx, TW_ERR_UNSUPPORTED, "grid spacing must be 4, 8, 16, 32 or 64");
    if (dtype != TW_U8 && dtype != TW_U16) return fail(ctx, TW_ERR_ARG, "dtype must be TW_U8 or TW_U16");
    for (int a = 0; a < 3; ++a)
        if (sz[a] < 1) return fail(ctx, TW_ERR_ARG, "volume size is invalid");
    if (!read_box || !write_box) return fail(ctx, TW_ERR_ARG, "tile source and sink are required");
    const int interp = opts ? opts->interp : 0;
    if (interp != 0 && interp != 1) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    const double scale = marker_scale > 0 ? marker_scale : 1.0;
    tw_tps *tp = nullptr;
    // the reference solves once per job with the markers scaled by 4
    // (q_imgwarp_tps_quicksmallmemory.cpp:1194-1203, :1212)
    TW_TRY(make_tps(ctx, ql_marker_sub, ql_marker_tar, n, 0.2, scale, ctx->stream, &tp));
    std::unique_ptr<tw_tps, void (*)(tw_tps *)> guard(tp, destroy_tps);
    const int64_t gsz[3] = {grid_size(sz[0], g), grid_size(sz[1], g), grid_size(sz[2], g)};
    void *nodes = nullptr;
    const size_t nbytes = sizeof(float4) * (size_t)(gsz[0] * gsz[1] * gsz[2]);
    TW_TRY(dmalloc(ctx, &nodes, nbytes));
    const int64_t off[3] = {0, 0, 0};
    tw_status s = eval_grid(ctx, tp, gsz, g, off, static_cast<float4 *>(nodes), ctx->stream);
    if (s == TW_OK) {
        TileIO io{read_box, read_user, write_box, write_user};
        s = run_tiled(ctx, 1, static_cast<const float4 *>(nodes), g, nullptr, dtype, interp, sz, sz, io, opts);
    }
    cudaStreamSynchronize(ctx->stream);
    dfree(ctx, nodes, nbytes);
    return s;
}

tw_status tw_warp_affine_tiled(tw_ctx *ctx, const double M[16], int dtype, const int64_t src_sz[3],
                               const int64_t out_sz[3], tw_read_box_fn read_box, void *read_user,
                               tw_write_box_fn write_box, void *write_user, const tw_tile_opts *opts)
{
    if (!ctx || !M || !src_sz || !out_sz) return TW_ERR_ARG;
    if (dtype != TW_U8 && dtype != TW_U16) return fail(ctx, TW_ERR_ARG, "dtype must be TW_U8 or TW_U16");
    for (int a = 0; a < 3; ++a)
        if (src_sz[a] < 1 || out_sz[a] < 1) return fail(ctx, TW_ERR_ARG, "volume size is invalid");
    if (!read_box || !write_box) return fail(ctx, TW_ERR_ARG, "tile source and sink are required");
    const int interp = opts ? opts->interp : 0;
    if (interp != 0 && interp != 1) return TW_ERR_ARG;
    TW_CUDA_TRY(cudaSetDevice(ctx->device));
    TileIO io{read_box, read_user, write_box, write_user};
    return run_tiled(ctx, 0, nullptr, 0, M, dtype, interp, src_sz, out_sz, io, opts);
}

}  // extern "C"
