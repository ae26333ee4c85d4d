// tw_host.h -- host-side helpers shared by the ABI translation units.
#pragma once

#include "tw_internal.h"

#include <functional>
#include <vector>

namespace tw {

bool is_device_ptr(const void *p);
bool is_pinned_ptr(const void *p);

// wait = false queues the whole solve on `st` and returns at once; the
// solve's status is then read with solve_status(ctx, t->d_status, st).
// h_stage: optional pinned staging for the landmark uploads (solve_tps_device).
tw_status make_tps(tw_ctx *ctx, const tw_marker *centres, const tw_marker *values, int n, double lambda,
                   double scale, cudaStream_t st, tw_tps **out, bool wait = true, double *h_stage = nullptr);
void destroy_tps(tw_tps *t);
tw_status eval_grid(tw_ctx *ctx, const tw_tps *t, const int64_t gsz[3], int g, const int64_t off[3], float4 *out,
                    cudaStream_t st);

// Whole-volume resample jobs (the region can be narrowed afterwards).
RJob tps_job(const void *src, const int64_t src_sz[3], void *dst, const int64_t dst_sz[3], const float4 *nodes, int g,
             int dtype, int interp);
RJob affine_job(const void *src, const int64_t src_sz[3], void *dst, const int64_t dst_sz[3], const double M[16],
                int dtype, int interp);
// Launches the jobs (all sharing dtype, kind, g, interp) in one persistent
// resample launch on `st`.  Fills brick counts and prefix sums.
tw_status run_jobs(tw_ctx *ctx, RJob *jobs, int njobs, cudaStream_t st);

// Per output cell-layer z hull of the TPS sample positions: for layer cz
// (output z in [cz*g, (cz+1)*g)), zmin/zmax of q_z.  Host vectors of size
// gsz[2]-3.
tw_status tps_layer_zhull(tw_ctx *ctx, const float4 *nodes, const int64_t gsz[3], int g, cudaStream_t st,
                          std::vector<float> &zmin, std::vector<float> &zmax);
// Per-box hull of TPS sample positions over the node grid: for each output
// box (in cells) [c0, c1) the min/max of q over its node support.
struct CellBox { int64_t c0[3], c1[3]; };
tw_status tps_box_hull(tw_ctx *ctx, const float4 *nodes, const int64_t gsz[3], int g,
                       const std::vector<CellBox> &boxes, cudaStream_t st, std::vector<float> &lo,
                       std::vector<float> &hi);

tw_status make_param_affine(int warp_mode, int deformation_mode, const double para[3], const int64_t in_sz[3],
                            const int64_t out_sz[3], double M[16]);

// Slab pipeline: streams a host (or device) source volume into HBM in z
// chunks and the output back in z slabs, overlapping H2D, compute and D2H on
// three streams.  `need(z0, z1, &lo, &hi)` returns the inclusive source z
// range output planes [z0, z1) read; `compute(z0, z1, d_src, d_dst, st)`
// enqueues the resample of those planes.
struct SlabIO {
    const void *src;          // host or device, src_planes x src_plane_bytes
    void *dst;                // host or device, dst_planes x dst_plane_bytes
    size_t src_plane_bytes, dst_plane_bytes;
    int64_t src_planes, dst_planes;
    int64_t slab;             // output planes per slab (multiple of g for TPS)
};
tw_status stream_slabs(tw_ctx *ctx, const SlabIO &io,
                       const std::function<void(int64_t, int64_t, int64_t &, int64_t &)> &need,
                       const std::function<tw_status(int64_t, int64_t, const void *, void *, cudaStream_t)> &compute);

}  // namespace tw
