// tw_stubs.cpp -- entry points declared in the ABI whose implementation
// lands in a later file; they fail loudly instead of falling back.
#include "tw_host.h"

extern "C" {

tw_status tw_imgwarp_smallmemory_tiled(tw_ctx *ctx, const tw_marker *, const tw_marker *, int, double, int, int,
                                       const int64_t *, tw_read_box_fn, void *, tw_write_box_fn, void *,
                                       const tw_tile_opts *)
{
    return tw::fail(ctx, TW_ERR_UNSUPPORTED, "tiled TPS not built");
}

tw_status tw_warp_affine_tiled(tw_ctx *ctx, const double *, int, const int64_t *, const int64_t *, tw_read_box_fn,
                               void *, tw_write_box_fn, void *, const tw_tile_opts *)
{
    return tw::fail(ctx, TW_ERR_UNSUPPORTED, "tiled affine not built");
}

tw_status tw_server_create(tw_ctx *, size_t, int, tw_server **) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_submit(tw_server *, const tw_job *, uint64_t *) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_poll(tw_server *, uint64_t, double *) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_wait(tw_server *, uint64_t, double, double *) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_destroy(tw_server *) { return TW_ERR_UNSUPPORTED; }
}
