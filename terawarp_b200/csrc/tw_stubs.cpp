// tw_stubs.cpp -- entry points declared in the ABI whose implementation
// lands in a later file; they fail loudly instead of falling back.
#include "tw_host.h"

extern "C" {

tw_status tw_server_create(tw_ctx *, size_t, int, tw_server **) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_submit(tw_server *, const tw_job *, uint64_t *) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_poll(tw_server *, uint64_t, double *) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_wait(tw_server *, uint64_t, double, double *) { return TW_ERR_UNSUPPORTED; }
tw_status tw_server_destroy(tw_server *) { return TW_ERR_UNSUPPORTED; }
}
