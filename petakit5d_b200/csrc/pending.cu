// Entry points whose implementation lands in later files of this library.
#include "pk_internal.h"

extern "C" {

pk_server* pk_server_create(pk_ctx*, const pk_server_config*) { return nullptr; }
pk_status pk_server_add_psf(pk_server*, int32_t, const float*, const float*, const int64_t[3]) { return PK_ERR_UNSUPPORTED; }
int64_t pk_server_submit(pk_server*, const uint16_t*, const int64_t[3], int32_t, int32_t, int32_t,
                         const pk_decon_params*) { return -PK_ERR_UNSUPPORTED; }
pk_status pk_server_wait(pk_server*, int64_t, void*, int32_t, double*) { return PK_ERR_UNSUPPORTED; }
pk_status pk_server_cancel(pk_server*, int64_t) { return PK_ERR_UNSUPPORTED; }
pk_status pk_server_stats(pk_server*, int64_t[4]) { return PK_ERR_UNSUPPORTED; }
void pk_server_destroy(pk_server*) {}
}
