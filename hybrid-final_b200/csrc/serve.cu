// serve.cu -- request loop over resident cases (continuous batching).
#include <cuda_runtime.h>

#include "capi_internal.hpp"

extern "C" {
hp_status hp_server_create(const hp_server_opts *, hp_server **) {
    hpi::set_error("server not built yet");
    return HP_ERR_UNSUPPORTED;
}
hp_status hp_server_destroy(hp_server *) { return HP_OK; }
hp_status hp_server_submit(hp_server *, const char *, size_t, int64_t, uint64_t, int64_t *) { return HP_ERR_UNSUPPORTED; }
hp_status hp_server_poll(hp_server *, void *, int *) { return HP_ERR_UNSUPPORTED; }
hp_status hp_server_take_result(hp_server *, hp_result *, double *, size_t, double *, size_t, int *) {
    return HP_ERR_UNSUPPORTED;
}
}
