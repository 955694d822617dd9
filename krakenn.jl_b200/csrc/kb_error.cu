// kb_error.cu -- error state, version and synchronisation entry points.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "kb_common.cuh"

namespace kb {

static thread_local char g_err[1024] = "";

int set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_err[0] = '\0'; }

int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(KB_ERR_CUDA, "%s: launch failed: %s", what, cudaGetErrorString(e));
    return KB_OK;
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

}  // namespace kb

extern "C" {

const char *kb_version(void) { return "krakenb200 0.1.0 sm_100a"; }

const char *kb_last_error(void) { return kb::g_err; }

int kb_sync(void *stream) {
    cudaError_t e = cudaStreamSynchronize(kb::as_stream(stream));
    if (e != cudaSuccess)
        return kb::set_error(KB_ERR_CUDA, "kb_sync: %s", cudaGetErrorString(e));
    return KB_OK;
}

}  // extern "C"
