// mk_capi.cpp -- library-level entry points of the C ABI: status text,
// per-thread last error, device query, version.
#include <cuda_runtime.h>

#include <string>

#include "mk_internal.h"

namespace mk {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

}  // namespace mk

extern "C" const char *mk_status_string(int status) {
    switch (status) {
        case MK_OK: return "ok";
        case MK_ERR_INVALID_ARGUMENT: return "invalid argument";
        case MK_ERR_CUDA: return "CUDA error";
        case MK_ERR_OUT_OF_MEMORY: return "out of device memory";
        case MK_ERR_NOT_READY: return "not ready";
        case MK_ERR_BUDGET: return "device memory budget exceeded";
        case MK_ERR_TIMEOUT: return "timed out";
        case MK_ERR_NO_DEVICE: return "no CUDA device";
        case MK_ERR_QUEUE_FULL: return "queue full";
        default: return "unknown status";
    }
}

extern "C" const char *mk_last_error(void) { return mk::g_last_error.c_str(); }

extern "C" int mk_device_count(int *count) {
    if (!count) return MK_ERR_INVALID_ARGUMENT;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return MK_OK;
}

extern "C" const char *mk_version(void) { return "0.1.0"; }
