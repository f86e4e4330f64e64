// Library-level entry points of libbugdef.so: status plumbing and device queries.
#include "common.cuh"

#include <stdarg.h>
#include <string.h>

namespace bd {

static thread_local char g_err[512] = {0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_status(cudaError_t e, const char* what) {
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    if (e == cudaErrorMemoryAllocation) return BD_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return BD_ERR_NO_DEVICE;
    return BD_ERR_CUDA;
}

}  // namespace bd

using namespace bd;

extern "C" int bd_abi_version(void) { return BD_ABI_VERSION; }

extern "C" int bd_last_error(char* buf, size_t n) {
    if (!buf || n == 0) return BD_ERR_INVALID_ARG;
    strncpy(buf, g_err, n - 1);
    buf[n - 1] = 0;
    return BD_OK;
}

extern "C" int bd_device_count(int* count) {
    BD_REQUIRE(count != nullptr, "bd_device_count: count is NULL");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        cudaGetLastError();  // clear the sticky "no device" error
        *count = 0;
        return BD_OK;
    }
    *count = c;
    return BD_OK;
}

extern "C" int bd_device_init(int device) {
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess || c == 0) return fail(BD_ERR_NO_DEVICE, "bd_device_init: no CUDA device");
    BD_REQUIRE(device >= 0 && device < c, "bd_device_init: device %d out of range [0, %d)", device, c);
    BD_CUDA(cudaSetDevice(device));
    BD_CUDA(cudaFree(nullptr));
    return BD_OK;
}

extern "C" int bd_stream_sync(void* stream) {
    BD_CUDA(cudaStreamSynchronize(as_stream(stream)));
    BD_CUDA(cudaGetLastError());
    return BD_OK;
}
