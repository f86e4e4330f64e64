// Library-level entry points of libbugdef.so: status plumbing and device queries.
#include <atomic>

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

static std::atomic<int> g_tune[BD_TUNE_COUNT] = {{0}, {8}, {4}, {BD_PLUME_KERNEL_DIRECT}, {0}};
static std::atomic<int> g_tune_gen{0};

int tune_value(int knob) { return g_tune[knob].load(std::memory_order_relaxed); }
int tune_generation() { return g_tune_gen.load(std::memory_order_relaxed); }

}  // namespace bd

using namespace bd;

extern "C" int bd_tune_set(int knob, int value) {
    BD_REQUIRE(knob >= 0 && knob < BD_TUNE_COUNT, "bd_tune_set: unknown knob %d", knob);
    if (knob == BD_TUNE_MC_BLOCKS_PER_SM)
        BD_REQUIRE(value >= 0 && value <= 16, "bd_tune_set: MC CTAs per SM must be 0..16, got %d", value);
    else if (knob == BD_TUNE_STENCIL_CAP)
        BD_REQUIRE(value >= 0 && value <= 16, "bd_tune_set: substep CTAs per SM cap must be 0..16, got %d", value);
    else if (knob == BD_TUNE_PLUME_KERNEL)
        BD_REQUIRE(value == BD_PLUME_KERNEL_DIRECT || value == BD_PLUME_KERNEL_COMPACT,
                   "bd_tune_set: plume kernel must be %d (direct) or %d (compact), got %d", BD_PLUME_KERNEL_DIRECT,
                   BD_PLUME_KERNEL_COMPACT, value);
    else
        BD_REQUIRE(value >= 1 && value <= 64, "bd_tune_set: x-planes per CTA must be 1..64, got %d", value);
    if (g_tune[knob].exchange(value) != value) g_tune_gen.fetch_add(1);
    return BD_OK;
}

extern "C" int bd_tune_get(int knob, int* value) {
    BD_REQUIRE(knob >= 0 && knob < BD_TUNE_COUNT, "bd_tune_get: unknown knob %d", knob);
    BD_REQUIRE(value != nullptr, "bd_tune_get: value is NULL");
    *value = tune_value(knob);
    return BD_OK;
}

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
