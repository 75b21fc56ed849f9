// Context, error reporting and budgeted device memory (the role of xmvb::cuda::Context,
// src/cuda/memory/context.hpp:66-405 in the reference: one device, one stream, a byte budget
// of 90 % of free HBM by default, allocation counters).
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>

#include "internal.h"
#include "kernels.h"

namespace {
std::mutex g_error_mutex;
std::string g_create_error;
}  // namespace

namespace vbcore {

vb_status set_error(vb_context* ctx, vb_status code, const std::string& message) {
    if (ctx) {
        ctx->last_error = message;
    } else {
        std::lock_guard<std::mutex> lock(g_error_mutex);
        g_create_error = message;
    }
    return code;
}

vb_status cuda_error(vb_context* ctx, cudaError_t err, const char* what) {
    return set_error(ctx, VB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

void* device_alloc(vb_context* ctx, size_t bytes, vb_status* status) {
    if (ctx->current + bytes > ctx->budget) {
        *status = set_error(ctx, VB_ERR_BUDGET,
                            "device budget exceeded: requested " + std::to_string(bytes) + " bytes with " +
                                std::to_string(ctx->current) + " of " + std::to_string(ctx->budget) + " in use");
        return nullptr;
    }
    void* p = nullptr;
    cudaError_t err = ctx->pool ? cudaMallocFromPoolAsync(&p, bytes, ctx->pool, ctx->stream)
                                : cudaMallocAsync(&p, bytes, ctx->stream);
    if (err != cudaSuccess) {
        *status = cuda_error(ctx, err, "cudaMallocAsync");
        return nullptr;
    }
    ctx->current += bytes;
    if (ctx->current > ctx->peak) ctx->peak = ctx->current;
    *status = VB_OK;
    return p;
}

void device_free(vb_context* ctx, void* ptr, size_t bytes) {
    if (!ptr) return;
    cudaFreeAsync(ptr, ctx->stream);
    ctx->current -= bytes;
}

cudaError_t allow_dynamic_smem(const void* kernel, size_t bytes) {
    static std::mutex mutex;
    static std::map<std::pair<const void*, int>, size_t> raised;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    std::lock_guard<std::mutex> lock(mutex);
    const auto key = std::make_pair(kernel, dev);
    const auto it = raised.find(key);
    if (it != raised.end() && it->second >= bytes) return cudaSuccess;
    int optin = 0;
    if ((err = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return err;
    cudaFuncAttributes fa{};
    if ((err = cudaFuncGetAttributes(&fa, kernel)) != cudaSuccess) return err;
    const size_t limit = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
    if (bytes > limit) return cudaErrorInvalidValue;
    if ((err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit)) != cudaSuccess)
        return err;
    raised[key] = limit;
    return cudaSuccess;
}

cudaError_t reserve_kernel_stack() {
    static std::mutex stack_mutex;
    std::lock_guard<std::mutex> lock(stack_mutex);
    const size_t need = std::max(exact_stack_bytes(), gradient_stack_bytes()) + 1024;
    size_t have = 0;
    cudaError_t err = cudaDeviceGetLimit(&have, cudaLimitStackSize);
    if (err != cudaSuccess) return err;
    if (have < need) err = cudaDeviceSetLimit(cudaLimitStackSize, need);
    return err;
}

void* context_scratch(vb_context* ctx, int slot, size_t bytes, vb_status* status) {
    *status = VB_OK;
    if (bytes == 0) bytes = 16;
    if (ctx->scratch_bytes[slot] >= bytes) return ctx->scratch[slot];
    device_free(ctx, ctx->scratch[slot], ctx->scratch_bytes[slot]);
    ctx->scratch[slot] = nullptr;
    ctx->scratch_bytes[slot] = 0;
    void* p = device_alloc(ctx, bytes, status);
    if (p) {
        ctx->scratch[slot] = p;
        ctx->scratch_bytes[slot] = bytes;
    }
    return p;
}

}  // namespace vbcore

using namespace vbcore;

extern "C" {

vb_status vb_context_create(int device, size_t hbm_budget_bytes, vb_context** out) {
    if (!out) return set_error(nullptr, VB_ERR_INVALID, "vb_context_create: out is null");
    *out = nullptr;
    int count = 0;
    cudaError_t err = cudaGetDeviceCount(&count);
    if (err != cudaSuccess || count == 0)
        return set_error(nullptr, VB_ERR_CUDA,
                         std::string("no CUDA device available: ") + cudaGetErrorString(err));
    if (device < 0 || device >= count) return set_error(nullptr, VB_ERR_INVALID, "device index out of range");
    cudaDeviceProp prop;
    err = cudaGetDeviceProperties(&prop, device);
    if (err != cudaSuccess) return set_error(nullptr, VB_ERR_CUDA, "cudaGetDeviceProperties failed");
    if (prop.major < 10)
        return set_error(nullptr, VB_ERR_UNSUPPORTED,
                         std::string("vbcore is built for sm_100a (B200); device is ") + prop.name);
    err = cudaSetDevice(device);
    if (err != cudaSuccess) return set_error(nullptr, VB_ERR_CUDA, "cudaSetDevice failed");
    vb_context* ctx = new (std::nothrow) vb_context();
    if (!ctx) return set_error(nullptr, VB_ERR_INVALID, "out of host memory");
    ctx->device = device;
    err = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        delete ctx;
        return set_error(nullptr, VB_ERR_CUDA, "cudaStreamCreate failed");
    }
    ctx->stream = ctx->own_stream;
    // a private pool whose freed blocks stay mapped between calls (a release threshold of 0,
    // the default pool's, would unmap them at every synchronization and re-map on the next call)
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&ctx->pool, &props) == cudaSuccess) {
        uint64_t keep = ~uint64_t{0};
        cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
        ctx->pool = nullptr;
        cudaGetLastError();
    }
    // Reserve the stack the exact-path kernels need once, up front (reserve_kernel_stack).
    reserve_kernel_stack();
    cudaGetLastError();
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    ctx->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(0.9 * (double)free_b);
    *out = ctx;
    return VB_OK;
}

vb_status vb_context_destroy(vb_context* ctx) {
    if (!ctx) return VB_OK;
    DeviceGuard guard(ctx->device);
    for (int i = 0; i < 6; ++i) device_free(ctx, ctx->scratch[i], ctx->scratch_bytes[i]);
    if (ctx->own_stream) {
        cudaStreamSynchronize(ctx->own_stream);
        cudaStreamDestroy(ctx->own_stream);
    }
    if (ctx->pool) {
        cudaDeviceSynchronize();
        cudaMemPoolDestroy(ctx->pool);
    }
    delete ctx;
    return VB_OK;
}

vb_status vb_context_set_stream(vb_context* ctx, void* cuda_stream) {
    if (!ctx) return VB_ERR_INVALID;
    cudaStream_t next = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
    if (next != ctx->stream && ctx->stream) {
        // the context's scratch and pool memory are reused in stream order: let the work queued
        // on the previous stream finish before anything is queued on the new one (the caller's
        // current device is restored afterwards)
        DeviceGuard guard(ctx->device);
        cudaError_t err = cudaStreamSynchronize(ctx->stream);
        if (err != cudaSuccess) return cuda_error(ctx, err, "vb_context_set_stream");
    }
    ctx->stream = next;
    return VB_OK;
}

vb_status vb_context_set_barrier_spin_limit(vb_context* ctx, long long polls) {
    if (!ctx || polls < 0) return set_error(ctx, VB_ERR_INVALID, "vb_context_set_barrier_spin_limit: bad arguments");
    ctx->barrier_spin_limit = polls;
    return VB_OK;
}

vb_status vb_context_synchronize(vb_context* ctx) {
    if (!ctx) return VB_ERR_INVALID;
    cudaError_t err = cudaStreamSynchronize(ctx->stream);
    if (err != cudaSuccess) return cuda_error(ctx, err, "cudaStreamSynchronize");
    return VB_OK;
}

const char* vb_last_error(const vb_context* ctx) {
    if (ctx) return ctx->last_error.c_str();
    std::lock_guard<std::mutex> lock(g_error_mutex);
    return g_create_error.c_str();
}

vb_status vb_context_memory(const vb_context* ctx, size_t* current_bytes, size_t* peak_bytes) {
    if (!ctx) return VB_ERR_INVALID;
    if (current_bytes) *current_bytes = ctx->current;
    if (peak_bytes) *peak_bytes = ctx->peak;
    return VB_OK;
}

}  // extern "C"
