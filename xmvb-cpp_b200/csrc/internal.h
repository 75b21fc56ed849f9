// Internal declarations shared by the vbcore host and device translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "vbcore.h"

struct vb_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaMemPool_t pool = nullptr;  // the context's own stream-ordered pool (keeps freed memory)
    // grow-only execute scratch shared by every plan of this context (plans of one context run
    // in order on its stream): the determinant-pair bands and the structure-reduce buffers
    void* scratch[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    size_t scratch_bytes[6] = {0, 0, 0, 0, 0, 0};
    size_t budget = 0;
    long long barrier_spin_limit = 0;  // grid-barrier polls before a timeout (0: the built-in default)
    size_t current = 0;
    size_t peak = 0;
    std::string last_error;
};

namespace vbcore {

// Linear-dependence threshold of the reference overlap resolver
// (src/vbscf/determinants/algebra/overlap.hpp:166).
constexpr double kLinearDependenceThreshold = 1.0e-12;

// Largest electron count per spin handled by the register-resident kernels; larger blocks
// run on the local-memory exact path only.
constexpr int kMaxFastElectrons = 8;
// Largest electron count per spin supported at all, and largest active space.
constexpr int kMaxElectrons = 16;
constexpr int kMaxOrbitals = 64;

vb_status set_error(vb_context* ctx, vb_status code, const std::string& message);
vb_status cuda_error(vb_context* ctx, cudaError_t err, const char* what);

// Makes `device` current for the lifetime of the guard and restores the caller's device after.
struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
        if (previous != device) cudaSetDevice(device);
    }
    ~DeviceGuard() {
        int now = -1;
        if (previous >= 0 && cudaGetDevice(&now) == cudaSuccess && now != previous) cudaSetDevice(previous);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Raises the current device's per-thread stack limit (never lowers it) to what the exact-path
// forward and gradient kernels need, under a process-wide lock.  Without it the runtime grows
// the device's local-memory reservation at the first launch of those kernels, which can fail
// while other host threads have work in flight.
cudaError_t reserve_kernel_stack();

// U^-1 of the Cholesky factor S = U^T U of a device matrix (linalg.cu); *info > 0 when the
// leading minor of that order is not positive definite.  Synchronizes the context stream.
vb_status factor_inverse_device(vb_context* ctx, const double* M, int n, double* Ui_out, int* info);

// Blocked Cholesky on the FP64 tensor cores (cholesky_blocked.cu): U (and U^-1 when Ui is not
// null) of the device matrix M, upper triangle read, lower triangles written as zeros; `work`
// holds blocked_cholesky_workspace(n, Ui != nullptr) bytes; *info = order of the first failing
// pivot (0 on success).  Synchronizes the stream.
size_t blocked_cholesky_workspace(int n, bool inverse);
cudaError_t blocked_cholesky(const double* M, int n, double* U, double* Ui, void* work, int* info, cudaStream_t s);

// Lets `kernel` launch with up to `bytes` of dynamic shared memory on the current device.  The
// limit is a process-wide function attribute, so it is raised once per kernel and device to the
// opt-in maximum (never lowered) under a lock: threads launching the same kernel with different
// sizes cannot undo each other's setting.
cudaError_t allow_dynamic_smem(const void* kernel, size_t bytes);

// Slot `slot` (< 6) of the context's execute scratch, grown to at least `bytes` (contents are
// not kept across growth); nullptr with *status set on failure.
void* context_scratch(vb_context* ctx, int slot, size_t bytes, vb_status* status);

// Budgeted device allocation; returns nullptr (and records VB_ERR_BUDGET / VB_ERR_CUDA) on failure.
void* device_alloc(vb_context* ctx, size_t bytes, vb_status* status);
void device_free(vb_context* ctx, void* ptr, size_t bytes);

// RAII device buffer tied to a context.
struct DeviceBuffer {
    vb_context* ctx = nullptr;
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ctx(o.ctx), ptr(o.ptr), bytes(o.bytes) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            ctx = o.ctx;
            ptr = o.ptr;
            bytes = o.bytes;
            o.ptr = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    vb_status allocate(vb_context* c, size_t n) {
        release();
        ctx = c;
        vb_status st = VB_OK;
        if (n == 0) n = 16;
        ptr = device_alloc(c, n, &st);
        if (ptr) bytes = n;
        return st;
    }
    void release() {
        if (ptr) device_free(ctx, ptr, bytes);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

// Host-side structure generation and expansion (structures.cpp).
struct Expansion {
    int n_structures = 0;
    int n_alpha = 0;
    int n_beta = 0;
    std::vector<uint64_t> alpha_strings;
    std::vector<uint64_t> beta_strings;
    std::vector<int32_t> det_alpha;
    std::vector<int32_t> det_beta;
    std::vector<int64_t> offsets;
    std::vector<int32_t> term_structure;
    std::vector<double> term_coefficient;
};

std::vector<std::vector<int>> generate_structures(const std::string& keyword, int n_orb, int n_el, int mult,
                                                  int n_inactive);
Expansion expand_structures(const std::vector<std::vector<int>>& rows, int n_el_active, int mult,
                            int n_inactive);

}  // namespace vbcore
