// Allocation-free spin-pair evaluation.
//
// Some callers cannot allocate device memory at the point where they need these numbers: a
// serving loop that reserves all of its HBM up front and forbids allocation on the request
// path, an application whose own allocator already owns the device budget, or code that runs
// where the CUDA runtime's allocator must not be entered.  vb_spin_pairs_noalloc serves them:
// it evaluates every unordered pair of one spin-string table with the same kernels as the
// structure H/S plan (integral tables, pair-kernel factorization, per-left-string
// decomposition tables, register-resident spin-pair kernel, exact path) and takes all of its
// scratch from one file-scope device array instead of cudaMalloc.
//
// The first call made with a device current is that device's set-up call: it raises the
// device's stack limit to what the exact-path kernels need (so that later calls never make the
// runtime grow the local-memory reservation), loads every kernel a call may launch (so that lazy
// module loading places no code in device memory during a later call) and obtains the array's
// address with cudaGetSymbolAddress; make that first call before any stream capture.  Every call reads the pair-kernel rank back to the host midway and
// waits for the stream to reach that point.
// Every call on a device shares the array, which keeps the last call's contents: the kernels
// clear what must start at zero (the exact-path counter), and calls that overlap on the GPU
// (different streams, or different host threads) race on the array.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "internal.h"
#include "kernels.h"

namespace vbcore {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;  // 32 MiB
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_address[kMaxDevices] = {};

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Occupation rows from masks, with device-side validation (bad[0] = 1 on any invalid mask).
__global__ void occupation_rows_kernel(const uint64_t* __restrict__ masks, int count, int k, int n,
                                       uint64_t* __restrict__ rows, int* __restrict__ bad) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
        const uint64_t m = masks[s];
        uint64_t w[2] = {~uint64_t{0}, ~uint64_t{0}};
        int found = 0;
        bool ok = true;
        for (int o = 0; o < 64; ++o)
            if ((m >> o) & 1) {
                if (o >= n || found >= 16) {
                    ok = false;
                    break;
                }
                const int word = found >> 3, shift = 8 * (found & 7);
                w[word] = (w[word] & ~(uint64_t{0xFF} << shift)) | ((uint64_t)o << shift);
                ++found;
            }
        if (!ok || found != k) atomicExch(bad, 1);
        rows[2 * s] = w[0];
        rows[2 * s + 1] = w[1];
    }
}

__global__ void extract_scalars_kernel(const double* __restrict__ records, int stride, int R, long long n_pairs,
                                       double* __restrict__ out) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n_pairs;
         t += (long long)gridDim.x * blockDim.x) {
        const double* rec = records + t * stride;
        out[4 * t + 0] = rec[R + 0];
        out[4 * t + 2] = rec[R + 1];
        out[4 * t + 1] = rec[R + 2];
        out[4 * t + 3] = rec[R + 3];
    }
}

int record_stride_for(int R) { return (R + 4 + 1) / 2 * 2; }

// Loads every kernel a call may launch, so that no later call loads code into device memory.
cudaError_t preload_kernels() {
    const void* own[] = {(const void*)occupation_rows_kernel, (const void*)extract_scalars_kernel};
    for (const void* f : own) {
        cudaFuncAttributes fa{};
        const cudaError_t err = cudaFuncGetAttributes(&fa, f);
        if (err != cudaSuccess) return err;
    }
    return preload_spin_pair_kernels();
}

}  // namespace
}  // namespace vbcore

using namespace vbcore;

extern "C" vb_status vb_spin_pairs_noalloc(void* cuda_stream, int n_orbitals, int k, int n_strings,
                                           const uint64_t* strings, const double* ovlp_act, const double* h1e_act,
                                           const double* eri_packed, double* out_scalars) {
    const int n = n_orbitals;
    if (n < 1 || n > kMaxOrbitals || k < 1 || k > kMaxElectrons || k > n || n_strings < 1 || !strings || !ovlp_act ||
        !h1e_act || !eri_packed || !out_scalars)
        return set_error(nullptr, VB_ERR_INVALID, "vb_spin_pairs_noalloc: bad arguments");
    // the exact-path stack reserved by the set-up call covers the instantiations for k <= 8; a
    // larger k would make the runtime grow the local-memory reservation during the call
    if (k > kMaxFastElectrons)
        return set_error(nullptr, VB_ERR_UNSUPPORTED,
                         "vb_spin_pairs_noalloc: at most 8 electrons per string (use the plan API for more)");
    const long long N = n_strings;
    const long long n_pairs = N * (N + 1) / 2;
    const int np = n * (n + 1) / 2, gd = n * (n - 1) / 2;
    // layout of the static scratch, sized for the largest factor rank (np columns)
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off = align256(off + bytes);
        return at;
    };
    const size_t o_rows = take(sizeof(uint64_t) * 2 * N);
    const size_t o_rlist = take(sizeof(int) * n_pairs);
    const size_t o_rdesc = take(sizeof(unsigned) * n_pairs);
    const size_t o_ebound = take(sizeof(int) * N * (k + 2));
    const size_t o_gamma = take(sizeof(double) * (size_t)(gd > 0 ? gd : 1) * (gd > 0 ? gd : 1));
    const size_t o_kfull = take(sizeof(double) * (size_t)np * np);
    const size_t o_lf = take(sizeof(double) * (size_t)np * np);
    const size_t o_fwork = take(sizeof(double) * (size_t)np * np);
    const size_t o_fcols = take(sizeof(double) * (size_t)np * np);
    const size_t o_signs = take(sizeof(int) * np);
    const size_t o_meta = take(sizeof(int) * 4);
    const size_t o_counters = take(sizeof(unsigned long long) * 8);
    const size_t o_tables = take(sizeof(double) * frame_table_doubles(n, k, np) * N);
    const size_t o_records = take(sizeof(double) * (size_t)record_stride_for(np) * n_pairs);
    const size_t o_list = take(sizeof(unsigned long long) * n_pairs);
    if (off > kNoAllocScratchBytes)
        return set_error(nullptr, VB_ERR_BUDGET,
                         "vb_spin_pairs_noalloc: this string table needs " + std::to_string(off) +
                             " bytes of scratch; the static scratch holds " + std::to_string(kNoAllocScratchBytes) +
                             " bytes (use vb_hs_plan_create / vb_hs_plan_execute for larger tables)");

    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices)
        return set_error(nullptr, VB_ERR_UNSUPPORTED, "vb_spin_pairs_noalloc: device index out of range");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_address[device]) {
            // set-up, once per device: the exact-path kernels' stack (so that no later call makes
            // the runtime grow the device's local-memory reservation), then the array's address
            err = reserve_kernel_stack();
            if (err != cudaSuccess) return cuda_error(nullptr, err, "cudaDeviceSetLimit (kernel stack)");
            err = preload_kernels();
            if (err != cudaSuccess) return cuda_error(nullptr, err, "cudaFuncGetAttributes (kernel preload)");
            void* ptr = nullptr;
            err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (err != cudaSuccess) return cuda_error(nullptr, err, "cudaGetSymbolAddress (static scratch)");
            g_scratch_address[device] = ptr;
        }
        base = g_scratch_address[device];
    }
    unsigned char* b = static_cast<unsigned char*>(base);
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    uint64_t* rows = reinterpret_cast<uint64_t*>(b + o_rows);
    int* rlist = reinterpret_cast<int*>(b + o_rlist);
    unsigned* rdesc = reinterpret_cast<unsigned*>(b + o_rdesc);
    int* ebound = reinterpret_cast<int*>(b + o_ebound);
    double* gamma = reinterpret_cast<double*>(b + o_gamma);
    double* kfull = reinterpret_cast<double*>(b + o_kfull);
    double* lf = reinterpret_cast<double*>(b + o_lf);
    int* meta_d = reinterpret_cast<int*>(b + o_meta);
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(b + o_counters);

    // validate and expand the string table
    err = cudaMemsetAsync(meta_d, 0, sizeof(int) * 4, s);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "cudaMemsetAsync");
    occupation_rows_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(strings, n_strings, k, n, rows, meta_d + 2);
    err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_error(nullptr, err, "occupation_rows_kernel");
    err = launch_prepare_tables(n, eri_packed, gamma, kfull, s);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "prepare_tables");
    err = launch_factor_pair_kernel(np, kfull, reinterpret_cast<double*>(b + o_fwork),
                                    reinterpret_cast<double*>(b + o_fcols), reinterpret_cast<int*>(b + o_signs), lf, np,
                                    meta_d, s);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "factor_pair_kernel");
    int meta[4] = {0, 0, 0, 0};
    err = cudaMemcpyAsync(meta, meta_d, sizeof(meta), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "vb_spin_pairs_noalloc read-back");
    if (meta[2] != 0)
        return set_error(nullptr, VB_ERR_INVALID,
                         "vb_spin_pairs_noalloc: a string mask has the wrong electron count or an orbital >= n");
    const int R = meta[0] + meta[1];

    err = cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * 8, s);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "cudaMemsetAsync");
    if (frame_spin_supported(n, k, 0)) {
        err = launch_sort_right_strings(k, n_strings, rows, rlist, rdesc, ebound, s);
        if (err != cudaSuccess) return cuda_error(nullptr, err, "sort_right_strings");
    }
    SpinTableArgs a{};
    a.n = n;
    a.k = k;
    a.n_strings = n_strings;
    a.occ = rows;
    a.n_pairs = n_pairs;
    a.S = ovlp_act;
    a.h = h1e_act;
    a.gamma = gamma;
    a.eri = eri_packed;
    a.gamma_dim = gd;
    a.lf = lf;
    a.ld = np;
    a.R = R;
    a.records = reinterpret_cast<double*>(b + o_records);
    a.rec_stride = record_stride_for(R);
    a.careful_count = counters;
    a.careful_list = reinterpret_cast<unsigned long long*>(b + o_list);
    a.items = nullptr;
    a.n_items = 0;
    a.all_careful = 0;
    a.r_pos = meta[0];
    a.rlist = rlist;
    a.rdesc = rdesc;
    a.ebound = ebound;
    a.task_counter = counters + 4;
    int launches = 0;
    err = launch_spin_tables(a, reinterpret_cast<double*>(b + o_tables), s, &launches);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "spin tables");
    err = launch_spin_pairs(a, reinterpret_cast<double*>(b + o_tables), s, &launches);
    if (err == cudaSuccess) err = launch_spin_pairs_exact(a, s, &launches);
    if (err != cudaSuccess) return cuda_error(nullptr, err, "spin_pairs");
    long long blocks = (n_pairs + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    extract_scalars_kernel<<<(unsigned)blocks, 256, 0, s>>>(a.records, a.rec_stride, R, n_pairs, out_scalars);
    err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_error(nullptr, err, "extract_scalars_kernel");
    return VB_OK;
}
