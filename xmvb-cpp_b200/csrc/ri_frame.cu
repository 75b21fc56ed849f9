// RI pair factors in a new orbital frame (sm_100a): the counterpart of transform_ri_pair_factors
// and its two directional forms (src/integrals/active/ri_transform.cpp:98-211).  Each auxiliary
// row P of the factor matrix packs a symmetric n x n factor B_P at (i, j), i >= j, i (i+1)/2 + j;
// the factors are stored column-major as [n_aux x n(n+1)/2] (row = auxiliary function).
//   forward:             Bbar_P = Q^T B_P Q
//   raw direction:       Q^T dB_P Q + dQ^T B_P Q + Q^T B_P dQ
//   orthogonal direction (from Bbar = Q^T B Q already in the frame, dQ = -Q K):
//                        Q^T dB_P Q - K^T Bbar_P - Bbar_P K
// One CTA per auxiliary row: Q (and the direction) and the expanded factor(s) are staged in shared
// memory; threads own output entries (i >= j) and form the two products through one shared
// n x n intermediate (B Q, then Q^T (B Q)).
#include <cuda_runtime.h>

#include <string>

#include "internal.h"

namespace vbcore {
namespace {

constexpr int kFrameMaxN = 64;

__device__ __forceinline__ int packed(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// dynamic shared memory: Q, D (direction, modes 1-2), X (expanded factor), Y (second factor),
// T (n x n intermediate): 5 n^2 doubles.
__global__ void __launch_bounds__(256) ri_frame_kernel(int mode, int n_aux, int n, const double* __restrict__ F,
                                                       const double* __restrict__ G, const double* __restrict__ Q,
                                                       const double* __restrict__ D, double* __restrict__ out) {
    extern __shared__ double sm[];
    const int n2 = n * n, np = n * (n + 1) / 2;
    double* sQ = sm;
    double* sD = sQ + n2;
    double* sX = sD + n2;
    double* sY = sX + n2;
    double* sT = sY + n2;
    for (int e = threadIdx.x; e < n2; e += blockDim.x) {
        sQ[e] = Q[e];
        sD[e] = mode ? D[e] : 0.0;
    }
    for (int P = blockIdx.x; P < n_aux; P += gridDim.x) {
        __syncthreads();
        // X = the factor the frame acts on, Y = the second factor of the directional forms
        for (int e = threadIdx.x; e < n2; e += blockDim.x) {
            const int i = e % n, j = e / n;
            const long long col = (long long)packed(i, j) * n_aux + P;
            sX[e] = mode == 0 ? F[col] : G[col];  // forward: B; raw: dB; orthogonal: dBraw
            sY[e] = mode ? F[col] : 0.0;          // raw: B; orthogonal: Bbar
        }
        __syncthreads();
        // T = X Q (column-major: T[i + j n] = sum_k X[i + k n] Q[k + j n])
        for (int e = threadIdx.x; e < n2; e += blockDim.x) {
            const int i = e % n, j = e / n;
            double acc = 0.0;
            for (int k = 0; k < n; ++k) acc = fma(sX[i + k * n], sQ[k + j * n], acc);
            sT[e] = acc;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < np; t += blockDim.x) {
            int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
            while (i * (i + 1) / 2 > t) --i;
            while ((i + 1) * (i + 2) / 2 <= t) ++i;
            const int j = t - i * (i + 1) / 2;
            // (Q^T T)[i, j]
            double v = 0.0;
            for (int k = 0; k < n; ++k) v = fma(sQ[k + i * n], sT[k + j * n], v);
            if (mode == 1) {
                // + dQ^T (B Q) + (B Q)^T dQ: (dQ^T B Q)[i, j] + (dQ^T B Q)[j, i]
                double a = 0.0, b = 0.0;
                for (int k = 0; k < n; ++k) {
                    double bq_kj = 0.0, bq_ki = 0.0;
                    for (int l = 0; l < n; ++l) {
                        bq_kj = fma(sY[k + l * n], sQ[l + j * n], bq_kj);
                        bq_ki = fma(sY[k + l * n], sQ[l + i * n], bq_ki);
                    }
                    a = fma(sD[k + i * n], bq_kj, a);
                    b = fma(sD[k + j * n], bq_ki, b);
                }
                v += a + b;
            } else if (mode == 2) {
                // - K^T Bbar - Bbar K: -(sum_k K[k, i] Bbar[k, j] + Bbar[i, k] K[k, j])
                double a = 0.0;
                for (int k = 0; k < n; ++k) a = fma(sD[k + i * n], sY[k + j * n], fma(sY[i + k * n], sD[k + j * n], a));
                v -= a;
            }
            out[(long long)t * n_aux + P] = v;
        }
    }
}

}  // namespace
}  // namespace vbcore

using namespace vbcore;

extern "C" vb_status vb_ri_pair_factors_frame(vb_context* ctx, int mode, const double* factors,
                                              const double* factor_direction, int n_aux, int n,
                                              const double* frame, const double* frame_direction, int mem_space,
                                              double* out) {
    if (!ctx) return VB_ERR_INVALID;
    const char* who = "vb_ri_pair_factors_frame";
    if (mode < 0 || mode > 2 || n_aux < 1 || n < 1 || !factors || !frame || !out ||
        (mode > 0 && (!factor_direction || !frame_direction)))
        return set_error(ctx, VB_ERR_INVALID, std::string(who) + ": bad arguments");
    if (n > kFrameMaxN) return set_error(ctx, VB_ERR_UNSUPPORTED, std::string(who) + ": at most 64 orbitals");
    if (mem_space != VB_MEM_HOST && mem_space != VB_MEM_DEVICE)
        return set_error(ctx, VB_ERR_INVALID, "bad memory space");
    DeviceGuard guard(ctx->device);
    cudaStream_t s = ctx->stream;
    const bool host = mem_space == VB_MEM_HOST;
    const size_t n2 = (size_t)n * n, np = (size_t)n * (n + 1) / 2;
    const size_t bF = sizeof(double) * np * n_aux, bQ = sizeof(double) * n2;
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, host ? 3 * bF + 2 * bQ + 64 : 16);
    if (st != VB_OK) return st;
    double* dF = const_cast<double*>(factors);
    double* dG = const_cast<double*>(factor_direction);
    double* dQ = const_cast<double*>(frame);
    double* dD = const_cast<double*>(frame_direction);
    double* dO = out;
    cudaError_t err = cudaSuccess;
    if (host) {
        unsigned char* b = static_cast<unsigned char*>(ws.ptr);
        dF = reinterpret_cast<double*>(b);
        dG = reinterpret_cast<double*>(b + bF);
        dO = reinterpret_cast<double*>(b + 2 * bF);
        dQ = reinterpret_cast<double*>(b + 3 * bF);
        dD = reinterpret_cast<double*>(b + 3 * bF + bQ);
        err = cudaMemcpyAsync(dF, factors, bF, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(dQ, frame, bQ, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess && mode > 0) err = cudaMemcpyAsync(dG, factor_direction, bF, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess && mode > 0) err = cudaMemcpyAsync(dD, frame_direction, bQ, cudaMemcpyHostToDevice, s);
    }
    const size_t smem = 5 * bQ;
    if (err == cudaSuccess) err = allow_dynamic_smem((const void*)ri_frame_kernel, smem);
    if (err == cudaSuccess) {
        const int grid = n_aux < 148 * 4 ? n_aux : 148 * 4;
        ri_frame_kernel<<<grid, 256, smem, s>>>(mode, n_aux, n, dF, mode ? dG : nullptr, dQ, mode ? dD : nullptr, dO);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess && host) err = cudaMemcpyAsync(out, dO, bF, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess && host) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, who);
    return VB_OK;
}
