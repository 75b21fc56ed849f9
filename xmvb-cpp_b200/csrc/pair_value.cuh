// Determinant-pair value from two spin-pair records (shared by the pair and assembly kernels).
#pragma once

#include <cuda_runtime.h>

#include "kernels.h"

namespace vbcore {

// Index of the unordered pair (u <= v) of an N-string table in row-major upper packing.
__device__ __forceinline__ long long record_index(long long u, long long v, long long N) {
    return u * N - u * (u - 1) / 2 + (v - u);
}

// S_de = S_a S_b, H_de = H_a S_b + H_b S_a + sum_m sigma_m u_a[m] u_b[m] for one determinant pair
// (evaluator.cpp:354-384 of the reference, with the opposite-spin term in factored form).
__device__ __forceinline__ void pair_value(const FullPairArgs& a, long long d, long long e, double* H, double* S) {
    double sa = 1.0, hsa = 0.0, sb = 1.0, hsb = 0.0, dot = 0.0;
    const double* ra = nullptr;
    const double* rb = nullptr;
    const int R = a.R;
    if (a.ka > 0) {
        const int ia = __ldg(a.det_alpha + d), ja = __ldg(a.det_alpha + e);
        const long long lo = min(ia, ja), hi = max(ia, ja);
        ra = a.rec_a + record_index(lo, hi, a.Na) * a.stride_a;
        sa = ra[R];
        hsa = ra[R + 1];
    }
    if (a.kb > 0) {
        const int ib = __ldg(a.det_beta + d), jb = __ldg(a.det_beta + e);
        const long long lo = min(ib, jb), hi = max(ib, jb);
        rb = a.rec_b + record_index(lo, hi, a.Nb) * a.stride_b;
        sb = rb[R];
        hsb = rb[R + 1];
    }
    if (ra && rb) {
        double pos = 0.0, neg = 0.0;
        int m = 0;
        for (; m + 1 < a.r_pos; m += 2) {
            const double2 x = *reinterpret_cast<const double2*>(ra + m);
            const double2 y = *reinterpret_cast<const double2*>(rb + m);
            pos = fma(x.x, y.x, pos);
            pos = fma(x.y, y.y, pos);
        }
        for (; m < a.r_pos; ++m) pos = fma(ra[m], rb[m], pos);
        for (; m < R; ++m) neg = fma(ra[m], rb[m], neg);
        dot = pos - neg;
    }
    *H = fma(hsa, sb, fma(hsb, sa, dot));
    *S = sa * sb;
}

}  // namespace vbcore
