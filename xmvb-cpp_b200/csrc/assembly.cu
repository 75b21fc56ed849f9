// Structure H/S assembly as HBM streams (sm_100a).
//
// The reference accumulates H_IJ = sum_{d in I, e in J} c_dI c_eJ H_de for left <= right
// structure pairs and mirrors the upper triangle (hamiltonian_overlap.cpp:437-450, 890-1022).
// Here the determinant matrix is symmetric and only its upper triangle is produced, in bands
// of columns, already weighted by the determinant-pair kernel (U' = upper triangle with halved
// diagonal, folded over the spin-flip symmetry when present), so that H_d = U' + U'^T and
//   Z  = T^T U'          (n_str x n_det; one streaming pass over every band, band_reduce)
//   W  = Z T             (n_str x n_str; structure_reduce)
//   H  = W + W^T         (symmetrize)
// Every sum runs in a fixed order (no atomics), so results are bitwise reproducible.
#include <cuda_runtime.h>

#include "internal.h"
#include "kernels.h"

namespace vbcore {
namespace {

constexpr int kPad = kBandReduceColumns + 1;

// One CTA per (32 band columns, structure chunk of at most 64 structures): every chunk's
// triples stream the band rows they need, and the small per-chunk accumulators let several
// CTAs share an SM.  Warp w owns the chunk's structures bucketed to it (local structure index
// = w mod warps), so each shared-memory accumulator has exactly one writer and the sum order is
// fixed.  A warp walks its (determinant, structure, coefficient) triples, sorted by
// determinant, 32 at a time: lane j fetches triple j, then the warp broadcasts them one by one;
// the band loads of consecutive triples are independent, which keeps many loads in flight.
__global__ void __launch_bounds__(kBandReduceWarps * 32) band_reduce_kernel(BandReduceArgs a) {
    extern __shared__ double zsm[];
    const int chunk = blockIdx.y;
    const int struct_begin = __ldg(a.chunk_begin + chunk), struct_count = __ldg(a.chunk_count + chunk);
    const long long* wbegin = a.wbegin + (size_t)chunk * (kBandReduceWarps + 1);
    double* zh = zsm;
    double* zs = zsm + (size_t)struct_count * kPad;
    for (int i = threadIdx.x; i < struct_count * kPad; i += blockDim.x) {
        zh[i] = 0.0;
        zs[i] = 0.0;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long j = (long long)blockIdx.x * kBandReduceColumns + lane;
    const bool valid = j < a.width;
    const long long e = a.e0 + j;
    long long row_end = a.e0 + (long long)blockIdx.x * kBandReduceColumns + kBandReduceColumns;
    if (row_end > a.e0 + a.width) row_end = a.e0 + a.width;
    const long long t_begin = wbegin[warp], t_end = wbegin[warp + 1];
    for (long long base = t_begin; base < t_end; base += 32) {
        const long long mine = base + lane;
        int d_l = 0x7fffffff, I_l = 0;
        double c_l = 0.0;
        if (mine < t_end) {
            d_l = __ldg(a.wdet + mine);
            I_l = __ldg(a.wstruct + mine);
            c_l = __ldg(a.wcoef + mine);
        }
        const int first = __shfl_sync(0xffffffffu, d_l, 0);
        if (first >= row_end) break;
        // eight independent band loads in flight per batch
#pragma unroll
        for (int q0 = 0; q0 < 32; q0 += 8) {
            int d[8], I[8];
            double c[8], hv[8], sv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                d[i] = __shfl_sync(0xffffffffu, d_l, q0 + i);
                I[i] = __shfl_sync(0xffffffffu, I_l, q0 + i);
                c[i] = __shfl_sync(0xffffffffu, c_l, q0 + i);
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const bool use = valid && d[i] <= e && d[i] < row_end;
                const long long o = use ? (long long)d[i] * a.width + j : 0;
                hv[i] = use ? __ldg(a.Hb + o) : 0.0;
                sv[i] = use ? __ldg(a.Sb + o) : 0.0;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (d[i] >= row_end) continue;  // padding triples and rows past this column block
                zh[I[i] * kPad + lane] = fma(c[i], hv[i], zh[I[i] * kPad + lane]);
                zs[I[i] * kPad + lane] = fma(c[i], sv[i], zs[I[i] * kPad + lane]);
            }
        }
    }
    __syncthreads();
    const long long col0 = a.e0 + (long long)blockIdx.x * kBandReduceColumns;
    for (int i = threadIdx.x; i < struct_count * kBandReduceColumns; i += blockDim.x) {
        const int I = i % struct_count, l = i / struct_count;
        if ((long long)blockIdx.x * kBandReduceColumns + l >= a.width) continue;
        const long long col = col0 + l;
        a.Zh[col * a.n_str + struct_begin + I] = zh[I * kPad + l];
        a.Zs[col * a.n_str + struct_begin + I] = zs[I * kPad + l];
    }
}

// W[I, J] = sum_{(e, c) in J} c Z[I, e]; one CTA per J, threads over I.
__global__ void structure_reduce_kernel(StructureReduceArgs a) {
    const int J = blockIdx.x;
    const long long t0 = a.str_off[J], t1 = a.str_off[J + 1];
    for (int I = threadIdx.x; I < a.n_str; I += blockDim.x) {
        double wh = 0.0, ws = 0.0;
        for (long long t = t0; t < t1; ++t) {
            const long long e = __ldg(a.str_det + t);
            const double c = __ldg(a.str_coef + t);
            wh = fma(c, __ldg(a.Zh + e * a.n_str + I), wh);
            ws = fma(c, __ldg(a.Zs + e * a.n_str + I), ws);
        }
        a.Wh[(long long)J * a.n_str + I] = wh;
        a.Ws[(long long)J * a.n_str + I] = ws;
    }
}

__global__ void symmetrize_kernel(int n, const double* __restrict__ Wh, const double* __restrict__ Ws,
                                  double* __restrict__ H, double* __restrict__ S) {
    const long long total = (long long)n * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long J = t / n, I = t % n;
        H[t] = Wh[t] + Wh[I * n + J];
        S[t] = Ws[t] + Ws[I * n + J];
    }
}

}  // namespace

size_t band_reduce_smem_bytes(int struct_count) { return sizeof(double) * 2 * (size_t)struct_count * kPad; }

// 64 structures per chunk: 33.8 KB of accumulators, six CTAs per SM.
int band_reduce_max_structures() { return 64; }

cudaError_t launch_band_reduce(const BandReduceArgs& a, cudaStream_t stream, int* launches) {
    const size_t smem = band_reduce_smem_bytes(a.max_count);
    cudaError_t err = allow_dynamic_smem((const void*)band_reduce_kernel, (int)smem);
    if (err != cudaSuccess) return err;
    const long long blocks = (a.width + kBandReduceColumns - 1) / kBandReduceColumns;
    band_reduce_kernel<<<dim3((unsigned)blocks, (unsigned)a.n_chunks), kBandReduceWarps * 32, smem, stream>>>(a);
    ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_structure_reduce(const StructureReduceArgs& a, double* H, double* S, cudaStream_t stream,
                                    int* launches) {
    structure_reduce_kernel<<<a.n_str, 128, 0, stream>>>(a);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    const long long total = (long long)a.n_str * a.n_str;
    long long blocks = (total + 255) / 256;
    if (blocks > 2048) blocks = 2048;
    symmetrize_kernel<<<(unsigned)blocks, 256, 0, stream>>>(a.n_str, a.Wh, a.Ws, H, S);
    *launches += 2;
    return cudaGetLastError();
}

}  // namespace vbcore
