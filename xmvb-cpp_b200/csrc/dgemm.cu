// FP64 contractions over the pair-kernel factor columns on the tensor cores (mma.sync m8n8k4 f64),
// for the gradient's spin-pair chunks (the two products that used to be library GEMMs):
//
//   factor_project:  C[q + c ldC] = sum_m Lf[q ld + m] Y[m + c ldY]        (np x cnt, K = R)
//       per spin pair c, the u-adjoint (R values) pulled back onto every packed pair q;
//   factor_outer:    G[m + q ldG] += sum_c Y[m + c ldY] Z[q + c ldZ]      (R x np, K = cnt)
//       the factor-column adjoint accumulated over all spin pairs of a chunk.
//
// factor_project: a CTA owns 64 spin pairs (columns c) and every packed pair q; Lf (np x R) and the
// 64 columns of Y are staged in shared memory, each warp keeps its 16 columns' B fragments for all
// k-steps in registers and sweeps the q tiles.  factor_outer: split over c, a CTA accumulates the
// whole R x np product of its c range (Y and Z staged 32 columns at a time, each warp a 2 x 2 block
// of 8 x 8 tiles per step) into its own partial; a second kernel adds the partials to G in a fixed
// order, so the result does not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "kernels.h"

namespace vbcore {
namespace {

constexpr int kProjCols = 64;     // spin pairs per CTA in factor_project
constexpr int kOuterChunk = 32;   // spin pairs staged per step in factor_outer
constexpr int kOuterWarps = 8;

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__host__ __device__ inline int up8(int x) { return (x + 7) / 8 * 8; }
__host__ __device__ inline int up4(int x) { return (x + 3) / 4 * 4; }

// C (np x cnt, column-major, ldC) = Lf^T-view (np x R: Lf[q * ld + m]) * Y (R x cnt, ldY); KS >= the
// number of 4-deep k-steps (the B fragments of all of them stay in registers).
template <int KS>
__global__ void __launch_bounds__(128) factor_project_kernel(int np, int R, const double* __restrict__ lf, int ld,
                                                             const double* __restrict__ Y, long long ldY, long long cnt,
                                                             double* __restrict__ C, long long ldC) {
    extern __shared__ double sm[];
    const int MQ = up8(np), KR = up4(R);
    const int LS = KR + 1;  // Lf row stride in shared memory (odd: conflict-free fragment reads)
    double* sL = sm;                               // [MQ][LS]
    double* sY = sL + (size_t)MQ * LS;             // [KR][kProjCols + 1]
    constexpr int YS = kProjCols + 1;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tq = lane & 3;
    for (int e = tid; e < MQ * KR; e += 128) {
        const int q = e / KR, m = e % KR;
        sL[q * LS + m] = (q < np && m < R) ? __ldg(lf + (long long)q * ld + m) : 0.0;
    }
    const long long ntiles = (cnt + kProjCols - 1) / kProjCols;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long c0 = t * kProjCols;
        __syncthreads();
        // m fastest: contiguous reads of each column; eight loads in flight per thread
        for (int e0 = tid; e0 < KR * kProjCols; e0 += 8 * 128) {
            double v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int e = e0 + 128 * j, cc = e / KR, m = e % KR;
                const long long c = c0 + cc;
                v[j] = (e < KR * kProjCols && m < R && c < cnt) ? __ldg(Y + c * ldY + m) : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int e = e0 + 128 * j;
                if (e < KR * kProjCols) sY[(e % KR) * YS + e / KR] = v[j];
            }
        }
        __syncthreads();
        // this warp's 16 columns: B fragments for every k-step, kept in registers
        constexpr int KMAXS = KS;
        double b0[KMAXS], b1[KMAXS];
        const int ks_n = KR / 4;
#pragma unroll
        for (int ks = 0; ks < KMAXS; ++ks) {
            if (ks < ks_n) {
                b0[ks] = sY[(4 * ks + tq) * YS + 16 * warp + g];
                b1[ks] = sY[(4 * ks + tq) * YS + 16 * warp + 8 + g];
            }
        }
        for (int mt = 0; mt < MQ / 8; ++mt) {
            double acc0[2] = {0.0, 0.0}, acc1[2] = {0.0, 0.0};
#pragma unroll
            for (int ks = 0; ks < KMAXS; ++ks) {
                if (ks < ks_n) {
                    const double a = sL[(8 * mt + g) * LS + 4 * ks + tq];
                    dmma(acc0, a, b0[ks]);
                    dmma(acc1, a, b1[ks]);
                }
            }
            const int q = 8 * mt + g;
            if (q < np) {
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const long long ca = c0 + 16 * warp + 2 * tq + i, cb = ca + 8;
                    if (ca < cnt) C[ca * ldC + q] = acc0[i];
                    if (cb < cnt) C[cb * ldC + q] = acc1[i];
                }
            }
        }
    }
}

// partial[blockIdx.x] (R x np, column-major, ld R) = sum over this CTA's c range of Y[:, c] Z[:, c]^T;
// BPW >= the 2 x 2 tile blocks each warp owns.
template <int BPW>
__global__ void __launch_bounds__(32 * kOuterWarps) factor_outer_kernel(int np, int R, const double* __restrict__ Y,
                                                                        long long ldY, const double* __restrict__ Z,
                                                                        long long ldZ, long long cnt,
                                                                        double* __restrict__ partial) {
    extern __shared__ double sm[];
    const int MR = up8(R), NQ = up8(np);
    constexpr int CS = kOuterChunk + 1;
    double* sY = sm;                       // [MR][CS]: Y rows m, staged columns c
    double* sZ = sY + (size_t)MR * CS;     // [NQ][CS]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tq = lane & 3;
    const int mt_n = MR / 8, nt_n = NQ / 8;
    const int bm_n = (mt_n + 1) / 2, bn_n = (nt_n + 1) / 2;  // 2 x 2 tile blocks
    const int nblocks = bm_n * bn_n;
    double acc[BPW][2][2][2];
#pragma unroll
    for (int i = 0; i < BPW; ++i)
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int y = 0; y < 2; ++y) acc[i][x][y][0] = acc[i][x][y][1] = 0.0;
    const long long per = (cnt + gridDim.x - 1) / gridDim.x;
    const long long c_begin = blockIdx.x * per, c_end = min(cnt, c_begin + per);
    for (long long c0 = c_begin; c0 < c_end; c0 += kOuterChunk) {
        __syncthreads();
        // row fastest: contiguous column reads; eight loads in flight per thread
        const int tot = (MR + NQ) * kOuterChunk;
        for (int e0 = tid; e0 < tot; e0 += 8 * 32 * kOuterWarps) {
            double v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int e = e0 + 32 * kOuterWarps * j;
                const int cc = e / (MR + NQ), r = e % (MR + NQ);
                const long long c = c0 + cc;
                v[j] = 0.0;
                if (e < tot && c < c_end) {
                    if (r < MR) {
                        if (r < R) v[j] = __ldg(Y + c * ldY + r);
                    } else if (r - MR < np) {
                        v[j] = __ldg(Z + c * ldZ + (r - MR));
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int e = e0 + 32 * kOuterWarps * j;
                if (e >= tot) break;
                const int cc = e / (MR + NQ), r = e % (MR + NQ);
                if (r < MR)
                    sY[r * CS + cc] = v[j];
                else
                    sZ[(r - MR) * CS + cc] = v[j];
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < BPW; ++i) {
            const int blk = warp + kOuterWarps * i;
            if (blk >= nblocks) continue;
            const int bm = blk / bn_n, bn = blk % bn_n;
#pragma unroll
            for (int ks = 0; ks < kOuterChunk / 4; ++ks) {
                double a[2], b[2];
#pragma unroll
                for (int x = 0; x < 2; ++x) {
                    const int mt = 2 * bm + x, nt = 2 * bn + x;
                    a[x] = mt < mt_n ? sY[(8 * mt + g) * CS + 4 * ks + tq] : 0.0;
                    b[x] = nt < nt_n ? sZ[(8 * nt + g) * CS + 4 * ks + tq] : 0.0;
                }
#pragma unroll
                for (int x = 0; x < 2; ++x)
#pragma unroll
                    for (int y = 0; y < 2; ++y) dmma(acc[i][x][y], a[x], b[y]);
            }
        }
    }
    double* out = partial + (size_t)blockIdx.x * R * np;
#pragma unroll
    for (int i = 0; i < BPW; ++i) {
        const int blk = warp + kOuterWarps * i;
        if (blk >= nblocks) continue;
        const int bm = blk / bn_n, bn = blk % bn_n;
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int y = 0; y < 2; ++y)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int m = 8 * (2 * bm + x) + g, q = 8 * (2 * bn + y) + 2 * tq + j;
                    if (m < R && q < np) out[(size_t)q * R + m] = acc[i][x][y][j];
                }
    }
}

// Shapes beyond the tensor-core kernels' envelope (R > 144 or np > 192): one thread per output
// element (and per c range for the outer product).
__global__ void factor_project_simt(int np, int R, const double* __restrict__ lf, int ld, const double* __restrict__ Y,
                                    long long ldY, long long cnt, double* __restrict__ C, long long ldC) {
    const long long total = (long long)np * cnt;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(e % np);
        const long long c = e / np;
        double acc = 0.0;
        for (int m = 0; m < R; ++m) acc = fma(__ldg(lf + (long long)q * ld + m), __ldg(Y + c * ldY + m), acc);
        C[c * ldC + q] = acc;
    }
}

__global__ void factor_outer_simt(int np, int R, const double* __restrict__ Y, long long ldY,
                                  const double* __restrict__ Z, long long ldZ, long long cnt, int parts,
                                  double* __restrict__ partial) {
    const long long total = (long long)R * np * parts;
    const long long per = (cnt + parts - 1) / parts;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(e % R);
        const long long rest = e / R;
        const int q = (int)(rest % np), b = (int)(rest / np);
        const long long c0 = b * per, c1 = min(cnt, c0 + per);
        double acc = 0.0;
        for (long long c = c0; c < c1; ++c) acc = fma(__ldg(Y + c * ldY + m), __ldg(Z + c * ldZ + q), acc);
        partial[(size_t)b * R * np + (size_t)q * R + m] = acc;
    }
}

// G[m + q ldG] += sum_b partial[b][m + q R], b in order.
__global__ void factor_outer_reduce_kernel(int np, int R, int nparts, const double* __restrict__ partial,
                                           double* __restrict__ G, long long ldG) {
    const int total = R * np;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nparts; ++b) s += partial[(size_t)b * total + e];
        const int m = e % R, q = e / R;
        G[(long long)q * ldG + m] += s;
    }
}

}  // namespace

size_t factor_project_smem(int np, int R) {
    return sizeof(double) * ((size_t)up8(np) * (up4(R) + 1) + (size_t)up4(R) * (kProjCols + 1));
}

bool factor_contractions_supported(int np, int R) {
    // register-resident k-steps (R <= 144) and tile blocks (12 per warp: R, np <= 192)
    return R <= 144 && np <= 192 && factor_project_smem(np, R) <= 200 * 1024 &&
           sizeof(double) * (size_t)(up8(R) + up8(np)) * (kOuterChunk + 1) <= 200 * 1024;
}

cudaError_t launch_factor_project(int np, int R, const double* lf, int ld, const double* Y, long long ldY,
                                  long long cnt, double* C, long long ldC, cudaStream_t stream) {
    if (cnt <= 0) return cudaSuccess;
    if (R <= 0) return cudaMemsetAsync(C, 0, sizeof(double) * (size_t)ldC * cnt, stream);
    if (!factor_contractions_supported(np, R)) {
        const long long blocks = std::min<long long>(148LL * 16, ((long long)np * cnt + 255) / 256);
        factor_project_simt<<<(unsigned)blocks, 256, 0, stream>>>(np, R, lf, ld, Y, ldY, cnt, C, ldC);
        return cudaGetLastError();
    }
    const size_t smem = factor_project_smem(np, R);
    const int ks = up4(R) / 4;
    const void* fn = ks <= 12 ? (const void*)factor_project_kernel<12>
                              : (ks <= 24 ? (const void*)factor_project_kernel<24> : (const void*)factor_project_kernel<36>);
    cudaError_t err = allow_dynamic_smem(fn, smem);
    if (err != cudaSuccess) return err;
    const long long tiles = (cnt + kProjCols - 1) / kProjCols;
    const int grid = (int)std::min<long long>(tiles, 148LL * 4);
    if (ks <= 12)
        factor_project_kernel<12><<<grid, 128, smem, stream>>>(np, R, lf, ld, Y, ldY, cnt, C, ldC);
    else if (ks <= 24)
        factor_project_kernel<24><<<grid, 128, smem, stream>>>(np, R, lf, ld, Y, ldY, cnt, C, ldC);
    else
        factor_project_kernel<36><<<grid, 128, smem, stream>>>(np, R, lf, ld, Y, ldY, cnt, C, ldC);
    return cudaGetLastError();
}

// Split-K parts of factor_outer: up to kOuterMaxParts CTAs (four per SM, so that enough column
// loads are in flight), at least 64 spin pairs (two staged chunks) each.
int factor_outer_parts(long long cnt) {
    return (int)std::max<long long>(1, std::min<long long>(kOuterMaxParts, (cnt + 63) / 64));
}

cudaError_t launch_factor_outer(int np, int R, const double* Y, long long ldY, const double* Z, long long ldZ,
                                long long cnt, double* G, long long ldG, double* partial, cudaStream_t stream) {
    if (cnt <= 0 || R <= 0) return cudaSuccess;
    const int parts = factor_outer_parts(cnt);
    if (!factor_contractions_supported(np, R)) {
        const long long total = (long long)R * np * parts;
        factor_outer_simt<<<(unsigned)std::min<long long>(148LL * 16, (total + 255) / 256), 256, 0, stream>>>(
            np, R, Y, ldY, Z, ldZ, cnt, parts, partial);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
        factor_outer_reduce_kernel<<<std::max(1, std::min(148, (R * np + 255) / 256)), 256, 0, stream>>>(
            np, R, parts, partial, G, ldG);
        return cudaGetLastError();
    }
    const size_t smem = sizeof(double) * (size_t)(up8(R) + up8(np)) * (kOuterChunk + 1);
    const int nblocks = ((up8(R) / 8 + 1) / 2) * ((up8(np) / 8 + 1) / 2);
    const int bpw = (nblocks + kOuterWarps - 1) / kOuterWarps;
    const void* fn = bpw <= 3 ? (const void*)factor_outer_kernel<3>
                              : (bpw <= 6 ? (const void*)factor_outer_kernel<6> : (const void*)factor_outer_kernel<12>);
    cudaError_t err = allow_dynamic_smem(fn, smem);
    if (err != cudaSuccess) return err;
    if (bpw <= 3)
        factor_outer_kernel<3><<<parts, 32 * kOuterWarps, smem, stream>>>(np, R, Y, ldY, Z, ldZ, cnt, partial);
    else if (bpw <= 6)
        factor_outer_kernel<6><<<parts, 32 * kOuterWarps, smem, stream>>>(np, R, Y, ldY, Z, ldZ, cnt, partial);
    else
        factor_outer_kernel<12><<<parts, 32 * kOuterWarps, smem, stream>>>(np, R, Y, ldY, Z, ldZ, cnt, partial);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    factor_outer_reduce_kernel<<<std::max(1, std::min(148, (R * np + 255) / 256)), 256, 0, stream>>>(np, R, parts,
                                                                                                     partial, G, ldG);
    return cudaGetLastError();
}

}  // namespace vbcore
