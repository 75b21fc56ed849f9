// Determinant-pair kernels for sm_100a.
//
//  * prepare_tables: the unpacked pair kernel K[p][q] = (p|q) over packed orbital pairs and the
//    antisymmetrized same-spin table Gamma[(i<k)][(j<l)] = (ij|kl) - (il|kj) used by the
//    same-spin two-electron sum (hamiltonian.cpp:83-123 sums exactly these differences).
//  * spin_pairs_fast<K>: one thread per unordered spin-string pair, K x K overlap block in
//    registers, Gauss-Jordan inversion with partial pivoting (row interchanges tracked as a
//    label permutation, no dynamic register indexing), determinant, first cofactors
//    A = det X^{-T}, one-electron and same-spin two-electron energies from shared-memory
//    tables.  A block is accepted only when ||X||_F ||X^{-1}||_F < 1e8 (kCertificate2): then the
//    last pivot of a complete-pivoting LU is at least 1 / ||X^{-1}||_F and the first at most
//    ||X||_F, so their ratio stays far above 1e-12 and the reference's FullPivLU would also find
//    full rank (overlap.cpp:60-71).  Every other block is appended to a list for the exact kernel.
//  * spin_pairs_exact<KM>: complete-pivoting LU / Jacobi SVD with the reference semantics
//    (device_algebra.cuh) for listed blocks, one thread per block, local arrays bounded by KM.
//  * full_pairs<KB>: one thread per determinant pair (d <= e) of a band of columns:
//    S = S_a S_b, H = H_a S_b + H_b S_a + sum A_a(r,c) A_b(r',c') (r c | r' c')
//    (evaluator.cpp:95-148, 354-384), the opposite-spin sum as k_a^2 k_b^2 gathers of the
//    shared-memory pair kernel against the beta cofactors held in registers.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <stdint.h>

#include <string>

#include "autotune.h"
#include "device_algebra.cuh"
#include "internal.h"
#include "kernels.h"
#include "pair_value.cuh"

namespace vbcore {
namespace {

constexpr double kThreshold = 1.0e-12;
constexpr double kFactorTolerance = 1.0e-15;  // relative pivot cut of the pair-kernel factorization
constexpr int kSms = 148;

__device__ __forceinline__ int occ_byte(const uint64_t* row, int i) {
    const uint64_t w = row[i >> 3];
    return (int)((w >> (8 * (i & 7))) & 0xFFu);
}

__global__ void prepare_tables_kernel(int n, const double* __restrict__ eri, double* __restrict__ gamma,
                                      double* __restrict__ kfull) {
    const int np = n * (n + 1) / 2;
    const int gd = n * (n - 1) / 2;
    const long long total_k = (long long)np * np;
    const long long total_g = (long long)gd * gd;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total_k + total_g; t += stride) {
        if (t < total_k) {
            const long long p = t / np, q = t % np;
            const long long hi = p > q ? p : q, lo = p > q ? q : p;
            kfull[t] = eri[hi * (hi + 1) / 2 + lo];
        } else {
            const long long g = t - total_k;
            const int row = (int)(g / gd), col = (int)(g % gd);
            // row = anti_index(i, kk) with i < kk; col = anti_index(j, l) with j < l
            int kk = (int)floor((1.0 + sqrt(1.0 + 8.0 * row)) * 0.5);
            while (kk * (kk - 1) / 2 > row) --kk;
            while ((kk + 1) * kk / 2 <= row) ++kk;
            const int i = row - kk * (kk - 1) / 2;
            int l = (int)floor((1.0 + sqrt(1.0 + 8.0 * col)) * 0.5);
            while (l * (l - 1) / 2 > col) --l;
            while ((l + 1) * l / 2 <= col) ++l;
            const int j = col - l * (l - 1) / 2;
            gamma[g] = dev::eri_packed(eri, i, j, kk, l) - dev::eri_packed(eri, i, l, kk, j);
        }
    }
}

// Pivoted LDL^T of the unpacked pair kernel with diagonal (complete) pivoting, one CTA.
// Stops when the largest remaining |diagonal| falls to rel_tol times the largest initial one;
// the dropped remainder then perturbs any opposite-spin energy by at most
// rel_tol * max|K_pp| * ||p_a||_1 ||p_b||_1.  Columns are emitted positive-sign first.
// The working matrix lives in shared memory when it fits (in_smem), else in `work`.
__global__ void __launch_bounds__(512) factor_pair_kernel(int np, const double* __restrict__ kfull,
                                                          double* __restrict__ work_g, double* __restrict__ cols,
                                                          int* __restrict__ signs, double* __restrict__ lf, int ld,
                                                          int* __restrict__ meta, double rel_tol, int in_smem) {
    extern __shared__ double fsm[];
    double* work = in_smem ? fsm : work_g;
    int* used = reinterpret_cast<int*>(in_smem ? fsm + (size_t)np * np : fsm);
    int* slot_col = used + np;  // emission map: output slot -> column
    __shared__ double red_v[32];
    __shared__ int red_i[32];
    __shared__ double s_piv;
    __shared__ int s_p;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nwarps = nt >> 5;
    const long long n2 = (long long)np * np;
    for (long long i = tid; i < n2; i += nt) work[i] = kfull[i];
    for (int i = tid; i < np; i += nt) used[i] = 0;
    __syncthreads();
    double local = 0.0;
    for (int i = tid; i < np; i += nt) local = fmax(local, fabs(work[(long long)i * np + i]));
    for (int o = 16; o > 0; o >>= 1) local = fmax(local, __shfl_xor_sync(0xffffffffu, local, o));
    if (lane == 0) red_v[warp] = local;
    __syncthreads();
    if (tid < 32) {
        double v = tid < nwarps ? red_v[tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (tid == 0) s_piv = v;
    }
    __syncthreads();
    const double cut = rel_tol * s_piv;
    int m = 0;
    for (; m < np; ++m) {
        double best = -1.0;
        int bi = -1;
        for (int i = tid; i < np; i += nt)
            if (!used[i]) {
                const double v = fabs(work[(long long)i * np + i]);
                if (v > best || (v == best && i < bi)) {
                    best = v;
                    bi = i;
                }
            }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi >= 0 && (bi < 0 || oi < bi))) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            red_v[warp] = best;
            red_i[warp] = bi;
        }
        __syncthreads();
        if (tid < 32) {
            double v = tid < nwarps ? red_v[tid] : -1.0;
            int vi = tid < nwarps ? red_i[tid] : -1;
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int oi = __shfl_xor_sync(0xffffffffu, vi, o);
                if (ov > v || (ov == v && oi >= 0 && (vi < 0 || oi < vi))) {
                    v = ov;
                    vi = oi;
                }
            }
            if (tid == 0) {
                s_p = vi;
                s_piv = vi >= 0 ? work[(long long)vi * np + vi] : 0.0;
            }
        }
        __syncthreads();
        const int p = s_p;
        const double piv = s_piv;
        if (p < 0 || !(fabs(piv) > cut) || fabs(piv) == 0.0) break;
        const double inv = 1.0 / sqrt(fabs(piv));
        const int sgn = piv > 0.0 ? 1 : -1;
        double* l = cols + (long long)m * np;
        for (int i = tid; i < np; i += nt) l[i] = used[i] ? 0.0 : work[(long long)i * np + p] * inv;
        if (tid == 0) signs[m] = sgn;
        __syncthreads();
        if (tid == 0) used[p] = 1;
        __syncthreads();
        // rank-1 update of the remaining block, one warp per row
        for (int i = warp; i < np; i += nwarps) {
            if (used[i]) continue;
            const double li = (double)sgn * l[i];
            double* row = work + (long long)i * np;
            for (int j = lane; j < np; j += 32)
                if (!used[j]) row[j] = fma(-li, l[j], row[j]);
        }
        __syncthreads();
    }
    if (tid == 0) {
        int pos = 0;
        for (int c = 0; c < m; ++c) pos += signs[c] > 0 ? 1 : 0;
        int ip = 0, in = pos;
        for (int c = 0; c < m; ++c) slot_col[signs[c] > 0 ? ip++ : in++] = c;
        meta[0] = pos;
        meta[1] = m - pos;
    }
    __syncthreads();
    for (int q = warp; q < np; q += nwarps)
        for (int slot = lane; slot < ld; slot += 32)
            lf[(long long)q * ld + slot] = slot < m ? cols[(long long)slot_col[slot] * np + q] : 0.0;
}

// Table geometry of the left-string decomposition (shared by host and device code).
//   nb_max(K)   complement orbitals held per left string (n - K <= nb_max)
//   kf(K)       GEMM depth: nb_max K entries of V, one trace slot, padded to 4
//   kfs(K)      shared-memory row stride >= kf with stride % 16 in {4, 12} (conflict-free
//               m8n8k4 fragment loads: the four rows of a half-warp land on disjoint banks)
//   nt_of(R)    8-row tiles covering the R + 1 table rows (factor columns and h)
__host__ __device__ constexpr int nb_max(int k) { return k <= 4 ? k + 4 : k; }
__host__ __device__ constexpr int kf(int k) { return (nb_max(k) * k + 1 + 3) / 4 * 4; }
__host__ __device__ constexpr int kfs(int k) {
    return (kf(k) % 16 == 4 || kf(k) % 16 == 12) ? kf(k) : kf(k) + 4;
}
__host__ __device__ constexpr int nt_of(int R) { return (R + 1 + 7) / 8; }
__host__ __device__ constexpr int table_stride_of(int k, int R) { return nt_of(R) * 8 * kfs(k); }

__device__ __forceinline__ void mma_f64(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// Complement decomposition per left string L (K orbitals; Lbar = the other NB = n - K orbitals).
// For a right string R with X = S[R, L], any n x K block W gives
//   tr(X^{-1} W[R, :]) = tr(T) + <V, Y^T>,   W = S[:, L] T + I[:, Lbar] V,
// with T = S[L,L]^{-1} W[L,:], V = W[Lbar,:] - S[Lbar,L] T, and Y = X^{-1} I[R, Lbar], a column
// selection of X^{-1}.  With W = B_m[:, L] (B_m[i][j] = lf(pair(i, j), m)) this is
// u[m] / det, and with W = h[:, L] it is H_1e / det (Jacobi's formula: both are first-order
// terms sum_{r,c} A(r,c) W(R_r, L_c) of det(X + eps W[R, :])).  T and V depend on L only.
//
// Table of left string L: row m (m < R factor columns, m = R one-electron h) of kfs(K) doubles
// holds V_m[b][c] at b K + c (b < nb_max(K), zero rows for b >= NB), tr T_m at nb_max(K) K,
// zeros elsewhere; rows R + 1 .. 8 nt_of(R) - 1 are zero.
template <int K>
__global__ void __launch_bounds__(128) left_string_tables(SpinTableArgs a, double* __restrict__ tables) {
    constexpr int NBMAX = nb_max(K);
    constexpr int KFS = kfs(K);
    const int table_stride = table_stride_of(K, a.R);
    __shared__ double sInv[K * K];
    __shared__ int sL[K], sLb[NBMAX];
    const int n = a.n;
    const int nb = n - K;
    const long long u = blockIdx.x;
    if (u >= a.n_strings) return;
    double* tab = tables + u * (long long)table_stride;
    for (int i = threadIdx.x; i < table_stride; i += blockDim.x) tab[i] = 0.0;
    if (threadIdx.x == 0) {
        const uint64_t w0 = a.occ[2 * u];
        int L[K];
#pragma unroll
        for (int c = 0; c < K; ++c) L[c] = (int)((w0 >> (8 * c)) & 0xFFu);
        uint64_t mask = 0;
#pragma unroll
        for (int c = 0; c < K; ++c) mask |= 1ull << L[c];
        int q = 0;
        for (int i = 0; i < n && q < NBMAX; ++i)
            if (!((mask >> i) & 1)) sLb[q++] = i;
        // S[L, L]^{-1} by Gauss-Jordan (S[L, L] is a principal block of an SPD matrix)
        double m[K][2 * K];
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
            for (int c = 0; c < 2 * K; ++c) m[r][c] = c < K ? a.S[L[r] * n + L[c]] : (c - K == r ? 1.0 : 0.0);
#pragma unroll
        for (int s = 0; s < K; ++s) {
            const double ip = 1.0 / m[s][s];
#pragma unroll
            for (int c = 0; c < 2 * K; ++c) m[s][c] *= ip;
#pragma unroll
            for (int r = 0; r < K; ++r) {
                if (r == s) continue;
                const double f = m[r][s];
#pragma unroll
                for (int c = 0; c < 2 * K; ++c) m[r][c] = fma(-f, m[s][c], m[r][c]);
            }
        }
#pragma unroll
        for (int r = 0; r < K; ++r) {
            sL[r] = L[r];
#pragma unroll
            for (int c = 0; c < K; ++c) sInv[r * K + c] = m[r][K + c];
        }
    }
    __syncthreads();
    const int blocks = a.R + 1;
    // one thread per (row m, column c): T[:, c] then V[:, c]; the c == 0 thread adds tr T_m
    for (int idx = threadIdx.x; idx < blocks * K; idx += blockDim.x) {
        const int mm = idx / K, c = idx % K;
        auto wval = [&](int i, int j) {
            return mm < a.R ? __ldg(a.lf + (long long)dev::pair_index(i, j) * a.ld + mm) : __ldg(a.h + i * n + j);
        };
        const int lc = sL[c];
        double wl[K];
#pragma unroll
        for (int ap = 0; ap < K; ++ap) wl[ap] = wval(sL[ap], lc);
        double tc[K];
#pragma unroll
        for (int r = 0; r < K; ++r) {
            double acc = 0.0;
#pragma unroll
            for (int ap = 0; ap < K; ++ap) acc = fma(sInv[r * K + ap], wl[ap], acc);
            tc[r] = acc;
        }
        double* row = tab + (long long)mm * KFS;
        for (int b = 0; b < nb && b < NBMAX; ++b) {
            const int ib = sLb[b];
            double acc = wval(ib, lc);
#pragma unroll
            for (int r = 0; r < K; ++r) acc = fma(-__ldg(a.S + ib * n + sL[r]), tc[r], acc);
            row[b * K + c] = acc;
        }
        if (c == 0) {
            double tr = 0.0;
            for (int cc = 0; cc < K; ++cc) {
                const int l2 = sL[cc];
                double acc = 0.0;
#pragma unroll
                for (int ap = 0; ap < K; ++ap) acc = fma(sInv[cc * K + ap], wval(sL[ap], l2), acc);
                tr += acc;
            }
            row[NBMAX * K] = tr;
        }
    }
}

// One CTA per contiguous range of work items (left string u, right strings v0 .. v0 + 127);
// the left string's tables live in shared memory and are reloaded only when u changes.
// Phase A (a thread per spin pair): overlap block, Gauss-Jordan inverse, certificate, the
// same-spin two-electron term, and the row Y of the pair (with 1 in the trace slot) to shared
// memory.  Phase B (a warp per 32 pairs): [u | H_1e] / det = Y V^T on the FP64 tensor cores
// (mma.sync m8n8k4), then the records.
template <int K>
__global__ void __launch_bounds__(kSpinBlock) spin_pairs_fast(SpinTableArgs a, const double* __restrict__ tables) {
    extern __shared__ double smem[];
    constexpr int CP = K * (K - 1) / 2;
    constexpr int NBMAX = nb_max(K);
    constexpr int KF = kf(K);
    constexpr int KFS = kfs(K);
    const int n = a.n;
    const int nb = n - K;
    const int gd = a.gamma_dim;
    const int R = a.R;
    const int NT = nt_of(R);
    const int table_stride = table_stride_of(K, R);
    double* sT = smem;                                // left-string table, row m = block m
    double* sY = sT + table_stride;                   // [pair][f] rows of Y
    double* sS = sY + kSpinBlock * KFS;               // [c][i] = S(i, L_c)
    double* sG = sS + ((K * n + 1) / 2 * 2);          // [cp][rp] = gamma(rp, pair(L_c1, L_c2))
    __shared__ int sLb[NBMAX];
    const long long N = a.n_strings;
    const int per = (a.n_items + gridDim.x - 1) / gridDim.x;
    const int item_begin = blockIdx.x * per;
    const int item_end = min(a.n_items, item_begin + per);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    long long loaded_u = -1;
    int L[K];
    for (int item = item_begin; item < item_end; ++item) {
        const int2 it = a.items[item];
        const long long u = it.x;
        if (u != loaded_u) {
            __syncthreads();
            const uint64_t wl = __ldg(a.occ + 2 * u);
#pragma unroll
            for (int c = 0; c < K; ++c) L[c] = (int)((wl >> (8 * c)) & 0xFFu);
            if (threadIdx.x == 0) {
                uint64_t mask = 0;
#pragma unroll
                for (int c = 0; c < K; ++c) mask |= 1ull << L[c];
                int q = 0;
                for (int i = 0; i < n && q < NBMAX; ++i)
                    if (!((mask >> i) & 1)) sLb[q++] = i;
            }
            for (int row = warp; row < K; row += nwarps) {
                int lc = 0;
#pragma unroll
                for (int cc = 0; cc < K; ++cc)
                    if (cc == row) lc = L[cc];
                for (int i = lane; i < n; i += 32) sS[row * n + i] = __ldg(a.S + lc * n + i);
            }
            if (K >= 2) {
                for (int cp = warp; cp < CP; cp += nwarps) {
                    int c2 = 1;
                    while ((c2 + 1) * c2 / 2 <= cp) ++c2;
                    const int c1 = cp - c2 * (c2 - 1) / 2;
                    int l1 = 0, l2 = 0;
#pragma unroll
                    for (int cc = 0; cc < K; ++cc) {
                        if (cc == c1) l1 = L[cc];
                        if (cc == c2) l2 = L[cc];
                    }
                    const double* src = a.gamma + (long long)dev::anti_index(l1, l2) * gd;
                    for (int rp = lane; rp < gd; rp += 32) sG[cp * gd + rp] = __ldg(src + rp);
                }
            }
            const double* tsrc = tables + u * (long long)table_stride;
            for (int i = threadIdx.x; i < table_stride; i += blockDim.x) sT[i] = __ldg(tsrc + i);
            loaded_u = u;
            __syncthreads();
        }
        // ---------------- phase A ----------------
        const long long v = (long long)it.y + threadIdx.x;
        bool ok = false;
        double det = 0.0, h2 = 0.0;
        long long t = 0;
        double* yrow = sY + threadIdx.x * KFS;
        if (v < N) {
            t = record_index(u, v, N);
            const uint64_t wr = __ldg(a.occ + 2 * v);
            int Rr[K];
#pragma unroll
            for (int c = 0; c < K; ++c) Rr[c] = (int)((wr >> (8 * c)) & 0xFFu);
            double x[K][K];
            double nx2 = 0.0;
#pragma unroll
            for (int r = 0; r < K; ++r)
#pragma unroll
                for (int c = 0; c < K; ++c) {
                    x[r][c] = sS[c * n + Rr[r]];
                    nx2 = fma(x[r][c], x[r][c], nx2);
                }
            constexpr int K0 = K <= 3 ? K : 1;
            double x0[K0][K0];
            if (K <= 3) {
#pragma unroll
                for (int r = 0; r < K0; ++r)
#pragma unroll
                    for (int c = 0; c < K0; ++c) x0[r][c] = x[r][c];
            }
            int lab[K];
#pragma unroll
            for (int r = 0; r < K; ++r) lab[r] = r;
            det = 1.0;
#pragma unroll
            for (int s = 0; s < K; ++s) {
                int p = s;
                double best = fabs(x[s][s]);
#pragma unroll
                for (int i = s + 1; i < K; ++i) {
                    const double av = fabs(x[i][s]);
                    if (av > best) {
                        best = av;
                        p = i;
                    }
                }
#pragma unroll
                for (int i = s + 1; i < K; ++i) {
                    const bool sw = (p == i);
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        const double a0 = x[s][j], a1 = x[i][j];
                        x[s][j] = sw ? a1 : a0;
                        x[i][j] = sw ? a0 : a1;
                    }
                    const int l0 = lab[s], l1 = lab[i];
                    lab[s] = sw ? l1 : l0;
                    lab[i] = sw ? l0 : l1;
                }
                if (p != s) det = -det;
                const double piv = x[s][s];
                det *= piv;
                const double ip = 1.0 / piv;
                x[s][s] = 1.0;
#pragma unroll
                for (int j = 0; j < K; ++j) x[s][j] *= ip;
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    if (i == s) continue;
                    const double f = x[i][s];
                    x[i][s] = 0.0;
#pragma unroll
                    for (int j = 0; j < K; ++j) x[i][j] = fma(-f, x[s][j], x[i][j]);
                }
            }
            double ni2 = 0.0;
#pragma unroll
            for (int r = 0; r < K; ++r)
#pragma unroll
                for (int c = 0; c < K; ++c) ni2 = fma(x[r][c], x[r][c], ni2);
            ok = isfinite(det) && det != 0.0 && (nx2 * ni2 < kCertificate2);
            if (!ok) {
                const unsigned long long slot = atomicAdd(a.careful_count, 1ull);
                a.careful_list[slot] = ((unsigned long long)u << 32) | (unsigned long long)v;
#pragma unroll
                for (int f = 0; f < KFS; ++f) yrow[f] = 0.0;
            } else {
                // x holds C = (P X)^{-1}: X^{-1}[c][lab[j]] = C[c][j]; row lab[j] carries orbital Rp[j]
                int Rp[K];
#pragma unroll
                for (int j = 0; j < K; ++j) Rp[j] = (int)((wr >> (8 * lab[j])) & 0xFFu);
                if (K == 2) {
                    h2 = sG[dev::anti_index(Rr[0], Rr[1])];
                } else if (K == 3) {
#pragma unroll
                    for (int r1 = 0; r1 < K0; ++r1)
#pragma unroll
                        for (int r2 = r1 + 1; r2 < K0; ++r2)
#pragma unroll
                            for (int c1 = 0; c1 < K0; ++c1)
#pragma unroll
                                for (int c2 = c1 + 1; c2 < K0; ++c2) {
                                    const double sign = ((r1 + r2 + c1 + c2) & 1) ? -1.0 : 1.0;
                                    const int cp = c2 * (c2 - 1) / 2 + c1;
                                    h2 = fma(sG[cp * gd + dev::anti_index(Rr[r1], Rr[r2])],
                                             sign * x0[3 - r1 - r2][3 - c1 - c2], h2);
                                }
                } else if (K >= 4) {
                    double acc2 = 0.0;
#pragma unroll
                    for (int j1 = 0; j1 < K; ++j1)
#pragma unroll
                        for (int j2 = j1 + 1; j2 < K; ++j2) {
                            const int ra = Rp[j1], rb = Rp[j2];
                            const bool ordered = ra < rb;
                            const int rp = dev::anti_index(ordered ? ra : rb, ordered ? rb : ra);
                            double part = 0.0;
#pragma unroll
                            for (int c1 = 0; c1 < K; ++c1)
#pragma unroll
                                for (int c2 = c1 + 1; c2 < K; ++c2) {
                                    const double m2 = fma(x[c1][j1], x[c2][j2], -x[c2][j1] * x[c1][j2]);
                                    part = fma(sG[(c2 * (c2 - 1) / 2 + c1) * gd + rp], m2, part);
                                }
                            acc2 += ordered ? part : -part;
                        }
                    h2 = det * acc2;
                }
                // Y[b K + c] = X^{-1}[c][r] for the row r carrying orbital Lbar_b (0 if Lbar_b not in R)
#pragma unroll
                for (int b = 0; b < NBMAX; ++b) {
                    const int ib = b < nb ? sLb[b] : -1;
#pragma unroll
                    for (int c = 0; c < K; ++c) {
                        double y = 0.0;
#pragma unroll
                        for (int j = 0; j < K; ++j) y = (Rp[j] == ib) ? x[c][j] : y;
                        yrow[b * K + c] = y;
                    }
                }
                yrow[NBMAX * K] = 1.0;
#pragma unroll
                for (int f = NBMAX * K + 1; f < KFS; ++f) yrow[f] = 0.0;
            }
        } else {
#pragma unroll
            for (int f = 0; f < KFS; ++f) yrow[f] = 0.0;
        }
        __syncwarp();
        // ---------------- phase B ----------------
        const double* Yw = sY + (warp * 32) * KFS;
        const int g = lane >> 2, tq = lane & 3;
        double det_m[4], h2_m[4];
        long long t_m[4];
        bool ok_m[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
            det_m[mt] = __shfl_sync(0xffffffffu, det, 8 * mt + g);
            h2_m[mt] = __shfl_sync(0xffffffffu, h2, 8 * mt + g);
            t_m[mt] = __shfl_sync(0xffffffffu, t, 8 * mt + g);
            ok_m[mt] = __shfl_sync(0xffffffffu, (int)ok, 8 * mt + g) != 0;
        }
        for (int nt0 = 0; nt0 < NT; nt0 += 6) {
            double acc[4][6][2];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int j = 0; j < 6; ++j) acc[mt][j][0] = acc[mt][j][1] = 0.0;
#pragma unroll
            for (int ks = 0; ks < KF / 4; ++ks) {
                double af[4], bf[6];
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) af[mt] = Yw[(8 * mt + g) * KFS + 4 * ks + tq];
#pragma unroll
                for (int j = 0; j < 6; ++j)
                    bf[j] = (nt0 + j < NT) ? sT[(8 * (nt0 + j) + g) * KFS + 4 * ks + tq] : 0.0;
#pragma unroll
                for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                    for (int j = 0; j < 6; ++j) mma_f64(acc[mt][j], af[mt], bf[j]);
            }
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) {
                if (!ok_m[mt]) continue;
                double* rec = a.records + t_m[mt] * (long long)a.rec_stride;
#pragma unroll
                for (int j = 0; j < 6; ++j)
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const int col = 8 * (nt0 + j) + 2 * tq + i;
                        const double val = det_m[mt] * acc[mt][j][i];
                        if (col < R) {
                            rec[col] = val;
                        } else if (col == R) {
                            rec[R + 0] = det_m[mt];
                            rec[R + 1] = val + h2_m[mt];
                            rec[R + 2] = val;
                            rec[R + 3] = 0.0;
                        }
                    }
            }
        }
        __syncwarp();
    }
}


// Listed blocks (or all blocks): one thread per block resolves it by the exact path; its first
// cofactors A go to the lane's shared slot (k^2 doubles).  The warp then treats its 32 blocks one
// at a time: the u-vectors of the records with the factor columns split over lanes, and, for
// full-rank blocks with k > 3, the regular two-electron sum (A11 A22 - A12 A21) / det
// (hamiltonian.cpp:83-123) with its C(k,2)^2 terms split over lanes, which keeps a block's
// latency short when only a few blocks are listed.  Rank-deficient blocks and k <= 3 are summed
// by their own thread: nullity 1 in the expanded form of the wedge second cofactors
//   parity prod sv * sum_{s<k-1} (u_s ^ u_n)(v_s ^ v_n) / sv_s            (contractions.cpp:937-963)
//   = Y(r1,c1) zu(r2) zv(c2) - Y(r1,c2) zu(r2) zv(c1) - Y(r2,c1) zu(r1) zv(c2) + Y(r2,c2) zu(r1) zv(c1),
// Y = parity sum_{s<k-1} u_s v_s^T prod_{l<k-1, l != s} sv_l; nullity 2 and k <= 3 by
// second_cofactor; nullity >= 3 is zero.  Dynamic shared memory: 32 k^2 doubles per warp.
template <int KM, int KC>  // KC > 0: electrons per string fixed at compile time (== KM)
__global__ void __launch_bounds__(64) spin_pairs_exact(SpinTableArgs a) {
    extern __shared__ double slots[];
    const long long count = a.all_careful ? a.n_pairs : (long long)(*a.careful_count);
    const int lane = threadIdx.x & 31;
    const int k = KC > 0 ? KC : a.k, kk = k * k, gd = a.gamma_dim;
    const int cp = k * (k - 1) / 2;
    double* wslot = slots + (size_t)(threadIdx.x >> 5) * 32 * kk;
    double* cof = wslot + (size_t)lane * kk;
    const long long N = a.n_strings;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < count; base += nwarps * 32) {
        const long long idx = base + lane;
        long long u = 0, v = 0;
        const bool valid = idx < count;
        double det = 0.0, h1 = 0.0, h2 = 0.0;
        int nullity = 3;
        bool regular = false;  // two-electron sum done by the warp
        if (valid) {
            if (a.all_careful) {
                const double b = 2.0 * (double)N + 1.0;
                long long uu = (long long)floor((b - sqrt(fmax(b * b - 8.0 * (double)idx, 0.0))) * 0.5);
                if (uu < 0) uu = 0;
                if (uu > N - 1) uu = N - 1;
                while (uu > 0 && uu * N - uu * (uu - 1) / 2 > idx) --uu;
                while (uu + 1 < N && (uu + 1) * N - (uu + 1) * uu / 2 <= idx) ++uu;
                u = uu;
                v = u + (idx - (u * N - u * (u - 1) / 2));
            } else {
                const unsigned long long w = a.careful_list[idx];
                u = (long long)(w >> 32);
                v = (long long)(w & 0xffffffffull);
            }
            int L[KM], R[KM];
            for (int c = 0; c < k; ++c) {
                L[c] = occ_byte(a.occ + 2 * u, c);
                R[c] = occ_byte(a.occ + 2 * v, c);
            }
            double x[KM * KM];
            for (int c = 0; c < k; ++c)
                for (int r = 0; r < k; ++r) x[c * k + r] = __ldg(a.S + R[r] * a.n + L[c]);
            dev::ResolutionT<KM> res;
            dev::resolve_exact<KM>(k, x, kThreshold, &res);
            dev::first_cofactor<KM>(res, cof);
            det = res.det;
            nullity = res.nullity;
            regular = res.nullity == 0 && k > 3;
            if (res.nullity < 3) {
                if (res.nullity <= 1)
                    for (int c = 0; c < k; ++c)
                        for (int r = 0; r < k; ++r) h1 = fma(__ldg(a.h + L[c] * a.n + R[r]), cof[c * k + r], h1);
                if (!regular) {
                    const bool rank1 = res.nullity == 1 && k > 3;
                    double Y[KM * KM], zu[KM], zv[KM];
                    if (rank1) {
                        const int ni = k - 1;
                        double w[KM];
                        for (int s2 = 0; s2 < ni; ++s2) {
                            double p = res.parity;
                            for (int l = 0; l < ni; ++l)
                                if (l != s2) p *= res.sv[l];
                            w[s2] = p;
                        }
                        for (int r = 0; r < k; ++r) {
                            zu[r] = res.u[ni * k + r];
                            zv[r] = res.v[ni * k + r];
                            for (int c = 0; c < k; ++c) {
                                double acc = 0.0;
                                for (int s2 = 0; s2 < ni; ++s2) acc = fma(res.u[s2 * k + r] * w[s2], res.v[s2 * k + c], acc);
                                Y[r * k + c] = acc;
                            }
                        }
                    }
                    for (int r2 = 1; r2 < k; ++r2)
                        for (int r1 = 0; r1 < r2; ++r1) {
                            const double* grow = a.gamma + (long long)dev::anti_index(R[r1], R[r2]) * gd;
                            double part = 0.0;
                            for (int c2 = 1; c2 < k; ++c2)
                                for (int c1 = 0; c1 < c2; ++c1) {
                                    const double g = __ldg(grow + dev::anti_index(L[c1], L[c2]));
                                    const double m2 = rank1 ? Y[r1 * k + c1] * zu[r2] * zv[c2] - Y[r1 * k + c2] * zu[r2] * zv[c1] -
                                                                  Y[r2 * k + c1] * zu[r1] * zv[c2] + Y[r2 * k + c2] * zu[r1] * zv[c1]
                                                            : dev::second_cofactor<KM>(res, r1, r2, c1, c2);
                                    part = fma(g, m2, part);
                                }
                            h2 += part;
                        }
                }
            }
            if (res.nullity > 1)
                for (int i = 0; i < kk; ++i) cof[i] = 0.0;
        }
        __syncwarp();
        for (int j = 0; j < 32; ++j) {
            const long long jdx = base + j;
            if (jdx >= count) break;
            const long long uj = __shfl_sync(0xffffffffu, u, j), vj = __shfl_sync(0xffffffffu, v, j);
            const uint64_t* ol = a.occ + 2 * uj;
            const uint64_t* orr = a.occ + 2 * vj;
            const double* cj = wslot + (size_t)j * kk;
            // regular two-electron sum of block j, terms split over lanes: gamma[(R r1, R r2)][(L c1, L c2)]
            // is (r1 c1 | r2 c2) - (r1 c2 | r2 c1)
            if (__shfl_sync(0xffffffffu, (int)regular, j)) {
                double part = 0.0;
                for (int q = lane; q < cp * cp; q += 32) {
                    const int rp = q / cp, cq = q % cp;
                    int r2 = 1;
                    while ((r2 + 1) * r2 / 2 <= rp) ++r2;
                    const int r1 = rp - r2 * (r2 - 1) / 2;
                    int c2 = 1;
                    while ((c2 + 1) * c2 / 2 <= cq) ++c2;
                    const int c1 = cq - c2 * (c2 - 1) / 2;
                    const double g = __ldg(a.gamma + (long long)dev::anti_index(occ_byte(orr, r1), occ_byte(orr, r2)) * gd +
                                           dev::anti_index(occ_byte(ol, c1), occ_byte(ol, c2)));
                    part = fma(g, cj[c1 * k + r1] * cj[c2 * k + r2] - cj[c2 * k + r1] * cj[c1 * k + r2], part);
                }
                for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
                if (lane == j) h2 = part / det;
            }
            // u-vectors: u_m = sum_{c,r} A(r,c) l_m[pair(R_r, L_c)]
            double* rec = a.records + record_index(uj, vj, N) * (long long)a.rec_stride;
            for (int m = lane; m < a.R; m += 32) {
                double acc = 0.0;
                for (int c = 0; c < k; ++c) {
                    const int lc = occ_byte(ol, c);
                    for (int r = 0; r < k; ++r) {
                        const double cv = cj[c * k + r];
                        if (cv != 0.0)
                            acc = fma(cv, __ldg(a.lf + (long long)dev::pair_index(occ_byte(orr, r), lc) * a.ld + m), acc);
                    }
                }
                rec[m] = acc;
            }
        }
        if (valid) {
            double* rec = a.records + record_index(u, v, N) * (long long)a.rec_stride;
            rec[a.R + 0] = det;
            rec[a.R + 1] = nullity < 3 ? h1 + h2 : 0.0;
            rec[a.R + 2] = nullity < 3 ? h1 : 0.0;
            rec[a.R + 3] = (double)nullity;
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void band_decode(long long t, long long e0, long long e1, long long* d, long long* e) {
    const long long B = e1 - e0;
    const long long rect = e0 * B;
    if (t < rect) {
        *d = t / B;
        *e = e0 + t % B;
        return;
    }
    const long long tp = t - rect;
    const double b2 = 2.0 * (double)B + 1.0;
    long long i = (long long)floor((b2 - sqrt(fmax(b2 * b2 - 8.0 * (double)tp, 0.0))) * 0.5);
    if (i < 0) i = 0;
    if (i > B - 1) i = B - 1;
    while (i > 0 && i * B - i * (i - 1) / 2 > tp) --i;
    while (i + 1 < B && (i + 1) * B - (i + 1) * i / 2 <= tp) ++i;
    *d = e0 + i;
    *e = *d + (tp - (i * B - i * (i - 1) / 2));
}

// Weight of the upper-triangle pair (d <= e) in H_d = U' + U'^T: 1/2 on the diagonal, and,
// with a spin-flip permutation, the unordered pairs {d, e} and {flip d, flip e} (same H_de and,
// for structures whose coefficients are flip-invariant, the same coefficient products) fold
// onto one representative with twice the weight; the other member gets weight 0.
__device__ __forceinline__ double pair_weight(const int* flip, long long d, long long e) {
    const double w = (d == e) ? 0.5 : 1.0;
    if (!flip) return w;
    const long long fd = __ldg(flip + d), fe = __ldg(flip + e);
    const long long d2 = fd < fe ? fd : fe, e2 = fd < fe ? fe : fd;
    if (d < d2 || (d == d2 && e < e2)) return 2.0 * w;
    if (d == d2 && e == e2) return w;
    return 0.0;
}

__global__ void __launch_bounds__(512) full_pairs_kernel(FullPairArgs a) {
    const long long B = a.e1 - a.e0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < a.n_items; t += stride) {
        long long d, e;
        band_decode(t, a.e0, a.e1, &d, &e);
        const double w = pair_weight(a.flip, d, e);
        double H = 0.0, S = 0.0;
        if (w != 0.0) {
            pair_value(a, d, e, &H, &S);
            H *= w;
            S *= w;
        }
        const long long o = d * B + (e - a.e0);
        a.Hb[o] = H;
        a.Sb[o] = S;
    }
}

// Listed determinant pairs (d, e) in any order.
__global__ void listed_pairs_kernel(FullPairArgs a, long long n_pairs, const long long* __restrict__ pairs,
                                    double* __restrict__ h_out, double* __restrict__ s_out) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n_pairs;
         t += (long long)gridDim.x * blockDim.x) {
        double H, S;
        pair_value(a, pairs[2 * t], pairs[2 * t + 1], &H, &S);
        h_out[t] = H;
        s_out[t] = S;
    }
}

__global__ void resolve_blocks_kernel(int k, long long batch, const double* __restrict__ blocks, double* det,
                                      int* nullity, double* cof_out) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < batch;
         t += (long long)gridDim.x * blockDim.x) {
        dev::Resolution res;
        dev::resolve_exact(k, blocks + t * k * k, kThreshold, &res);
        double cof[dev::KMAX * dev::KMAX];
        dev::first_cofactor(res, cof);
        det[t] = res.det;
        nullity[t] = res.nullity;
        if (cof_out)
            for (int i = 0; i < k * k; ++i) cof_out[t * k * k + i] = res.nullity <= 1 ? cof[i] : 0.0;
    }
}

__global__ void same_spin_list_kernel(int n, int k, long long batch, const int* __restrict__ occ_left,
                                      const int* __restrict__ occ_right, const double* __restrict__ S,
                                      const double* __restrict__ h, const double* __restrict__ eri, double* scalars,
                                      double* cof_out) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < batch;
         t += (long long)gridDim.x * blockDim.x) {
        int L[dev::KMAX], R[dev::KMAX];
        for (int i = 0; i < k; ++i) {
            L[i] = occ_left[t * k + i];
            R[i] = occ_right[t * k + i];
        }
        double x[dev::KMAX * dev::KMAX];
        for (int c = 0; c < k; ++c)
            for (int r = 0; r < k; ++r) x[c * k + r] = S[L[c] * n + R[r]];
        dev::Resolution res;
        dev::resolve_exact(k, x, kThreshold, &res);
        double cof[dev::KMAX * dev::KMAX];
        dev::first_cofactor(res, cof);
        double h1 = 0.0, htot = 0.0;
        if (k > 0 && res.nullity < 3) htot = dev::same_spin_exact(n, k, L, R, res, cof, h, eri, &h1);
        scalars[4 * t + 0] = res.det;
        scalars[4 * t + 1] = h1;
        scalars[4 * t + 2] = htot;
        scalars[4 * t + 3] = (double)res.nullity;
        if (cof_out)
            for (int i = 0; i < k * k; ++i) cof_out[t * k * k + i] = res.nullity <= 1 ? cof[i] : 0.0;
    }
}

template <int K>
cudaError_t launch_fast(const SpinTableArgs& a, size_t smem, double* tables, cudaStream_t stream) {
    left_string_tables<K><<<a.n_strings, 128, 0, stream>>>(a, tables);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    err = allow_dynamic_smem((const void*)spin_pairs_fast<K>, (int)smem);
    if (err != cudaSuccess) return err;
    int per_sm = 1;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spin_pairs_fast<K>, kSpinBlock, smem);
    if (err != cudaSuccess) return err;
    int blocks = kSms * (per_sm > 0 ? per_sm : 1);
    if (blocks > a.n_items) blocks = a.n_items;
    if (blocks < 1) blocks = 1;
    spin_pairs_fast<K><<<blocks, kSpinBlock, smem, stream>>>(a, tables);
    return cudaGetLastError();
}

}  // namespace

size_t left_table_doubles(int n, int k, int R) {
    (void)n;
    return (size_t)table_stride_of(k, R);
}

size_t factored_spin_smem_bytes(int n, int k, int R) {
    const size_t gd = (size_t)n * (n - 1) / 2;
    const size_t cp = (size_t)k * (k - 1) / 2;
    return sizeof(double) * (left_table_doubles(n, k, R) + (size_t)kSpinBlock * kfs(k) + (size_t)((k * n + 1) / 2 * 2) +
                             (k >= 2 ? cp * gd : 0));
}

bool fast_spin_supported(int n, int k, int R) {
    return k >= 1 && k <= 8 && n - k >= 0 && n - k <= nb_max(k) && factored_spin_smem_bytes(n, k, R) <= 200 * 1024;
}

cudaError_t launch_factor_pair_kernel(int np, const double* kfull, double* work, double* cols, int* signs, double* lf,
                                      int ld, int* meta, cudaStream_t stream) {
    const size_t in_smem_bytes = sizeof(double) * (size_t)np * np + sizeof(int) * 2 * (size_t)np;
    const int in_smem = in_smem_bytes <= 200 * 1024 ? 1 : 0;
    const size_t smem = in_smem ? in_smem_bytes : sizeof(int) * 2 * (size_t)np;
    cudaError_t err = allow_dynamic_smem((const void*)factor_pair_kernel, (int)smem);
    if (err != cudaSuccess) return err;
    factor_pair_kernel<<<1, 512, smem, stream>>>(np, kfull, work, cols, signs, lf, ld, meta, kFactorTolerance, in_smem);
    return cudaGetLastError();
}

cudaError_t launch_prepare_tables(int n, const double* eri, double* gamma, double* kfull, cudaStream_t stream) {
    const long long np = (long long)n * (n + 1) / 2, gd = (long long)n * (n - 1) / 2;
    long long total = np * np + gd * gd;
    long long blocks = (total + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    prepare_tables_kernel<<<(unsigned)blocks, 256, 0, stream>>>(n, eri, gamma, kfull);
    return cudaGetLastError();
}

size_t exact_stack_bytes() {
    size_t m = 0;
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, spin_pairs_exact<8, 0>) == cudaSuccess) m = std::max(m, fa.localSizeBytes);
    if (cudaFuncGetAttributes(&fa, spin_pairs_exact<7, 7>) == cudaSuccess) m = std::max(m, fa.localSizeBytes);
    return m;
}

cudaError_t preload_spin_pair_kernels() {
    // cudaFuncGetAttributes loads a function that lazy module loading has not loaded yet
    const void* fns[] = {(const void*)prepare_tables_kernel, (const void*)factor_pair_kernel,
                         (const void*)left_string_tables<1>, (const void*)left_string_tables<2>,
                         (const void*)left_string_tables<3>, (const void*)left_string_tables<4>,
                         (const void*)left_string_tables<5>, (const void*)left_string_tables<6>,
                         (const void*)left_string_tables<7>, (const void*)left_string_tables<8>,
                         (const void*)spin_pairs_fast<1>, (const void*)spin_pairs_fast<2>,
                         (const void*)spin_pairs_fast<3>, (const void*)spin_pairs_fast<4>,
                         (const void*)spin_pairs_fast<5>, (const void*)spin_pairs_fast<6>,
                         (const void*)spin_pairs_fast<7>, (const void*)spin_pairs_fast<8>,
                         (const void*)spin_pairs_exact<7, 7>, (const void*)spin_pairs_exact<8, 0>,
                         (const void*)spin_pairs_exact<dev::KMAX, 0>};
    for (const void* f : fns) {
        cudaFuncAttributes fa{};
        const cudaError_t err = cudaFuncGetAttributes(&fa, f);
        if (err != cudaSuccess) return err;
    }
    return preload_frame_kernels();
}

cudaError_t launch_spin_tables(const SpinTableArgs& a, double* tables, cudaStream_t stream, int* launches) {
    if (a.n_pairs <= 0 || a.k <= 0 || a.all_careful || !frame_spin_supported(a.n, a.k, a.R)) return cudaSuccess;
    ++*launches;
    return launch_frame_tables(a, tables, stream);
}

cudaError_t launch_spin_pairs(const SpinTableArgs& a, double* tables, cudaStream_t stream, int* launches) {
    if (a.n_pairs <= 0 || a.k <= 0) return cudaSuccess;
    cudaError_t err = cudaSuccess;
    const bool fast_ok = !a.all_careful && frame_spin_supported(a.n, a.k, a.R);
    if (fast_ok) {
        // the pair-to-warp schedule (warps per CTA) is chosen by the autotuner per shape; the
        // listed-pair counter and the task counter are restored before every timed launch
        const std::string key = "spin_pairs_frame k=" + std::to_string(a.k) + " n=" + std::to_string(a.n) +
                                " R=" + std::to_string(a.R) + " N=" + std::to_string(a.n_strings);
        const int tuned = autotune_run(
            key, frame_pair_variants(a.n, a.k, a.R), stream, [&](int v) { return launch_frame_pairs(a, tables, stream, v); },
            [&]() {
                cudaError_t e = cudaMemsetAsync(a.careful_count, 0, sizeof(unsigned long long), stream);
                if (e == cudaSuccess) e = cudaMemsetAsync(a.task_counter, 0, sizeof(unsigned long long), stream);
                return e;
            },
            &err);
        (void)tuned;
        if (err != cudaSuccess) return err;
        ++*launches;
    }
    SpinTableArgs b = a;
    b.all_careful = fast_ok ? 0 : 1;
    auto exact = a.k == 7 ? spin_pairs_exact<7, 7> : (a.k <= 8 ? spin_pairs_exact<8, 0> : spin_pairs_exact<dev::KMAX, 0>);
    const size_t slot_bytes = sizeof(double) * 64 * (size_t)a.k * a.k;  // two warps
    if (slot_bytes > 48 * 1024) {
        err = allow_dynamic_smem((const void*)exact, (int)slot_bytes);
        if (err != cudaSuccess) return err;
    }
    exact<<<kSms * 8, 64, slot_bytes, stream>>>(b);
    ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_full_pairs(const FullPairArgs& a, cudaStream_t stream, int* launches) {
    if (a.n_items <= 0) return cudaSuccess;
    // launch variants (block size, CTAs per SM), chosen by the autotuner per band shape
    constexpr int kVariants = 4;
    constexpr int threads[kVariants] = {256, 128, 256, 512};
    constexpr int per_sm[kVariants] = {16, 16, 8, 4};
    const std::string key = "full_pairs_kernel R=" + std::to_string(a.R) + " ndet=" + std::to_string(a.n_det) +
                            " items=" + std::to_string(a.n_items) + " flip=" + std::to_string(a.flip ? 1 : 0);
    cudaError_t err = cudaSuccess;
    autotune_run(
        key, kVariants, stream,
        [&](int v) {
            long long blocks = (a.n_items + threads[v] - 1) / threads[v];
            if (blocks > (long long)kSms * per_sm[v]) blocks = (long long)kSms * per_sm[v];
            full_pairs_kernel<<<(unsigned)blocks, threads[v], 0, stream>>>(a);
            return cudaGetLastError();
        },
        {}, &err);
    ++*launches;
    return err;
}

cudaError_t launch_listed_pairs(const FullPairArgs& a, long long n_pairs, const long long* pairs, double* h_out,
                                double* s_out, cudaStream_t stream) {
    if (n_pairs <= 0) return cudaSuccess;
    long long blocks = (n_pairs + 127) / 128;
    if (blocks > kSms * 16) blocks = kSms * 16;
    listed_pairs_kernel<<<(unsigned)blocks, 128, 0, stream>>>(a, n_pairs, pairs, h_out, s_out);
    return cudaGetLastError();
}

cudaError_t launch_resolve_blocks(int k, long long batch, const double* blocks, double* det, int* nullity, double* cof,
                                  cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    long long g = (batch + 63) / 64;
    if (g > kSms * 8) g = kSms * 8;
    resolve_blocks_kernel<<<(unsigned)g, 64, 0, stream>>>(k, batch, blocks, det, nullity, cof);
    return cudaGetLastError();
}

cudaError_t launch_same_spin_list(int n, int k, long long batch, const int* occ_left, const int* occ_right,
                                  const double* S, const double* h, const double* eri, double* scalars, double* cof,
                                  cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    long long g = (batch + 63) / 64;
    if (g > kSms * 8) g = kSms * 8;
    same_spin_list_kernel<<<(unsigned)g, 64, 0, stream>>>(n, k, batch, occ_left, occ_right, S, h, eri, scalars, cof);
    return cudaGetLastError();
}

}  // namespace vbcore
