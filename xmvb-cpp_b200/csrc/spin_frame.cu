// Spin-pair records in the left string's biorthogonal frame (sm_100a).
//
// For a left string L (K orbitals; Lbar = the other NB = n - K orbitals) let S_LL = S[L, L],
// Sinv = S_LL^-1 and P = S[:, L] Sinv (so P[L, :] = I).  For a right string R with holes
// h_1 < ... < h_E (positions of L's orbitals missing from R) and particles p_1 < ... < p_E
// (R's orbitals outside L, as Lbar indices), the overlap block X = S[R, L] (rows = right string)
// factors as X = P[R, :] S_LL, and P[R, :] is the identity on the rows R shares with L.  So
//   det X = sign det S_LL det B,      B(i, j) = P[p_i, h_j]   (E x E),
// with sign the parity of the row-to-column assignment, and with W = B^-1 every first-order
// quantity tr(X^-1 Z[R, :]) of an n x K block Z = Z_m[:, L] is
//   tr(T_m) + sum_{i,j} W(j, i) Vt_m(p_i, h_j),   T_m = Sinv Z[L, :],
//   Vt_m = (Z[Lbar, :] - S[Lbar, L] T_m) Sinv,
// (Jacobi's formula in the L frame).  Z_m = B_m[:, L] (factor column m of the pair kernel)
// gives the u-vector u_m / det X, Z = h[:, L] the one-electron energy / det X.  With the
// factored pair kernel (ij|kl) = sum_m sigma_m B_m(ij) B_m(kl), the same-spin two-electron
// energy of hamiltonian.cpp:83-123 (sum over c1<c2, r1<r2 of [(r1c1|r2c2) - (r1c2|r2c1)] times
// the second cofactor) divided by det X is (1/2) sum_m sigma_m [tr(M_m)^2 - tr(M_m^2)] with
// M_m = T'_m + Y' Vt_m in the same frame (Y' carries W on the hole x particle block), i.e.
//   E2c(L) + sum_{i,j} W(j, i) l(p_i, h_j) + sum_{i<i', j<j'} Q(p_i p_i', h_j h_j') minor_W,
//   E2c = 1/2 sum sigma (tr T^2... ) [constant], l = sum sigma (tr T Vt - V T Sinv) [linear],
//   Q(b b', c c') = sum sigma [Vt(b,c) Vt(b',c') - Vt(b,c') Vt(b',c)]           [quadratic],
// and minor_W the 2 x 2 minor of W on holes (j, j') and particles (i, i').  Per pair this leaves
// an E x E inverse and C(E,2)^2 quadratic terms instead of a K x K inverse and C(K,2)^2 terms.
//
// Kernels:
//  * sort_right_strings<K> (once per string table): for each left string u, the right strings
//    v >= u bucketed by hole set, buckets in order of excitation level E then hole mask, each with
//    a descriptor (hole mask, particle mask, sign of the assignment);
//  * frame_tables<K> (per evaluation, one CTA per left string): Sinv, P, the table rows
//    [h | 2e linear | factor columns] over the (hole position x particle) grid plus a trace slot,
//    Q, and the norms of the conditioning certificate;
//  * spin_pairs_frame<K> (persistent): a CTA takes left strings from a counter, stages the
//    string's block in shared memory, and its warps take chunks of 32 pairs of one excitation
//    level E (so every lane runs the same compile-time-E code).  Phase A, a lane per pair: B,
//    Gauss-Jordan with partial pivoting, sign, certificate, quadratic two-electron term, and the
//    pair's row Y' (W scattered onto the grid, 1 in the trace slot) to shared memory.  Phase B,
//    per 8-pair tile: [h | 2e-linear | u] / det X = Y' Table^T on the FP64 tensor cores
//    (mma.sync m8n8k4), k-steps only over the hole positions present in the tile (pairs are
//    sorted by hole set, so a tile's union is usually its own hole set).
// Blocks failing the certificate go to the exact path (spin_pairs_exact) through the list.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "device_algebra.cuh"
#include "internal.h"
#include "kernels.h"
#include "pair_value.cuh"

namespace vbcore {
namespace {

constexpr int kFrameWarps = 4;  // warps per CTA of the bucketing kernel
constexpr int kFrameThreads = 32 * kFrameWarps;
constexpr int kFrameMaxWarps = 8;  // warps per CTA of the pair kernel: a launch variant (2, 4 or 8)

__host__ __device__ constexpr int fr_nbmax(int K) { return K <= 4 ? K + 4 : K; }
__host__ __device__ constexpr int fr_kfs(int K) { return 8 * K + 4; }  // 8 columns per hole position + trace block
__host__ __device__ constexpr int fr_cp(int K) { return K * (K - 1) / 2; }
__host__ __device__ constexpr int fr_bp(int K) { return fr_nbmax(K) * (fr_nbmax(K) - 1) / 2; }

// Layout of one left string's block (doubles; every part starts on a 2-double boundary).
struct FrameLayout {
    int rows;    // table rows: 0 = h, 1 = two-electron linear part, 2 + m = factor column m; padded to 8
    int kfs;     // table row stride
    int o_q;     // Q[bp * CP + cp]
    int o_p;     // P[b * K + c]
    int o_rowsq; // sum_c S(o, L_c)^2 for o = L_0 .. L_{K-1}, then o = Lbar_0 .. Lbar_{NBM-1}
    int o_prow2; // sum_c P(b, c)^2
    int o_scal;  // det S_LL, ||Sinv||_F^2, sum_c rowsq(L_c)
    int total;
};

__host__ __device__ inline int even_up(int x) { return (x + 1) / 2 * 2; }

__host__ __device__ inline FrameLayout frame_layout(int n, int K, int R) {
    (void)n;
    FrameLayout f{};
    f.rows = (R + 2 + 7) / 8 * 8;
    f.kfs = fr_kfs(K);
    int o = f.rows * f.kfs;
    f.o_q = o;
    o += even_up(fr_bp(K) * fr_cp(K));
    f.o_p = o;
    o += even_up(fr_nbmax(K) * K);
    f.o_rowsq = o;
    o += even_up(K + fr_nbmax(K));
    f.o_prow2 = o;
    o += even_up(fr_nbmax(K));
    f.o_scal = o;
    o += 4;
    f.total = o;
    return f;
}

__device__ __forceinline__ void mma_f64(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ uint64_t occ_mask(uint64_t w, int k) {
    uint64_t m = 0;
    for (int c = 0; c < k; ++c) m |= 1ull << ((w >> (8 * c)) & 0xFFu);
    return m;
}

// Hole mask of (L, R): bit c set when L's c-th orbital is not in R.
template <int K>
__device__ __forceinline__ unsigned hole_mask(uint64_t wL, uint64_t mR) {
    unsigned hm = 0;
#pragma unroll
    for (int c = 0; c < K; ++c) hm |= ((mR >> ((wL >> (8 * c)) & 0xFFu)) & 1ull) ? 0u : (1u << c);
    return hm;
}

// One warp per left string u.  Buckets: hole mask x (2^K of them), ordered by (popcount, x);
// within a bucket, v ascending (the scatter walks v in order and ranks lanes within a warp).
// Descriptor of the pair (L, R): bits 0-7 hole mask (positions in L), bits 8-15 particle mask
// (indices in Lbar), bit 16 the parity of the row (R order) -> column (L position) assignment
// that takes common orbitals to their positions and the i-th particle to the i-th hole.
template <int K>
__device__ __forceinline__ unsigned pair_descriptor(uint64_t wL, uint64_t mL, uint64_t mR) {
    const unsigned hm = hole_mask<K>(wL, mR);
    unsigned pbar = 0;
    uint64_t pm = mR & ~mL;
    while (pm) {
        const int o = __ffsll((long long)pm) - 1;
        pm &= pm - 1;
        pbar |= 1u << __popcll(~mL & ((1ull << o) - 1ull));
    }
    int inv = 0;
    uint64_t rest = mR;
    unsigned hrest = hm, seen = 0;
#pragma unroll
    for (int r = 0; r < K; ++r) {
        const int o = __ffsll((long long)rest) - 1;
        rest &= rest - 1;
        int t;
        if ((mL >> o) & 1ull) {
            t = __popcll(mL & ((1ull << o) - 1ull));
        } else {
            t = __ffs(hrest) - 1;
            hrest &= hrest - 1;
        }
        inv += __popc(seen >> t);
        seen |= 1u << t;
    }
    return hm | (pbar << 8) | ((unsigned)(inv & 1) << 16);
}

template <int K>
__global__ void __launch_bounds__(kFrameThreads) sort_right_strings(int N, const uint64_t* __restrict__ occ,
                                                                   int* __restrict__ rlist, unsigned* __restrict__ rdesc,
                                                                   int* __restrict__ ebound) {
    constexpr int NBINS = 1 << K;
    __shared__ int cursor[kFrameWarps][NBINS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int u = blockIdx.x * kFrameWarps + warp;
    if (u >= N) return;
    int* cur = cursor[warp];
    for (int x = lane; x < NBINS; x += 32) cur[x] = 0;
    __syncwarp();
    const uint64_t wL = __ldg(occ + 2 * (long long)u);
    for (int v0 = u; v0 < N; v0 += 32) {
        const int v = v0 + lane;
        const int hm = v < N ? (int)hole_mask<K>(wL, occ_mask(__ldg(occ + 2 * (long long)v), K)) : -1;
        const unsigned same = __match_any_sync(0xffffffffu, hm);
        if (hm >= 0 && lane == __ffs(same) - 1) cur[hm] += __popc(same);
        __syncwarp();
    }
    if (lane == 0) {
        int run = 0;
        int* eb = ebound + (long long)u * (K + 2);
        for (int e = 0; e <= K; ++e) {
            eb[e] = run;
            for (int x = 0; x < NBINS; ++x)
                if (__popc(x) == e) {
                    const int c = cur[x];
                    cur[x] = run;
                    run += c;
                }
        }
        eb[K + 1] = run;
    }
    __syncwarp();
    const long long base = record_index(u, u, N);
    const uint64_t mL = occ_mask(wL, K);
    for (int v0 = u; v0 < N; v0 += 32) {
        const int v = v0 + lane;
        const uint64_t mR = v < N ? occ_mask(__ldg(occ + 2 * (long long)v), K) : 0;
        const int hm = v < N ? (int)hole_mask<K>(wL, mR) : -1;
        const unsigned same = __match_any_sync(0xffffffffu, hm);
        int pos = 0;
        if (hm >= 0) pos = cur[hm] + __popc(same & ((1u << lane) - 1u));
        __syncwarp();
        if (hm >= 0) {
            rlist[base + pos] = v;
            rdesc[base + pos] = pair_descriptor<K>(wL, mL, mR);
            if (lane == __ffs(same) - 1) cur[hm] += __popc(same);
        }
        __syncwarp();
    }
}

constexpr int kTableThreads = 128;  // four warps
constexpr int kTableWarps = kTableThreads / 32;
constexpr int kTableSources = 20;   // pair-kernel sources (h and factor columns) staged per pass
constexpr int kZS = 129;            // shared-memory stride of one staged source (odd: no conflicts)
constexpr int kXS = 20;             // stride of one Vt entry over the sources (>= kTableSources,
                                    // = 4 mod 16: fragment loads without bank conflicts)

__host__ __device__ inline int table_sources(int R) { return R + 1 < kTableSources ? R + 1 : kTableSources; }

// Per-left-string tables, one CTA per string u (dynamic shared memory: frame_tables_smem).  With
// Y_s = Z_s[:, L] Sinv for each source s (Z_0 = h, Z_{1+m} = B_m), taken on the rows L (YL_s) and
// Lbar (YB_s):
//   Vt_s = YB_s - P YL_s,  tr T_s = tr YL_s,  tr T_s^2 = tr YL_s^2,  V_s T_s Sinv = Vt_s YL_s,
// every product is an 8 x 8 tile (K, the complement and the hole positions are at most 8) on the
// FP64 tensor cores (mma.sync m8n8k4): per source, Y_s from the staged rows [L; Lbar] of Z_s
// (two row tiles), Vt_s with the accumulator started at YB_s, and Vt_s YL_s; the linear table
// accumulates sigma_s (tr T_s Vt_s - Vt_s YL_s) in each warp's accumulator fragments.  The
// quadratic table needs M = sum_s sigma_s x_s x_s^T over x_s = vec Vt_s (64 x 64, its 36 upper
// tiles spread over the warps, k-steps over four sources at a time):
//   Q(b b', c c') = M[(b c), (b' c')] - M[(b c'), (b' c)].
template <int K>
__global__ void __launch_bounds__(kTableThreads, 4) frame_tables(SpinTableArgs a, double* __restrict__ tables) {
    constexpr int NBM = fr_nbmax(K);
    constexpr int CP = fr_cp(K);
    constexpr int BP = fr_bp(K);
    constexpr int KFS = fr_kfs(K);
    constexpr int NQ = BP * CP;
    constexpr int MT = 36;                                     // upper 8 x 8 tiles of M
    constexpr int MT_W = (MT + kTableWarps - 1) / kTableWarps;  // tiles per warp
    extern __shared__ double dsm[];
    const int n = a.n, R = a.R;
    const int nb = n - K;
    const int SC = table_sources(R);
    const FrameLayout F = frame_layout(n, K, R);
    __shared__ int sL[8], sLb[8];
    __shared__ double sM[K][2 * K], sF[K], sSinv[64], sP[64], sDet;
    __shared__ double sE2[kTableWarps];
    __shared__ int sOff[128];  // per staged slot (row, column): offset of its pair row in lf / in h
    // Shared-memory layouts are chosen so that every fragment load of the tensor-core steps reads
    // 32 consecutive doubles (lane order) or an odd stride, i.e. without bank conflicts:
    //  sZ  [SC][kZS]: rows [L; Lbar] of Z_s as (k half, row, k mod 4): h * 64 + row * 4 + c % 4,
    //                 then M (64 x 64) at the end
    //  sX  [64][kXS]: Vt_s entry (b * 8 + c), source fastest
    //  sYL [warps][64]: YL_s as a B operand (k half, column, k mod 4)
    //  sVA [warps][64]: Vt_s as an A operand (k half, row, k mod 4)
    double* sZ = dsm;
    double* sX = sZ + (SC * kZS > 4096 ? SC * kZS : 4096);
    double* sYL = sX + 64 * kXS;
    double* sVA = sYL + kTableWarps * 64;
    double* sLin = sVA + kTableWarps * 64;                  // [warps][64] linear-table partials
    const long long u = blockIdx.x;
    if (u >= a.n_strings) return;
    double* blk = tables + u * (long long)F.total;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gr = lane >> 2, gc = lane & 3;  // fragment row / column-in-group
    const uint64_t w0 = a.occ[2 * u];
    for (int i = tid; i < F.total; i += kTableThreads) blk[i] = 0.0;
    if (tid == 0) {
        const uint64_t mask = occ_mask(w0, K);
        int q = 0;
        for (int i = 0; i < n && q < NBM; ++i)
            if (!((mask >> i) & 1)) sLb[q++] = i;
        for (; q < 8; ++q) sLb[q] = -1;
    }
    if (tid < 8) sL[tid] = tid < K ? (int)((w0 >> (8 * tid)) & 0xFFu) : -1;
    for (int e = tid; e < 64; e += kTableThreads) {
        sSinv[e] = 0.0;
        sP[e] = 0.0;
    }
    __syncthreads();
    // slot (r, c) of a staged source holds Z_s(i, L_c) for i = L_r (r < 8) or Lbar_{r - 8}
    for (int rc = tid; rc < 128; rc += kTableThreads) {
        const int r = rc >> 3, c = rc & 7;
        const int i = r < 8 ? sL[r] : sLb[r - 8];
        sOff[rc] = (c < K && i >= 0) ? (int)((long long)dev::pair_index(i, sL[c]) * a.ld) : -1;
    }
    __syncthreads();
    // stage sources [s0, s0 + sc) (lanes over sources, so factor columns read coalesced; the
    // smem stride kZS is odd) by the warps [w_first, kTableWarps), eight loads in flight
    auto stage = [&](int s0, int sc, int w_first) {
        const int nw = kTableWarps - w_first, s = s0 + lane;
        for (int rc0 = warp - w_first; rc0 < 128; rc0 += 8 * nw) {
            double v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int rc = rc0 + j * nw;
                v[j] = 0.0;
                if (rc < 128 && lane < sc) {
                    const int o = sOff[rc];
                    if (o >= 0) {
                        const int i = (rc >> 3) < 8 ? sL[rc >> 3] : sLb[(rc >> 3) - 8];
                        v[j] = s == 0 ? __ldg(a.h + i * n + sL[rc & 7]) : __ldg(a.lf + o + (s - 1));
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int rc = rc0 + j * nw;
                if (rc < 128 && lane < sc)
                    sZ[lane * kZS + ((rc & 7) >> 2) * 64 + (rc >> 3) * 4 + (rc & 3)] = v[j];
            }
        }
    };
    // S_LL^-1 by Gauss-Jordan on [S_LL | I] (S_LL is a principal block of an SPD matrix: the
    // diagonal pivots are positive), warp 0 over the augmented entries, while the other warps
    // stage the first sources
    if (warp != 0) stage(0, min(SC, R + 1), 1);
    if (warp == 0) {
        for (int e = lane; e < K * 2 * K; e += 32) {
            const int r = e / (2 * K), c = e % (2 * K);
            sM[r][c] = c < K ? __ldg(a.S + sL[r] * n + sL[c]) : (c - K == r ? 1.0 : 0.0);
        }
        double det = 1.0;
        __syncwarp();
        for (int st = 0; st < K; ++st) {
            const double piv = sM[st][st];
            det *= piv;
            const double inv = 1.0 / piv;
            if (lane < K) sF[lane] = sM[lane][st];
            __syncwarp();
            for (int c = lane; c < 2 * K; c += 32) sM[st][c] *= inv;
            __syncwarp();
            for (int e = lane; e < K * 2 * K; e += 32) {
                const int r = e / (2 * K), c = e % (2 * K);
                if (r != st) sM[r][c] = fma(-sF[r], sM[st][c], sM[r][c]);
            }
            __syncwarp();
        }
        for (int e = lane; e < K * K; e += 32) sSinv[(e / K) * 8 + e % K] = sM[e / K][K + e % K];
        if (lane == 0) sDet = det;
    }
    __syncthreads();
    // P = S[Lbar, L] Sinv, the squared row norms of S[:, L], certificate scalars
    for (int e = tid; e < NBM * K; e += kTableThreads) {
        const int b = e / K, c = e % K;
        double acc = 0.0;
        if (b < nb)
#pragma unroll
            for (int t = 0; t < K; ++t) acc = fma(__ldg(a.S + sLb[b] * n + sL[t]), sSinv[t * 8 + c], acc);
        sP[b * 8 + c] = acc;
        blk[F.o_p + e] = acc;
    }
    for (int e = tid; e < K + NBM; e += kTableThreads) {
        double acc = 0.0;
        if (e < K || e - K < nb) {
            const int o = e < K ? sL[e] : sLb[e - K];
#pragma unroll
            for (int c = 0; c < K; ++c) {
                const double v = __ldg(a.S + o * n + sL[c]);
                acc = fma(v, v, acc);
            }
        }
        blk[F.o_rowsq + e] = acc;
    }
    if (tid == kTableThreads - 1) {
        double s2 = 0.0, x2 = 0.0;
        for (int e = 0; e < 64; ++e) s2 = fma(sSinv[e], sSinv[e], s2);
        for (int c = 0; c < K; ++c)
            for (int t = 0; t < K; ++t) {
                const double v = __ldg(a.S + sL[c] * n + sL[t]);
                x2 = fma(v, v, x2);
            }
        blk[F.o_scal + 0] = sDet;
        blk[F.o_scal + 1] = s2;
        blk[F.o_scal + 2] = x2;
    }
    __syncthreads();
    if (tid < NBM) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < K; ++c) acc = fma(sP[tid * 8 + c], sP[tid * 8 + c], acc);
        blk[F.o_prow2 + tid] = acc;
    }
    // per-lane fragments that do not change with the source: Sinv as B (k x n), -P as A (m x k)
    double sinv_b[2], negp_a[2];
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
        sinv_b[ks] = sSinv[(4 * ks + gc) * 8 + gr];
        negp_a[ks] = -sP[gr * 8 + 4 * ks + gc];
    }
    double lin[2] = {0.0, 0.0}, e2 = 0.0;
    double mq[MT_W][2];
#pragma unroll
    for (int t = 0; t < MT_W; ++t) mq[t][0] = mq[t][1] = 0.0;
    double* yl = sYL + warp * 64;
    double* va = sVA + warp * 64;
    for (int s0 = 0; s0 < R + 1; s0 += SC) {
        const int sc = min(SC, R + 1 - s0);
        if (s0 > 0) {
            stage(s0, sc, 0);
            __syncthreads();
        }
        for (int sl = warp; sl < sc; sl += kTableWarps) {
            const int s = s0 + sl;
            const double* z = sZ + (size_t)sl * kZS;
            // Y' = [L; Lbar] rows of Z_s times Sinv: tile 0 = YL, tile 1 = YB
            double y0[2] = {0.0, 0.0}, y1[2] = {0.0, 0.0};
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                mma_f64(y0, z[ks * 64 + lane], sinv_b[ks]);
                mma_f64(y1, z[ks * 64 + 32 + lane], sinv_b[ks]);
            }
            // YL(r, c) at (r / 4) * 32 + c * 4 + r % 4
#pragma unroll
            for (int h = 0; h < 2; ++h) yl[(gr >> 2) * 32 + (2 * gc + h) * 4 + (gr & 3)] = y0[h];
            __syncwarp();
            // Vt = YB - P YL (accumulator started at YB)
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) mma_f64(y1, negp_a[ks], yl[ks * 32 + lane]);
            // Vt to the source's column of sX and, as an A operand, to va
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = 2 * gc + h;
                sX[(gr * 8 + c) * kXS + sl] = y1[h];
                va[(c >> 2) * 32 + gr * 4 + (c & 3)] = y1[h];
            }
            // traces of YL and YL^2
            double tr = 0.0, tr2 = 0.0;
            if (lane < K) {
                auto YL = [&](int r, int c) { return yl[(r >> 2) * 32 + c * 4 + (r & 3)]; };
                tr = YL(lane, lane);
#pragma unroll
                for (int t = 0; t < K; ++t) tr2 = fma(YL(lane, t), YL(t, lane), tr2);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                tr += __shfl_xor_sync(0xffffffffu, tr, o);
                tr2 += __shfl_xor_sync(0xffffffffu, tr2, o);
            }
            // table row of this source: Vt on the (hole position c, complement b) grid, trace
            double* row = blk + (long long)(s == 0 ? 0 : s + 1) * KFS;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int b = gr, c = 2 * gc + h;
                if (c < K && b < nb) row[c * 8 + b] = y1[h];
            }
            if (lane == 0) row[8 * K] = tr;
            // with at most 7 complement orbitals, column 7 of every hole block is free: the trace
            // there lets a pair with holes pick it up in its first hole block (no trace k-step)
            if (nb <= 7 && lane < K) row[lane * 8 + 7] = tr;
            __syncwarp();
            if (s > 0) {
                const double sg = (s - 1) < a.r_pos ? 1.0 : -1.0;
                // V T Sinv = Vt YL
                double vts[2] = {0.0, 0.0};
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) mma_f64(vts, va[ks * 32 + lane], yl[ks * 32 + lane]);
                lin[0] = fma(sg, fma(tr, y1[0], -vts[0]), lin[0]);
                lin[1] = fma(sg, fma(tr, y1[1], -vts[1]), lin[1]);
                e2 = fma(sg, tr * tr - tr2, e2);
            }
            __syncwarp();
        }
        __syncthreads();
        // M += sum_s sigma_s x_s x_s^T over this pass's sources, four per k-step
        for (int k0 = 0; k0 < sc; k0 += 4) {
            const int sl = k0 + gc, s = s0 + sl;
            const bool ok = sl < sc && s > 0;
            const double sg = ok ? ((s - 1) < a.r_pos ? 1.0 : -1.0) : 0.0;
            const double* x = sX + (ok ? sl : 0);
#pragma unroll
            for (int t = 0; t < MT_W; ++t) {
                const int tile = warp + kTableWarps * t;
                if (tile >= MT) break;
                int ti = 0, rem = tile;
                while (rem >= 8 - ti) {
                    rem -= 8 - ti;
                    ++ti;
                }
                const int tj = ti + rem;
                mma_f64(mq[t], sg * x[(ti * 8 + gr) * kXS], ok ? x[(tj * 8 + gr) * kXS] : 0.0);
            }
        }
    }
    // combine the warps' partial linear tables, the constant, and M
    sLin[warp * 64 + gr * 8 + 2 * gc] = lin[0];
    sLin[warp * 64 + gr * 8 + 2 * gc + 1] = lin[1];
    if (lane == 0) sE2[warp] = e2;
    double* sMq = sZ;  // 64 x 64
    __syncthreads();
#pragma unroll
    for (int t = 0; t < MT_W; ++t) {
        const int tile = warp + kTableWarps * t;
        if (tile >= MT) break;
        int ti = 0, rem = tile;
        while (rem >= 8 - ti) {
            rem -= 8 - ti;
            ++ti;
        }
        const int tj = ti + rem;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = ti * 8 + gr, c = tj * 8 + 2 * gc + h;
            sMq[r * 64 + c] = mq[t][h];
            if (ti != tj) sMq[c * 64 + r] = mq[t][h];
        }
    }
    __syncthreads();
    for (int e = tid; e < 64; e += kTableThreads) {
        const int b = e >> 3, c = e & 7;
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < kTableWarps; ++w) x += sLin[w * 64 + e];
        if (c < K && b < nb) blk[1 * KFS + c * 8 + b] = x;
    }
    if (tid == 0) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < kTableWarps; ++w) x += sE2[w];
        blk[1 * KFS + 8 * K] = 0.5 * x;
        if (nb <= 7)
            for (int c = 0; c < K; ++c) blk[1 * KFS + c * 8 + 7] = 0.5 * x;
    }
    for (int e = tid; e < NQ; e += kTableThreads) {
        constexpr int CPD = CP > 0 ? CP : 1;
        const int bp = e / CPD, cp = e % CPD;
        int b2 = 1;
        while ((b2 + 1) * b2 / 2 <= bp) ++b2;
        const int b1 = bp - b2 * (b2 - 1) / 2;
        int c2 = 1;
        while ((c2 + 1) * c2 / 2 <= cp) ++c2;
        const int c1 = cp - c2 * (c2 - 1) / 2;
        blk[F.o_q + e] = sMq[(b1 * 8 + c1) * 64 + b2 * 8 + c2] - sMq[(b1 * 8 + c2) * 64 + b2 * 8 + c1];
    }
}

template <int K>
size_t frame_tables_smem(int n, int R) {
    (void)n;
    const size_t sc = (size_t)table_sources(R);
    return sizeof(double) * ((sc * kZS > 4096 ? sc * kZS : 4096) + 64 * kXS + 3 * (size_t)kTableWarps * 64);
}

// Phase A of one pair at excitation level E (compile time).  Writes the pair's Y' row and
// returns the certificate, det X, the quadratic two-electron term / det X and the hole mask.
// COMPACT: W is stored in canonical order (hole slot j, particle slot i) at yrow[j E + i] and the
// slot maps are returned (*hmap: nibble c = hole slot of position c, *pmap: nibble b = particle
// slot of complement index b, 0xF elsewhere); otherwise W is scattered on the pair's dense row
// (zeroed beforehand) with 1 in the trace slot.
template <int K, int E, bool COMPACT>
__device__ __forceinline__ void frame_pair(const double* __restrict__ blk, const FrameLayout& F, unsigned desc,
                                           double* __restrict__ yrow, bool* ok_out, double* det_out,
                                           double* quad_out, unsigned* hm_out, unsigned* hmap_out,
                                           unsigned* pmap_out) {
    constexpr int CP = fr_cp(K);
    const unsigned hm = desc & 0xFFu;
    // holes (positions in L, ascending) and particles (Lbar indices, ascending)
    int hc[E > 0 ? E : 1], pb[E > 0 ? E : 1];
    {
        unsigned h = hm, pm = (desc >> 8) & 0xFFu;
#pragma unroll
        for (int j = 0; j < E; ++j) {
            hc[j] = __ffs(h) - 1;
            h &= h - 1;
            pb[j] = __ffs(pm) - 1;
            pm &= pm - 1;
        }
    }
    const double* P = blk + F.o_p;
    double x[E > 0 ? E : 1][E > 0 ? E : 1];
#pragma unroll
    for (int i = 0; i < E; ++i)
#pragma unroll
        for (int j = 0; j < E; ++j) x[i][j] = P[pb[i] * K + hc[j]];
    int lab[E > 0 ? E : 1];
#pragma unroll
    for (int i = 0; i < E; ++i) lab[i] = i;
    double detb = 1.0;
#pragma unroll
    for (int s = 0; s < E; ++s) {
        int p = s;
        double best = fabs(x[s][s]);
#pragma unroll
        for (int i = s + 1; i < E; ++i) {
            const double av = fabs(x[i][s]);
            if (av > best) {
                best = av;
                p = i;
            }
        }
#pragma unroll
        for (int i = s + 1; i < E; ++i) {
            const bool sw = (p == i);
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const double a0 = x[s][j], a1 = x[i][j];
                x[s][j] = sw ? a1 : a0;
                x[i][j] = sw ? a0 : a1;
            }
            const int l0 = lab[s], l1 = lab[i];
            lab[s] = sw ? l1 : l0;
            lab[i] = sw ? l0 : l1;
        }
        if (p != s) detb = -detb;
        const double piv = x[s][s];
        detb *= piv;
        const double ip = 1.0 / piv;
        x[s][s] = 1.0;
#pragma unroll
        for (int j = 0; j < E; ++j) x[s][j] *= ip;
#pragma unroll
        for (int i = 0; i < E; ++i) {
            if (i == s) continue;
            const double f = x[i][s];
            x[i][s] = 0.0;
#pragma unroll
            for (int j = 0; j < E; ++j) x[i][j] = fma(-f, x[s][j], x[i][j]);
        }
    }
    // x[j][jj] = W(j, lab[jj]): hole slot j, particle slot lab[jj]
    const double* scal = blk + F.o_scal;
    const double det = ((desc >> 16) & 1u ? -1.0 : 1.0) * scal[0] * detb;
    double nw2 = 0.0;
#pragma unroll
    for (int i = 0; i < E; ++i)
#pragma unroll
        for (int j = 0; j < E; ++j) nw2 = fma(x[i][j], x[i][j], nw2);
    const double* rowsq = blk + F.o_rowsq;
    const double* prow2 = blk + F.o_prow2;
    double nx2 = scal[2], pr = 0.0;
#pragma unroll
    for (int j = 0; j < E; ++j) {
        nx2 += rowsq[K + pb[j]] - rowsq[hc[j]];
        pr += prow2[pb[j]];
    }
    const double bnd = scal[1] * ((double)(K - E) + nw2 * (1.0 + pr));
    const bool ok = isfinite(det) && det != 0.0 && (nx2 * bnd < kCertificate2);
    // packed particle Lbar indices by slot, to read the particle of a permuted column
    uint64_t bword = 0;
#pragma unroll
    for (int i = 0; i < E; ++i) bword |= (uint64_t)pb[i] << (8 * i);
    int bj[E > 0 ? E : 1];
#pragma unroll
    for (int jj = 0; jj < E; ++jj) bj[jj] = (int)((bword >> (8 * lab[jj])) & 0xFFu);
    double quad = 0.0;
    if (E >= 2) {
        const double* Q = blk + F.o_q;
#pragma unroll
        for (int j1 = 0; j1 < E; ++j1)
#pragma unroll
            for (int j2 = j1 + 1; j2 < E; ++j2) {
                const int cp = hc[j2] * (hc[j2] - 1) / 2 + hc[j1];
                double part = 0.0;
#pragma unroll
                for (int jj1 = 0; jj1 < E; ++jj1)
#pragma unroll
                    for (int jj2 = jj1 + 1; jj2 < E; ++jj2) {
                        const int ba = bj[jj1], bb = bj[jj2];
                        const bool ordered = ba < bb;
                        const int lo = ordered ? ba : bb, hi = ordered ? bb : ba;
                        const double m2 = fma(x[j1][jj1], x[j2][jj2], -x[j1][jj2] * x[j2][jj1]);
                        const double qv = Q[(hi * (hi - 1) / 2 + lo) * CP + cp];
                        part = fma(ordered ? qv : -qv, m2, part);
                    }
                quad += part;
            }
    }
    unsigned hmap = 0xFFFFFFFFu, pmap = 0xFFFFFFFFu;
    if (COMPACT) {
        if (ok) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                hmap &= ~(0xFu << (4 * hc[j]));
                hmap |= (unsigned)j << (4 * hc[j]);
                pmap &= ~(0xFu << (4 * pb[j]));
                pmap |= (unsigned)j << (4 * pb[j]);
#pragma unroll
                for (int jj = 0; jj < E; ++jj) yrow[j * E + lab[jj]] = x[j][jj];
            }
        }
    } else if (ok) {
        // the pair's row (zeroed by the warp beforehand): W on the (hole position, particle)
        // grid, 1 in the trace slot
#pragma unroll
        for (int j = 0; j < E; ++j)
#pragma unroll
            for (int jj = 0; jj < E; ++jj) yrow[hc[j] * 8 + bj[jj]] = x[j][jj];
        yrow[8 * K] = 1.0;
    }
    *hmap_out = hmap;
    *pmap_out = pmap;
    *ok_out = ok;
    *det_out = det;
    *quad_out = quad;
    *hm_out = hm;
}

// Compact slots: W of an E <= 5 pair (25 doubles; stride 26 spreads a tile's pairs over banks).
// Higher levels use fewer pairs per chunk with E^2 + 1 doubles per slot in the same 32 x 26
// doubles of the warp: 16 pairs for E = 6, 7, 8 pairs for E = 8.
constexpr int kCompactEMax = 5;
constexpr int kCompactSlot = 26;

__host__ __device__ constexpr int compact_chunk_pairs(int e) { return e <= kCompactEMax ? 32 : (e <= 7 ? 16 : 8); }
__host__ __device__ constexpr int compact_slot(int e) { return e <= kCompactEMax ? kCompactSlot : e * e + 1; }

// The high excitation levels (E > kCompactEMax, about 1.5 % of the pairs at K = 7) out of line:
// their E x E registers do not count against the register budget of the common levels.
struct PairOut {
    double det, quad;
    unsigned hm, hmap, pmap;
    bool ok;
};

template <int K, int E>
__device__ __noinline__ PairOut frame_pair_out_of_line(const double* __restrict__ blk, const FrameLayout* F,
                                                       unsigned desc, double* __restrict__ yrow) {
    PairOut o;
    frame_pair<K, E, true>(blk, *F, desc, yrow, &o.ok, &o.det, &o.quad, &o.hm, &o.hmap, &o.pmap);
    return o;
}

template <int K, int ELO, int EHI, bool COMPACT>
__device__ __forceinline__ void frame_pair_dispatch(int e, const double* blk, const FrameLayout& F, unsigned desc,
                                                    double* yrow, bool* ok, double* det, double* quad, unsigned* hm,
                                                    unsigned* hmap, unsigned* pmap) {
#define VB_FRAME_CASE(E_)                                                                             \
    case E_:                                                                                          \
        if constexpr (E_ >= ELO && E_ <= EHI && E_ <= K) {                                            \
            if constexpr (COMPACT && E_ > kCompactEMax) {                                             \
                const PairOut o = frame_pair_out_of_line<K, E_>(blk, &F, desc, yrow);                 \
                *ok = o.ok;                                                                           \
                *det = o.det;                                                                         \
                *quad = o.quad;                                                                       \
                *hm = o.hm;                                                                           \
                *hmap = o.hmap;                                                                       \
                *pmap = o.pmap;                                                                       \
            } else {                                                                                  \
                frame_pair<K, E_, COMPACT>(blk, F, desc, yrow, ok, det, quad, hm, hmap, pmap);         \
            }                                                                                         \
        }                                                                                             \
        break;
    switch (e) {
        VB_FRAME_CASE(0)
        VB_FRAME_CASE(1)
        VB_FRAME_CASE(2)
        VB_FRAME_CASE(3)
        VB_FRAME_CASE(4)
        VB_FRAME_CASE(5)
        VB_FRAME_CASE(6)
        VB_FRAME_CASE(7)
        VB_FRAME_CASE(8)
        default: break;
    }
#undef VB_FRAME_CASE
}


__host__ __device__ constexpr int frame_row_doubles(int K, bool compact) { return compact ? kCompactSlot : fr_kfs(K); }

// The pairs of excitation levels ELO .. EHI of every left string.  COMPACT (EHI <= 4): each pair's
// W is kept as an E x E slot and the tensor-core A fragments are read through the pair's slot
// maps (a few registers and 4.3 KB of shared memory per warp); otherwise each pair has a dense row
// on the (hole position x particle) grid.  Task counter: a.task_counter (+2 for the dense kernel).
template <int K, int ELO, int EHI, bool COMPACT>
__global__ void __launch_bounds__(32 * kFrameMaxWarps, COMPACT ? 2 : 1)
    spin_pairs_frame(SpinTableArgs a, const double* __restrict__ tables) {
    extern __shared__ double smem[];
    constexpr int KFS = fr_kfs(K);
    constexpr int ROW = frame_row_doubles(K, COMPACT);
    const int R = a.R;
    const FrameLayout F = frame_layout(a.n, K, R);
    const int NT = F.rows / 8;
    double* sBlk = smem;
    double* sY = smem + F.total;
    __shared__ int s_task, s_chunk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    const long long N = a.n_strings;
    double* yw = sY + (size_t)warp * 32 * ROW;
    unsigned long long* task_counter = a.task_counter + (COMPACT ? 0 : 2);
    for (;;) {
        if (threadIdx.x == 0) {
            s_task = (int)atomicAdd(task_counter, 1ull);
            s_chunk = 0;
        }
        __syncthreads();
        const int u = s_task;
        if (u >= N) break;
        const int* eb = a.ebound + (long long)u * (K + 2);
        int bound[K + 2];
#pragma unroll
        for (int e = 0; e < K + 2; ++e) bound[e] = __ldg(eb + e);
        int nchunks = 0;
#pragma unroll
        for (int e = ELO; e <= EHI && e <= K; ++e) {
            const int cs = COMPACT ? compact_chunk_pairs(e) : 32;
            nchunks += (bound[e + 1] - bound[e] + cs - 1) / cs;
        }
        if (nchunks == 0) {
            __syncthreads();
            continue;
        }
        {
            const double2* src = reinterpret_cast<const double2*>(tables + (long long)u * F.total);
            double2* dst = reinterpret_cast<double2*>(sBlk);
            for (int i = threadIdx.x; i < F.total / 2; i += blockDim.x) dst[i] = __ldg(src + i);
        }
        const long long base = record_index(u, u, N);
        __syncthreads();
        // warps take 32-pair chunks dynamically, highest excitation level (the costliest) first;
        // the next chunk is claimed and its right strings and descriptors are loaded while the
        // current one is evaluated
        auto claim = [&](int* e_out, int* cnt_out, int* v_out, unsigned* d_out) {
            int ch = 0;
            if (lane == 0) ch = atomicAdd(&s_chunk, 1);
            ch = __shfl_sync(0xffffffffu, ch, 0);
            int e = -1, start = 0, cnt = 0, left = ch;
#pragma unroll
            for (int ee = (EHI < K ? EHI : K); ee >= ELO; --ee) {
                const int cs = COMPACT ? compact_chunk_pairs(ee) : 32;
                const int c = (bound[ee + 1] - bound[ee] + cs - 1) / cs;
                if (left >= 0 && left < c) {
                    e = ee;
                    start = bound[ee] + cs * left;
                    cnt = min(cs, bound[ee + 1] - start);
                }
                left -= c;
            }
            const bool valid = e >= 0 && lane < cnt;
            *v_out = valid ? __ldg(a.rlist + base + start + lane) : u;
            *d_out = valid ? __ldg(a.rdesc + base + start + lane) : 0u;
            *e_out = e;
            *cnt_out = cnt;
        };
        int e_next, cnt_next, v_next;
        unsigned d_next;
        claim(&e_next, &cnt_next, &v_next, &d_next);
        for (;;) {
            const int e = e_next, cnt = cnt_next, v = v_next;
            const unsigned desc = d_next;
            if (e < 0) break;
            claim(&e_next, &cnt_next, &v_next, &d_next);
            const bool valid = lane < cnt;
            if (!COMPACT) {
                // zero the warp's 32 rows, consecutive lanes on consecutive 16-byte words
                double2* z = reinterpret_cast<double2*>(yw);
#pragma unroll
                for (int f = lane; f < 16 * KFS; f += 32) z[f] = make_double2(0.0, 0.0);
                __syncwarp();
            }
            const int slot = COMPACT ? compact_slot(e) : ROW;
            double* yrow = yw + lane * slot;
            bool ok = false;
            double det = 0.0, quad = 0.0;
            unsigned hm = 0, hmap = 0xFFFFFFFFu, pmap = 0xFFFFFFFFu;
            if (valid) {
                frame_pair_dispatch<K, ELO, EHI, COMPACT>(e, sBlk, F, desc, yrow, &ok, &det, &quad, &hm, &hmap,
                                                          &pmap);
                if (!ok) {
                    const unsigned long long slot = atomicAdd(a.careful_count, 1ull);
                    a.careful_list[slot] = ((unsigned long long)u << 32) | (unsigned long long)v;
                }
            }
            const long long t = record_index(u, v, N);
            const unsigned okbits = __ballot_sync(0xffffffffu, ok);
            __syncwarp();
            // phase B, one 8-pair tile at a time
            const int tiles = COMPACT ? compact_chunk_pairs(e) / 8 : 4;
#pragma unroll 1
            for (int mt = 0; mt < tiles; ++mt) {
                const unsigned uh = __reduce_or_sync(0xffffffffu, ((lane >> 3) == mt && ok) ? hm : 0u);
                if (((okbits >> (8 * mt)) & 0xFFu) == 0) continue;
                const int owner = 8 * mt + g;
                const double det_g = __shfl_sync(0xffffffffu, det, owner);
                const double quad_g = __shfl_sync(0xffffffffu, quad, owner);
                const long long t_g = __shfl_sync(0xffffffffu, t, owner);
                const unsigned hmap_g = __shfl_sync(0xffffffffu, hmap, owner);
                const unsigned pmap_g = __shfl_sync(0xffffffffu, pmap, owner);
                const bool ok_g = (okbits >> owner) & 1u;
                const double* yr = yw + owner * slot;
                double* rec = a.records + t_g * (long long)a.rec_stride;
                // this lane's particle slots for the two k-steps of a hole block (b = tq, tq + 4)
                const unsigned i0 = (pmap_g >> (4 * tq)) & 0xFu, i1 = (pmap_g >> (4 * (tq + 4))) & 0xFu;
                // the trace from column 7 of each pair's first hole block (compact, level >= 1,
                // at most 7 complement orbitals) instead of a separate k-step
                const bool pad_trace = COMPACT && e >= 1 && a.n - K <= 7;
#pragma unroll 1
                for (int nt0 = 0; nt0 < NT; nt0 += 6) {
                    double acc[6][2];
#pragma unroll
                    for (int j = 0; j < 6; ++j) acc[j][0] = acc[j][1] = 0.0;
                    if (!pad_trace) {
                        const double af = COMPACT ? ((tq == 0 && ok_g) ? 1.0 : 0.0) : yr[8 * K + tq];
#pragma unroll
                        for (int j = 0; j < 6; ++j) {
                            const double bf = (nt0 + j < NT) ? sBlk[(8 * (nt0 + j) + g) * KFS + 8 * K + tq] : 0.0;
                            mma_f64(acc[j], af, bf);
                        }
                    }
                    unsigned rest = uh;
                    while (rest) {
                        const int c = __ffs(rest) - 1;
                        rest &= rest - 1;
                        const unsigned jh = (hmap_g >> (4 * c)) & 0xFu;
#pragma unroll
                        for (int ks = 0; ks < 2; ++ks) {
                            const int col = 8 * c + 4 * ks + tq;
                            double af;
                            if (COMPACT) {
                                const unsigned ip = ks ? i1 : i0;
                                af = (jh < (unsigned)e && ip < (unsigned)e) ? yr[jh * e + ip] : 0.0;
                                if (pad_trace && ks == 1 && tq == 3) af = jh == 0 ? 1.0 : 0.0;
                            } else {
                                af = yr[col];
                            }
#pragma unroll
                            for (int j = 0; j < 6; ++j) {
                                const double bf = (nt0 + j < NT) ? sBlk[(8 * (nt0 + j) + g) * KFS + col] : 0.0;
                                mma_f64(acc[j], af, bf);
                            }
                        }
                    }
                    if (ok_g) {
#pragma unroll
                        for (int j = 0; j < 6; ++j)
#pragma unroll
                            for (int i = 0; i < 2; ++i) {
                                const int row = 8 * (nt0 + j) + 2 * tq + i;
                                if (row >= 2 && row < R + 2) rec[row - 2] = det_g * acc[j][i];
                            }
                        if (nt0 == 0 && tq == 0) {
                            const double h1 = acc[0][0], e2 = acc[0][1];
                            rec[R + 0] = det_g;
                            rec[R + 1] = det_g * (h1 + e2 + quad_g);
                            rec[R + 2] = det_g * h1;
                            rec[R + 3] = 0.0;
                        }
                    }
                }
            }
            __syncwarp();
        }
        __syncthreads();
    }
}

template <int K>
size_t frame_spin_smem(int n, int R, int warps = 4, bool compact = false) {
    return sizeof(double) * ((size_t)frame_layout(n, K, R).total + (size_t)warps * 32 * frame_row_doubles(K, compact));
}

// Shared memory of the largest launch variant (8 warps per CTA).
template <int K>
size_t frame_spin_smem_max(int n, int R) {
    return frame_spin_smem<K>(n, R, 8, true);
}

size_t frame_spin_smem_rt(int n, int k, int R) {
    switch (k) {
        case 1: return frame_spin_smem_max<1>(n, R);
        case 2: return frame_spin_smem_max<2>(n, R);
        case 3: return frame_spin_smem_max<3>(n, R);
        case 4: return frame_spin_smem_max<4>(n, R);
        case 5: return frame_spin_smem_max<5>(n, R);
        case 6: return frame_spin_smem_max<6>(n, R);
        case 7: return frame_spin_smem_max<7>(n, R);
        case 8: return frame_spin_smem_max<8>(n, R);
        default: return ~size_t{0};
    }
}

template <int K>
cudaError_t launch_tables(const SpinTableArgs& a, double* tables, cudaStream_t stream) {
    const size_t tsmem = frame_tables_smem<K>(a.n, a.R);
    cudaError_t err = allow_dynamic_smem((const void*)frame_tables<K>, tsmem);
    if (err != cudaSuccess) return err;
    frame_tables<K><<<a.n_strings, kTableThreads, tsmem, stream>>>(a, tables);
    return cudaGetLastError();
}

// Launch variants of the pair kernel (the autotuner's choices): 0 = 8 warps per CTA, 1 = 4,
// 2 = 2; every variant fills each SM with as many resident CTAs as fit.
constexpr int kFrameVariants = 3;
constexpr int kFrameVariantWarps[kFrameVariants] = {8, 4, 2};

template <int K, int ELO, int EHI, bool COMPACT>
cudaError_t launch_frame_part(const SpinTableArgs& a, const double* tables, cudaStream_t stream, int warps) {
    const size_t smem = frame_spin_smem<K>(a.n, a.R, warps, COMPACT);
    auto kernel = spin_pairs_frame<K, ELO, EHI, COMPACT>;
    cudaError_t err = allow_dynamic_smem((const void*)kernel, smem);
    if (err != cudaSuccess) return err;
    int per_sm = 1, dev = 0, sms = 148;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * warps, smem);
    if (err != cudaSuccess) return err;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long blocks = (long long)sms * (per_sm > 0 ? per_sm : 1);
    if (blocks > a.n_strings) blocks = a.n_strings;
    if (blocks < 1) blocks = 1;
    kernel<<<(unsigned)blocks, 32 * warps, smem, stream>>>(a, tables);
    return cudaGetLastError();
}

template <int K>
cudaError_t launch_frame(const SpinTableArgs& a, const double* tables, cudaStream_t stream, int variant) {
    return launch_frame_part<K, 0, K, true>(a, tables, stream, kFrameVariantWarps[variant]);
}

template <int K>
cudaError_t launch_sort(int N, const uint64_t* occ, int* rlist, unsigned* rdesc, int* ebound, cudaStream_t stream) {
    sort_right_strings<K><<<(N + kFrameWarps - 1) / kFrameWarps, kFrameThreads, 0, stream>>>(N, occ, rlist, rdesc,
                                                                                            ebound);
    return cudaGetLastError();
}

}  // namespace

size_t frame_table_doubles(int n, int k, int R) { return (size_t)frame_layout(n, k, R).total; }

bool frame_spin_supported(int n, int k, int R) {
    return k >= 1 && k <= 8 && n - k >= 0 && n - k <= fr_nbmax(k) && frame_spin_smem_rt(n, k, R) <= 200 * 1024;
}

cudaError_t launch_sort_right_strings(int k, int N, const uint64_t* occ, int* rlist, unsigned* rdesc, int* ebound,
                                      cudaStream_t stream) {
    if (N <= 0) return cudaSuccess;
    switch (k) {
        case 1: return launch_sort<1>(N, occ, rlist, rdesc, ebound, stream);
        case 2: return launch_sort<2>(N, occ, rlist, rdesc, ebound, stream);
        case 3: return launch_sort<3>(N, occ, rlist, rdesc, ebound, stream);
        case 4: return launch_sort<4>(N, occ, rlist, rdesc, ebound, stream);
        case 5: return launch_sort<5>(N, occ, rlist, rdesc, ebound, stream);
        case 6: return launch_sort<6>(N, occ, rlist, rdesc, ebound, stream);
        case 7: return launch_sort<7>(N, occ, rlist, rdesc, ebound, stream);
        case 8: return launch_sort<8>(N, occ, rlist, rdesc, ebound, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_frame_tables(const SpinTableArgs& a, double* tables, cudaStream_t stream) {
    switch (a.k) {
        case 1: return launch_tables<1>(a, tables, stream);
        case 2: return launch_tables<2>(a, tables, stream);
        case 3: return launch_tables<3>(a, tables, stream);
        case 4: return launch_tables<4>(a, tables, stream);
        case 5: return launch_tables<5>(a, tables, stream);
        case 6: return launch_tables<6>(a, tables, stream);
        case 7: return launch_tables<7>(a, tables, stream);
        case 8: return launch_tables<8>(a, tables, stream);
        default: return cudaErrorInvalidValue;
    }
}

int frame_pair_variants(int n, int k, int R) {
    (void)n;
    (void)k;
    (void)R;
    return kFrameVariants;
}

cudaError_t launch_frame_pairs(const SpinTableArgs& a, const double* tables, cudaStream_t stream, int variant) {
    if (variant < 0 || variant >= kFrameVariants) variant = 0;
    switch (a.k) {
        case 1: return launch_frame<1>(a, tables, stream, variant);
        case 2: return launch_frame<2>(a, tables, stream, variant);
        case 3: return launch_frame<3>(a, tables, stream, variant);
        case 4: return launch_frame<4>(a, tables, stream, variant);
        case 5: return launch_frame<5>(a, tables, stream, variant);
        case 6: return launch_frame<6>(a, tables, stream, variant);
        case 7: return launch_frame<7>(a, tables, stream, variant);
        case 8: return launch_frame<8>(a, tables, stream, variant);
        default: return cudaErrorInvalidValue;
    }
}

template <int K>
cudaError_t preload_k() {
    cudaFuncAttributes fa{};
    cudaError_t err = cudaFuncGetAttributes(&fa, (const void*)sort_right_strings<K>);
    if (err == cudaSuccess) err = cudaFuncGetAttributes(&fa, (const void*)frame_tables<K>);
    if (err == cudaSuccess) err = cudaFuncGetAttributes(&fa, (const void*)spin_pairs_frame<K, 0, K, true>);
    return err;
}

cudaError_t preload_frame_kernels() {
    cudaError_t err = preload_k<1>();
    if (err == cudaSuccess) err = preload_k<2>();
    if (err == cudaSuccess) err = preload_k<3>();
    if (err == cudaSuccess) err = preload_k<4>();
    if (err == cudaSuccess) err = preload_k<5>();
    if (err == cudaSuccess) err = preload_k<6>();
    if (err == cudaSuccess) err = preload_k<7>();
    if (err == cudaSuccess) err = preload_k<8>();
    return err;
}

}  // namespace vbcore
