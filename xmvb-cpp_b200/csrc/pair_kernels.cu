// Determinant-pair kernels for sm_100a.
//
//  * prepare_tables: the unpacked pair kernel K[p][q] = (p|q) over packed orbital pairs and the
//    antisymmetrized same-spin table Gamma[(i<k)][(j<l)] = (ij|kl) - (il|kj) used by the
//    same-spin two-electron sum (hamiltonian.cpp:83-123 sums exactly these differences).
//  * spin_pairs_fast<K>: one thread per unordered spin-string pair, K x K overlap block in
//    registers, Gauss-Jordan inversion with partial pivoting (row interchanges tracked as a
//    label permutation, no dynamic register indexing), determinant, first cofactors
//    A = det X^{-T}, one-electron and same-spin two-electron energies from shared-memory
//    tables.  A block is accepted only when ||X||_F ||X^{-1}||_F < 1e9: then every pivot of a
//    complete-pivoting LU exceeds sigma_min / k >= 1e-12 * (growth bound) * max pivot for
//    k <= 16, i.e. the reference's FullPivLU would also find full rank
//    (overlap.cpp:60-71).  Every other block is appended to a list for the exact kernel.
//  * spin_pairs_exact: complete-pivoting LU / Jacobi SVD with the reference semantics
//    (device_algebra.cuh) for listed blocks.
//  * full_pairs<KB>: one thread per determinant pair (d <= e) of a band of columns:
//    S = S_a S_b, H = H_a S_b + H_b S_a + sum A_a(r,c) A_b(r',c') (r c | r' c')
//    (evaluator.cpp:95-148, 354-384), the opposite-spin sum as k_a^2 k_b^2 gathers of the
//    shared-memory pair kernel against the beta cofactors held in registers.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "device_algebra.cuh"
#include "kernels.h"

namespace vbcore {
namespace {

constexpr double kThreshold = 1.0e-12;
constexpr double kCertificate2 = 1.0e18;  // (1e9)^2 on ||X||_F^2 ||X^-1||_F^2
constexpr int kSms = 148;

__device__ __forceinline__ int occ_byte(const uint64_t* row, int i) {
    const uint64_t w = row[i >> 3];
    return (int)((w >> (8 * (i & 7))) & 0xFFu);
}

__device__ __forceinline__ void decode_upper(long long t, long long* u, long long* v) {
    long long vv = (long long)floor((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (vv * (vv + 1) / 2 > t) --vv;
    while ((vv + 1) * (vv + 2) / 2 <= t) ++vv;
    *v = vv;
    *u = t - vv * (vv + 1) / 2;
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

template <int K>
__global__ void __launch_bounds__(128) spin_pairs_fast(SpinTableArgs a) {
    extern __shared__ double smem[];
    const int n = a.n;
    const int gd = a.gamma_dim;
    double* sS = smem;
    double* sh = smem + n * n;
    double* sG = smem + 2 * n * n;
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
        sS[i] = a.S[i];
        sh[i] = a.h[i];
    }
    if (K >= 2)
        for (int i = threadIdx.x; i < gd * gd; i += blockDim.x) sG[i] = a.gamma[i];
    __syncthreads();

    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < a.n_pairs; t += stride) {
        long long u, v;
        decode_upper(t, &u, &v);
        const uint64_t wl = __ldg(a.occ + 2 * u);
        const uint64_t wr = __ldg(a.occ + 2 * v);
        int L[K], R[K];
#pragma unroll
        for (int c = 0; c < K; ++c) {
            L[c] = (int)((wl >> (8 * c)) & 0xFFu);
            R[c] = (int)((wr >> (8 * c)) & 0xFFu);
        }
        double x[K][K];
        double nx2 = 0.0;
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
            for (int c = 0; c < K; ++c) {
                x[r][c] = sS[R[r] * n + L[c]];
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
        double det = 1.0;
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
        const bool accepted = isfinite(det) && det != 0.0 && (nx2 * ni2 < kCertificate2);
        if (!accepted) {
            const unsigned long long slot = atomicAdd(a.careful_count, 1ull);
            a.careful_list[slot] = t;
            continue;
        }
        double* rec = a.records + t * (long long)a.rec_stride;
        double h1 = 0.0, h2 = 0.0;
        if (K <= 3) {
            // closed-form cofactors and second cofactors (contractions.cpp:187-205, 915-923)
            double cof[K0][K0];
#pragma unroll
            for (int i = 0; i < K0; ++i)
#pragma unroll
                for (int j = 0; j < K0; ++j) {
                    double value = 1.0;
                    if (K == 2) {
                        value = x0[1 - i][1 - j];
                    } else if (K == 3) {
                        const int rr = i == 0 ? 1 : 0, ss = i == 2 ? 1 : 2;
                        const int cc = j == 0 ? 1 : 0, dd = j == 2 ? 1 : 2;
                        const double product = x0[rr][dd] * x0[ss][cc];
                        value = fma(x0[rr][cc], x0[ss][dd], -product) - fma(x0[rr][dd], x0[ss][cc], -product);
                    }
                    cof[i][j] = ((i + j) & 1) ? -value : value;
                    h1 = fma(sh[R[i] * n + L[j]], cof[i][j], h1);
                    rec[i * K + j] = cof[i][j];
                }
            if (K == 2) {
                h2 = sG[dev::anti_index(R[0], R[1]) * gd + dev::anti_index(L[0], L[1])];
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
                                const double c2nd = sign * x0[3 - r1 - r2][3 - c1 - c2];
                                h2 = fma(sG[dev::anti_index(R[r1], R[r2]) * gd + dev::anti_index(L[c1], L[c2])], c2nd,
                                         h2);
                            }
            }
        } else {
            // x now holds C = (P X)^{-1}; X^{-1}[c][lab[j]] = C[c][j], A(lab[j], c) = det C[c][j].
            int Rp[K];
#pragma unroll
            for (int j = 0; j < K; ++j) Rp[j] = (int)((wr >> (8 * lab[j])) & 0xFFu);
            double acc1 = 0.0;
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int c = 0; c < K; ++c) acc1 = fma(sh[Rp[j] * n + L[c]], x[c][j], acc1);
            h1 = det * acc1;
            int cidx[K][K];
#pragma unroll
            for (int c1 = 0; c1 < K; ++c1)
#pragma unroll
                for (int c2 = c1 + 1; c2 < K; ++c2) cidx[c1][c2] = dev::anti_index(L[c1], L[c2]);
            double acc2 = 0.0;
#pragma unroll
            for (int j1 = 0; j1 < K; ++j1)
#pragma unroll
                for (int j2 = j1 + 1; j2 < K; ++j2) {
                    const int ra = Rp[j1], rb = Rp[j2];
                    const bool ordered = ra < rb;
                    const double* grow = sG + dev::anti_index(ordered ? ra : rb, ordered ? rb : ra) * gd;
                    double part = 0.0;
#pragma unroll
                    for (int c1 = 0; c1 < K; ++c1)
#pragma unroll
                        for (int c2 = c1 + 1; c2 < K; ++c2) {
                            const double m2 = fma(x[c1][j1], x[c2][j2], -x[c2][j1] * x[c1][j2]);
                            part = fma(grow[cidx[c1][c2]], m2, part);
                        }
                    acc2 += ordered ? part : -part;
                }
            h2 = det * acc2;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                double* row = rec + lab[j] * K;
#pragma unroll
                for (int c = 0; c < K; ++c) row[c] = det * x[c][j];
            }
        }
        rec[K * K + 0] = det;
        rec[K * K + 1] = h1 + h2;
        rec[K * K + 2] = h1;
        rec[K * K + 3] = 0.0;
    }
}

__global__ void __launch_bounds__(64) spin_pairs_exact(SpinTableArgs a) {
    const long long count = a.all_careful ? a.n_pairs : (long long)(*a.careful_count);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int k = a.k;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < count; idx += stride) {
        const long long t = a.all_careful ? idx : a.careful_list[idx];
        long long u, v;
        decode_upper(t, &u, &v);
        int L[dev::KMAX], R[dev::KMAX];
        for (int c = 0; c < k; ++c) {
            L[c] = occ_byte(a.occ + 2 * u, c);
            R[c] = occ_byte(a.occ + 2 * v, c);
        }
        double x[dev::KMAX * dev::KMAX];
        for (int c = 0; c < k; ++c)
            for (int r = 0; r < k; ++r) x[c * k + r] = __ldg(a.S + R[r] * a.n + L[c]);
        dev::Resolution res;
        dev::resolve_exact(k, x, kThreshold, &res);
        double cof[dev::KMAX * dev::KMAX];
        dev::first_cofactor(res, cof);
        double h1 = 0.0, htot = 0.0;
        if (res.nullity < 3) htot = dev::same_spin_exact(a.n, k, L, R, res, cof, a.h, a.eri, &h1);
        double* rec = a.records + t * (long long)a.rec_stride;
        for (int r = 0; r < k; ++r)
            for (int c = 0; c < k; ++c) rec[r * k + c] = res.nullity <= 1 ? cof[c * k + r] : 0.0;
        rec[k * k + 0] = res.det;
        rec[k * k + 1] = htot;
        rec[k * k + 2] = h1;
        rec[k * k + 3] = (double)res.nullity;
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

__device__ __forceinline__ long long upper_record(int a, int b) {
    const long long hi = a > b ? a : b, lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

template <int KB>
__global__ void __launch_bounds__(128) full_pairs_kernel(FullPairArgs a) {
    extern __shared__ double sK[];
    const int np = a.np;
    if (a.kfull_in_smem) {
        for (int i = threadIdx.x; i < np * np; i += blockDim.x) sK[i] = a.kfull[i];
        __syncthreads();
    }
    const double* K = a.kfull_in_smem ? sK : a.kfull;
    const long long B = a.e1 - a.e0;
    const int ka = a.ka;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < a.n_items; t += stride) {
        long long d, e;
        band_decode(t, a.e0, a.e1, &d, &e);
        const int ia = __ldg(a.det_alpha + d), ja = __ldg(a.det_alpha + e);
        const int ib = __ldg(a.det_beta + d), jb = __ldg(a.det_beta + e);
        const int la = min(ia, ja), ha = max(ia, ja), lb = min(ib, jb), hb = max(ib, jb);
        const double* ra = a.rec_a + upper_record(la, ha) * a.stride_a;
        const double* rb = a.rec_b + upper_record(lb, hb) * a.stride_b;
        const double sa = ra[ka * ka], hsa = ra[ka * ka + 1], nua = ra[ka * ka + 3];
        const double sb = rb[KB * KB], hsb = rb[KB * KB + 1], nub = rb[KB * KB + 3];
        double H = fma(hsa, sb, hsb * sa);
        const double S = sa * sb;
        if (nua < 1.5 && nub < 1.5) {
            const uint64_t wbl = __ldg(a.occ_b + 2 * lb), wbr = __ldg(a.occ_b + 2 * hb);
            double Ab[KB * KB];
            int qb[KB * KB];
#pragma unroll
            for (int r = 0; r < KB; ++r)
#pragma unroll
                for (int c = 0; c < KB; ++c) {
                    Ab[r * KB + c] = rb[r * KB + c];
                    qb[r * KB + c] = dev::pair_index((int)((wbr >> (8 * r)) & 0xFFu), (int)((wbl >> (8 * c)) & 0xFFu));
                }
            const uint64_t* occl = a.occ_a + 2 * la;
            const uint64_t* occr = a.occ_a + 2 * ha;
            double opp = 0.0;
            for (int r = 0; r < ka; ++r) {
                const int Ra = occ_byte(occr, r);
                for (int c = 0; c < ka; ++c) {
                    const double av = ra[r * ka + c];
                    const double* krow = K + dev::pair_index(Ra, occ_byte(occl, c)) * np;
                    double tt = 0.0;
#pragma unroll
                    for (int i = 0; i < KB * KB; ++i) tt = fma(Ab[i], krow[qb[i]], tt);
                    opp = fma(av, tt, opp);
                }
            }
            H += opp;
        }
        const long long o = d * B + (e - a.e0);
        a.Hb[o] = H;
        a.Sb[o] = S;
    }
}

// Generic variant: any k_a, k_b <= 16 (either may be zero); both cofactor blocks streamed.
__global__ void __launch_bounds__(128) full_pairs_generic(FullPairArgs a) {
    extern __shared__ double sK[];
    const int np = a.np;
    if (a.kfull_in_smem) {
        for (int i = threadIdx.x; i < np * np; i += blockDim.x) sK[i] = a.kfull[i];
        __syncthreads();
    }
    const double* K = a.kfull_in_smem ? sK : a.kfull;
    const long long B = a.e1 - a.e0;
    const int ka = a.ka, kb = a.kb;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < a.n_items; t += stride) {
        long long d, e;
        band_decode(t, a.e0, a.e1, &d, &e);
        double sa = 1.0, hsa = 0.0, nua = 0.0, sb = 1.0, hsb = 0.0, nub = 0.0;
        const double* ra = nullptr;
        const double* rb = nullptr;
        int la = 0, ha = 0, lb = 0, hb = 0;
        if (ka > 0) {
            const int ia = __ldg(a.det_alpha + d), ja = __ldg(a.det_alpha + e);
            la = min(ia, ja);
            ha = max(ia, ja);
            ra = a.rec_a + upper_record(la, ha) * a.stride_a;
            sa = ra[ka * ka];
            hsa = ra[ka * ka + 1];
            nua = ra[ka * ka + 3];
        }
        if (kb > 0) {
            const int ib = __ldg(a.det_beta + d), jb = __ldg(a.det_beta + e);
            lb = min(ib, jb);
            hb = max(ib, jb);
            rb = a.rec_b + upper_record(lb, hb) * a.stride_b;
            sb = rb[kb * kb];
            hsb = rb[kb * kb + 1];
            nub = rb[kb * kb + 3];
        }
        double H = fma(hsa, sb, hsb * sa);
        const double S = sa * sb;
        if (ka > 0 && kb > 0 && nua < 1.5 && nub < 1.5) {
            double opp = 0.0;
            for (int r = 0; r < ka; ++r) {
                const int Ra = occ_byte(a.occ_a + 2 * ha, r);
                for (int c = 0; c < ka; ++c) {
                    const double av = ra[r * ka + c];
                    const double* krow = K + dev::pair_index(Ra, occ_byte(a.occ_a + 2 * la, c)) * np;
                    double tt = 0.0;
                    for (int r2 = 0; r2 < kb; ++r2) {
                        const int Rb = occ_byte(a.occ_b + 2 * hb, r2);
                        for (int c2 = 0; c2 < kb; ++c2)
                            tt = fma(rb[r2 * kb + c2], krow[dev::pair_index(Rb, occ_byte(a.occ_b + 2 * lb, c2))], tt);
                    }
                    opp = fma(av, tt, opp);
                }
            }
            H += opp;
        }
        const long long o = d * B + (e - a.e0);
        a.Hb[o] = H;
        a.Sb[o] = S;
    }
}

// Listed determinant pairs (d, e) in any order, full orientation handled through records.
__global__ void listed_pairs_kernel(FullPairArgs a, long long n_pairs, const long long* __restrict__ pairs,
                                    double* __restrict__ h_out, double* __restrict__ s_out) {
    const int np = a.np;
    const double* K = a.kfull;
    const int ka = a.ka, kb = a.kb;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n_pairs;
         t += (long long)gridDim.x * blockDim.x) {
        const long long d = pairs[2 * t], e = pairs[2 * t + 1];
        double sa = 1.0, hsa = 0.0, nua = 0.0, sb = 1.0, hsb = 0.0, nub = 0.0;
        const double* ra = nullptr;
        const double* rb = nullptr;
        int la = 0, ha = 0, lb = 0, hb = 0;
        if (ka > 0) {
            const int ia = a.det_alpha[d], ja = a.det_alpha[e];
            la = min(ia, ja);
            ha = max(ia, ja);
            ra = a.rec_a + upper_record(la, ha) * a.stride_a;
            sa = ra[ka * ka];
            hsa = ra[ka * ka + 1];
            nua = ra[ka * ka + 3];
        }
        if (kb > 0) {
            const int ib = a.det_beta[d], jb = a.det_beta[e];
            lb = min(ib, jb);
            hb = max(ib, jb);
            rb = a.rec_b + upper_record(lb, hb) * a.stride_b;
            sb = rb[kb * kb];
            hsb = rb[kb * kb + 1];
            nub = rb[kb * kb + 3];
        }
        double H = fma(hsa, sb, hsb * sa);
        if (ka > 0 && kb > 0 && nua < 1.5 && nub < 1.5) {
            double opp = 0.0;
            for (int r = 0; r < ka; ++r)
                for (int c = 0; c < ka; ++c) {
                    const double* krow =
                        K + dev::pair_index(occ_byte(a.occ_a + 2 * ha, r), occ_byte(a.occ_a + 2 * la, c)) * np;
                    double tt = 0.0;
                    for (int r2 = 0; r2 < kb; ++r2)
                        for (int c2 = 0; c2 < kb; ++c2)
                            tt = fma(rb[r2 * kb + c2],
                                     krow[dev::pair_index(occ_byte(a.occ_b + 2 * hb, r2), occ_byte(a.occ_b + 2 * lb, c2))],
                                     tt);
                    opp = fma(ra[r * ka + c], tt, opp);
                }
            H += opp;
        }
        h_out[t] = H;
        s_out[t] = sa * sb;
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
cudaError_t launch_fast(const SpinTableArgs& a, cudaStream_t stream) {
    const size_t smem = sizeof(double) * (2 * (size_t)a.n * a.n + (K >= 2 ? (size_t)a.gamma_dim * a.gamma_dim : 0));
    cudaError_t err = cudaFuncSetAttribute(spin_pairs_fast<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    long long blocks = (a.n_pairs + 127) / 128;
    if (blocks > kSms * 16) blocks = kSms * 16;
    if (blocks < 1) blocks = 1;
    spin_pairs_fast<K><<<(unsigned)blocks, 128, smem, stream>>>(a);
    return cudaGetLastError();
}

template <int KB>
cudaError_t launch_full(const FullPairArgs& a, size_t smem, cudaStream_t stream) {
    cudaError_t err = cudaFuncSetAttribute(full_pairs_kernel<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    long long blocks = (a.n_items + 127) / 128;
    if (blocks > kSms * 32) blocks = kSms * 32;
    if (blocks < 1) blocks = 1;
    full_pairs_kernel<KB><<<(unsigned)blocks, 128, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace

size_t fast_spin_smem_bytes(int n, int k) {
    const size_t gd = (size_t)n * (n - 1) / 2;
    return sizeof(double) * (2 * (size_t)n * n + (k >= 2 ? gd * gd : 0));
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

cudaError_t launch_spin_pairs(const SpinTableArgs& a, cudaStream_t stream, int* launches) {
    if (a.n_pairs <= 0 || a.k <= 0) return cudaSuccess;
    cudaError_t err = cudaSuccess;
    const bool fast_ok = !a.all_careful && a.k <= 8 && fast_spin_smem_bytes(a.n, a.k) <= 227 * 1024;
    if (fast_ok) {
        switch (a.k) {
            case 1: err = launch_fast<1>(a, stream); break;
            case 2: err = launch_fast<2>(a, stream); break;
            case 3: err = launch_fast<3>(a, stream); break;
            case 4: err = launch_fast<4>(a, stream); break;
            case 5: err = launch_fast<5>(a, stream); break;
            case 6: err = launch_fast<6>(a, stream); break;
            case 7: err = launch_fast<7>(a, stream); break;
            case 8: err = launch_fast<8>(a, stream); break;
            default: break;
        }
        if (err != cudaSuccess) return err;
        ++*launches;
    }
    SpinTableArgs b = a;
    b.all_careful = fast_ok ? 0 : 1;
    spin_pairs_exact<<<kSms * 8, 64, 0, stream>>>(b);
    ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_full_pairs(const FullPairArgs& a0, cudaStream_t stream, int* launches) {
    if (a0.n_items <= 0) return cudaSuccess;
    FullPairArgs a = a0;
    const size_t ksmem = sizeof(double) * (size_t)a.np * a.np;
    a.kfull_in_smem = ksmem <= 200 * 1024 ? 1 : 0;
    const size_t smem = a.kfull_in_smem ? ksmem : 0;
    cudaError_t err;
    ++*launches;
    if (a.ka > 0 && a.kb >= 1 && a.kb <= 8 && a.ka <= 16) {
        switch (a.kb) {
            case 1: return launch_full<1>(a, smem, stream);
            case 2: return launch_full<2>(a, smem, stream);
            case 3: return launch_full<3>(a, smem, stream);
            case 4: return launch_full<4>(a, smem, stream);
            case 5: return launch_full<5>(a, smem, stream);
            case 6: return launch_full<6>(a, smem, stream);
            case 7: return launch_full<7>(a, smem, stream);
            case 8: return launch_full<8>(a, smem, stream);
            default: break;
        }
    }
    err = cudaFuncSetAttribute(full_pairs_generic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    long long blocks = (a.n_items + 127) / 128;
    if (blocks > kSms * 32) blocks = kSms * 32;
    full_pairs_generic<<<(unsigned)blocks, 128, smem, stream>>>(a);
    return cudaGetLastError();
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
