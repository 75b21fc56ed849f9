// Determinant-pair kernels for sm_100a.
//
//  * prepare_tables: the unpacked pair kernel K[p][q] = (p|q) over packed orbital pairs and the
//    antisymmetrized same-spin table Gamma[(i<k)][(j<l)] = (ij|kl) - (il|kj) used by the
//    same-spin two-electron sum (hamiltonian.cpp:83-123 sums exactly these differences).
//  * factor_pair_kernel: pivoted LDL^T of the pair kernel, K = sum_m sigma_m l_m l_m^T.
//  * the register-resident spin-pair path lives in spin_frame.cu (left-string frame kernels); a
//    block is accepted there only under the conditioning certificate (kCertificate2): then the
//    last pivot of a complete-pivoting LU is at least 1 / ||X^{-1}||_F and the first at most
//    ||X||_F, so their ratio stays far above 1e-12 and the reference's FullPivLU would also find
//    full rank (overlap.cpp:60-71).  Every other block is appended to a list for the exact kernel.
//  * spin_pairs_exact<KM>: complete-pivoting LU / Jacobi SVD with the reference semantics
//    (device_algebra.cuh) for listed blocks, one thread per block, local arrays bounded by KM.
//  * full_pairs_kernel: one thread per determinant pair (d <= e) of a band of columns:
//    S = S_a S_b, H = H_a S_b + H_b S_a + sum_m sigma_m u_a[m] u_b[m] (evaluator.cpp:95-148,
//    354-384 with the opposite-spin term in factored form), folded over the spin-flip orbit.
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
// Relative pivot cut of the pair-kernel factorization.  Once the numerical rank is exhausted the
// Schur complement holds rounding noise of about (steps) * eps * max|K_pp|, so a cut of 8 np eps
// (at least 1e-15) ends the factorization there instead of emitting columns of noise.
double factor_tolerance(int np) { return fmax(1.0e-15, 8.0 * np * 2.220446049250313e-16); }
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

// Pivoted LDL^T of the unpacked pair kernel with diagonal (complete) pivoting, one CTA, in the
// left-looking form.  Thread t owns rows t, t + nt, ... (at most kFactorRows) and keeps their
// diagonal in registers.  Step m: with the pivot p and its value known, every owned row forms its
// entry of the Schur-complement column, K[i, p] - sum_{m' < m} sigma_m' l_m'[p] l_m'[i], scales it
// into l_m[i] and updates its diagonal; each warp then reduces its rows' largest |diagonal| and
// one barrier publishes the warp results, from which every thread picks the next pivot.
// Stops when the largest remaining |diagonal| falls to rel_tol times the largest initial one;
// the dropped remainder then perturbs any opposite-spin energy by at most
// rel_tol * max|K_pp| * ||p_a||_1 ||p_b||_1.  Columns are emitted positive-sign first.
// K and the columns l_m (l_m[i] at [m np + i]) sit in shared memory when they fit (in_smem),
// else K is read from `kfull` and the columns live in `cols`.  `work_g` is not used.
constexpr int kFactorRows = 4;

template <bool in_smem>  // compile-time, so that the shared-memory path uses shared loads
__global__ void __launch_bounds__(1024) factor_pair_kernel(int np, const double* __restrict__ kfull,
                                                           double* __restrict__ work_g, double* __restrict__ cols,
                                                           int* __restrict__ signs, double* __restrict__ lf, int ld,
                                                           int* __restrict__ meta, double rel_tol) {
    (void)work_g;
    extern __shared__ double fsm[];
    double* sig = fsm;                                        // np
    int* slot_col = reinterpret_cast<int*>(sig + np);         // np (+1 pad)
    double* Ks = sig + np + (np + 2) / 2;                     // np^2 when in_smem
    const double* K = in_smem ? Ks : kfull;
    double* L = in_smem ? Ks + (size_t)np * np : cols;
    __shared__ double red_v[2][32], red_d[2][32];
    __shared__ int red_i[2][32];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    if (in_smem)
        for (long long i = tid; i < (long long)np * np; i += nt) Ks[i] = __ldg(kfull + i);
    double dg[kFactorRows];
    bool used[kFactorRows];
#pragma unroll
    for (int r = 0; r < kFactorRows; ++r) {
        const int i = tid + r * nt;
        dg[r] = i < np ? __ldg(kfull + (long long)i * np + i) : 0.0;
        used[r] = i >= np;
    }
    // publishes this thread's best unused row to the warp slots of buffer b (largest |diagonal|,
    // smallest index on ties)
    auto publish = [&](int b) {
        double best = -1.0, bd = 0.0;
        int bi = -1;
#pragma unroll
        for (int r = 0; r < kFactorRows; ++r)
            if (!used[r] && fabs(dg[r]) > best) {
                best = fabs(dg[r]);
                bd = dg[r];
                bi = tid + r * nt;
            }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const double od = __shfl_xor_sync(0xffffffffu, bd, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi >= 0 && (bi < 0 || oi < bi))) {
                best = ov;
                bd = od;
                bi = oi;
            }
        }
        if (lane == 0) {
            red_v[b][warp] = best;
            red_d[b][warp] = bd;
            red_i[b][warp] = bi;
        }
    };
    auto pick = [&](int b, int* p, double* piv) {
        double best = -1.0, bd = 0.0;
        int bi = -1;
        for (int w = 0; w < nwarps; ++w) {
            const double ov = red_v[b][w];
            const int oi = red_i[b][w];
            if (ov > best || (ov == best && oi >= 0 && (bi < 0 || oi < bi))) {
                best = ov;
                bd = red_d[b][w];
                bi = oi;
            }
        }
        *p = bi;
        *piv = bd;
    };
    publish(0);
    __syncthreads();
    int p;
    double piv;
    pick(0, &p, &piv);
    const double cut = rel_tol * fmax(fabs(piv), 0.0);
    int m = 0;
    for (; m < np; ++m) {
        if (p < 0 || !(fabs(piv) > cut) || piv == 0.0) break;
        const double inv = rsqrt(fabs(piv));
        const double sgn = piv > 0.0 ? 1.0 : -1.0;
        double* lm = L + (long long)m * np;
#pragma unroll
        for (int r = 0; r < kFactorRows; ++r) {
            const int i = tid + r * nt;
            if (i >= np) continue;
            double v = 0.0;
            if (!used[r]) {
                double acc0 = K[(long long)p * np + i], acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
                int q = 0;
                for (; q + 3 < m; q += 4) {
                    const double* l0 = L + (long long)q * np;
                    acc0 = fma(-sig[q] * l0[p], l0[i], acc0);
                    acc1 = fma(-sig[q + 1] * l0[np + p], l0[np + i], acc1);
                    acc2 = fma(-sig[q + 2] * l0[2 * np + p], l0[2 * np + i], acc2);
                    acc3 = fma(-sig[q + 3] * l0[3 * np + p], l0[3 * np + i], acc3);
                }
                for (; q < m; ++q) acc0 = fma(-sig[q] * L[(long long)q * np + p], L[(long long)q * np + i], acc0);
                v = ((acc0 + acc1) + (acc2 + acc3)) * inv;
                if (i == p)
                    used[r] = true;
                else
                    dg[r] = fma(-sgn * v, v, dg[r]);
            }
            lm[i] = v;
        }
        if (tid == 0) {
            sig[m] = sgn;
            signs[m] = (int)sgn;
        }
        publish((m + 1) & 1);
        __syncthreads();
        pick((m + 1) & 1, &p, &piv);
    }
    if (tid == 0) {
        int pos = 0;
        for (int c = 0; c < m; ++c) pos += sig[c] > 0.0 ? 1 : 0;
        int ip = 0, in = pos;
        for (int c = 0; c < m; ++c) slot_col[sig[c] > 0.0 ? ip++ : in++] = c;
        meta[0] = pos;
        meta[1] = m - pos;
    }
    __syncthreads();
    for (int q = warp; q < np; q += nwarps)
        for (int slot = lane; slot < ld; slot += 32)
            lf[(long long)q * ld + slot] = slot < m ? L[(long long)slot_col[slot] * np + q] : 0.0;
}

// The same factorization for np <= 32 (active spaces of up to 7 orbitals) in one warp: lane i
// owns row i, the pivot search is a shuffle reduction and the steps need no block barrier.
__global__ void __launch_bounds__(32) factor_pair_warp_kernel(int np, const double* __restrict__ kfull,
                                                             int* __restrict__ signs, double* __restrict__ lf,
                                                             int ld, int* __restrict__ meta, double rel_tol) {
    __shared__ double sL[32][33];  // column m of the factor in sL[m][.]
    __shared__ double sig[32];
    __shared__ int slot_col[32];
    const int lane = threadIdx.x;
    double dg = lane < np ? __ldg(kfull + (long long)lane * np + lane) : 0.0;
    bool used = lane >= np;
    auto argmax = [&](int* p, double* piv) {
        double best = used ? -1.0 : fabs(dg), bd = dg;
        int bi = used ? -1 : lane;
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const double od = __shfl_xor_sync(0xffffffffu, bd, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi >= 0 && (bi < 0 || oi < bi))) {
                best = ov;
                bd = od;
                bi = oi;
            }
        }
        *p = bi;
        *piv = bd;
    };
    int p;
    double piv;
    argmax(&p, &piv);
    const double cut = rel_tol * fmax(fabs(piv), 0.0);
    int m = 0;
    for (; m < np; ++m) {
        if (p < 0 || !(fabs(piv) > cut) || piv == 0.0) break;
        const double inv = rsqrt(fabs(piv));
        const double sgn = piv > 0.0 ? 1.0 : -1.0;
        double v = 0.0;
        if (!used) {
            double acc = __ldg(kfull + (long long)p * np + lane);
            for (int q = 0; q < m; ++q) acc = fma(-sig[q] * sL[q][p], sL[q][lane], acc);
            v = acc * inv;
            if (lane == p)
                used = true;
            else
                dg = fma(-sgn * v, v, dg);
        }
        sL[m][lane] = v;
        if (lane == 0) {
            sig[m] = sgn;
            signs[m] = (int)sgn;
        }
        __syncwarp();
        argmax(&p, &piv);
    }
    if (lane == 0) {
        int pos = 0;
        for (int c = 0; c < m; ++c) pos += sig[c] > 0.0 ? 1 : 0;
        int ip = 0, in = pos;
        for (int c = 0; c < m; ++c) slot_col[sig[c] > 0.0 ? ip++ : in++] = c;
        meta[0] = pos;
        meta[1] = m - pos;
    }
    __syncwarp();
    for (int q = 0; q < np; ++q)
        for (int slot = lane; slot < ld; slot += 32)
            lf[(long long)q * ld + slot] = slot < m ? sL[slot_col[slot]][q] : 0.0;
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
    // blocks per warp: 32 (one per lane) when there are enough, fewer so that a short list
    // spreads over as many warps as it has blocks
    long long chunk = (count + nwarps - 1) / nwarps;
    chunk = chunk < 1 ? 1 : (chunk > 32 ? 32 : chunk);
    for (long long base = warp * chunk; base < count; base += nwarps * chunk) {
        const long long idx = base + lane;
        long long u = 0, v = 0;
        const bool valid = lane < chunk && idx < count;
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
        for (int j = 0; j < chunk; ++j) {
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
                if constexpr (KC > 0) {
                    // k fixed: every lane's terms unrolled, occupations from registers, loads batched
                    constexpr int CPK = KC * (KC - 1) / 2;
                    constexpr int PER = (CPK * CPK + 31) / 32;
                    const uint64_t wl = __ldg(ol), wr = __ldg(orr);
#pragma unroll 2
                    for (int t = 0; t < PER; ++t) {
                        const int q = lane + 32 * t;
                        if (q < CPK * CPK) {
                            const int rp = q / CPK, cq = q % CPK;
                            int r2 = 1;
                            while ((r2 + 1) * r2 / 2 <= rp) ++r2;
                            const int r1 = rp - r2 * (r2 - 1) / 2;
                            int c2 = 1;
                            while ((c2 + 1) * c2 / 2 <= cq) ++c2;
                            const int c1 = cq - c2 * (c2 - 1) / 2;
                            const int R1 = (int)((wr >> (8 * r1)) & 0xFFu), R2 = (int)((wr >> (8 * r2)) & 0xFFu);
                            const int L1 = (int)((wl >> (8 * c1)) & 0xFFu), L2 = (int)((wl >> (8 * c2)) & 0xFFu);
                            const double g = __ldg(a.gamma + (long long)dev::anti_index(R1, R2) * gd + dev::anti_index(L1, L2));
                            part = fma(g, cj[c1 * KC + r1] * cj[c2 * KC + r2] - cj[c2 * KC + r1] * cj[c1 * KC + r2], part);
                        }
                    }
                } else {
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
                }
                for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
                if (lane == j) h2 = part / det;
            }
            // u-vectors: u_m = sum_{c,r} A(r,c) l_m[pair(R_r, L_c)]
            double* rec = a.records + record_index(uj, vj, N) * (long long)a.rec_stride;
            if constexpr (KC > 0) {
                // k fixed: the k^2 factor-row loads of a column issued together
                const uint64_t wl = __ldg(ol), wr = __ldg(orr);
                for (int m = lane; m < a.R; m += 32) {
                    double acc = 0.0;
#pragma unroll 1
                    for (int c = 0; c < KC; ++c) {
                        const int lc = (int)((wl >> (8 * c)) & 0xFFu);
                        double v[KC];
#pragma unroll
                        for (int r = 0; r < KC; ++r)
                            v[r] = __ldg(a.lf + (long long)dev::pair_index((int)((wr >> (8 * r)) & 0xFFu), lc) * a.ld + m);
#pragma unroll
                        for (int r = 0; r < KC; ++r) acc = fma(cj[c * KC + r], v[r], acc);
                    }
                    rec[m] = acc;
                }
            } else {
                for (int m = lane; m < a.R; m += 32) {
                    double acc = 0.0;
                    for (int c = 0; c < k; ++c) {
                        const int lc = occ_byte(ol, c);
                        for (int r = 0; r < k; ++r) {
                            const double cv = cj[c * k + r];
                            if (cv != 0.0)
                                acc = fma(cv, __ldg(a.lf + (long long)dev::pair_index(occ_byte(orr, r), lc) * a.ld + m),
                                          acc);
                        }
                    }
                    rec[m] = acc;
                }
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
        const long long o = d * a.ldb + (e - a.e0);
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

}  // namespace

cudaError_t launch_factor_pair_kernel(int np, const double* kfull, double* work, double* cols, int* signs, double* lf,
                                      int ld, int* meta, cudaStream_t stream) {
    if (np <= 32) {
        factor_pair_warp_kernel<<<1, 32, 0, stream>>>(np, kfull, signs, lf, ld, meta, factor_tolerance(np));
        return cudaGetLastError();
    }
    int threads = (np + 31) / 32 * 32;
    threads = threads < 64 ? 64 : (threads > 1024 ? 1024 : threads);
    if (np > threads * kFactorRows) return cudaErrorInvalidValue;
    const size_t aux_bytes = sizeof(double) * ((size_t)np + (np + 2) / 2);
    const size_t in_smem_bytes = aux_bytes + 2 * sizeof(double) * (size_t)np * np;
    const int in_smem = in_smem_bytes <= 200 * 1024 ? 1 : 0;
    const size_t smem = in_smem ? in_smem_bytes : aux_bytes;
    cudaError_t err = allow_dynamic_smem(in_smem ? (const void*)factor_pair_kernel<true>
                                                 : (const void*)factor_pair_kernel<false>,
                                         (int)smem);
    if (err != cudaSuccess) return err;
    if (in_smem)
        factor_pair_kernel<true><<<1, threads, smem, stream>>>(np, kfull, work, cols, signs, lf, ld, meta,
                                                               factor_tolerance(np));
    else
        factor_pair_kernel<false><<<1, threads, smem, stream>>>(np, kfull, work, cols, signs, lf, ld, meta,
                                                                factor_tolerance(np));
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
    const void* fns[] = {(const void*)prepare_tables_kernel, (const void*)factor_pair_kernel<true>,
                         (const void*)factor_pair_kernel<false>, (const void*)factor_pair_warp_kernel,
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
                // the listed-pair counter and the task counter
                cudaError_t e = cudaMemsetAsync(a.careful_count, 0, sizeof(unsigned long long), stream);
                if (e == cudaSuccess) e = cudaMemsetAsync(a.task_counter, 0, sizeof(unsigned long long), stream);
                return e;
            },
            &err);
        (void)tuned;
        if (err != cudaSuccess) return err;
        ++*launches;
    }
    return cudaSuccess;
}

cudaError_t launch_spin_pairs_exact(const SpinTableArgs& a, cudaStream_t stream, int* launches) {
    if (a.n_pairs <= 0 || a.k <= 0) return cudaSuccess;
    cudaError_t err = cudaSuccess;
    const bool fast_ok = !a.all_careful && frame_spin_supported(a.n, a.k, a.R);
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
