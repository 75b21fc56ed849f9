// Analytic gradient of a structure eigenvalue with respect to the active-space inputs
// (the device counterpart of accumulate_active_space_gradient and its same-spin /
// opposite-spin backward contributions, src/vbscf/derivatives/gradient/active_space/
// evaluator.cpp:1046-1133, src/vbscf/derivatives/hessian/responses/same_spin/backward.cpp,
// .../opposite_spin/backward.cpp).
//
// With c the S-normalized structure eigenvector of eigenvalue lambda, dE = c^T (dH - lambda dS) c
// (the Rayleigh quotient is stationary in c), i.e. with determinant weights w = T c,
//   dE = sum_{d,e} w_d w_e (dH_de - lambda dS_de).
// Reverse mode through the plan's pipeline:
//   1. det_pair_adjoint_kernel: every determinant pair (d <= e) scatters its weight onto the
//      two spin-pair records it was built from (H_de = H_a S_b + H_b S_a + sum_m s_m u_a u_b):
//      adj(det_a) += w (H_b - lambda S_b), adj(H_a) += w S_b, adj(u_a[m]) += w s_m u_b[m], and
//      the same with a <-> b.  With a spin-flip symmetric determinant list the scatter is grouped
//      by alpha record (det_pair_adjoint_flip_kernel, no atomics), and in two stages through a
//      per-alpha-string table in shared memory when alpha strings carry several determinants
//      (det_pair_adjoint_two_stage_kernel).
//   2. spin_backward_kernel<K>: per spin pair, with X = S[R, L], B = X^-1 and d = det X:
//      det = d, A = d B^T, H_1 = <h[R, L], A>, H_2 = d q(B) (q: the same-spin two-electron form
//      in B), u[m] = <l_m[pair(R, L)], A>.  The adjoint with respect to X is
//        d ( s B^T - (B M B)^T ),  s = adj_det + <G_A, B^T> + adj_H q,  M = G_A + adj_H Q^T,
//      G_A = adj_H h[R, L] + sum_m adj_u[m] l_m[pair(R, L)], Q = dq/dB; the linear inputs get
//      adj_H A (h), adj_H d B-minors (the antisymmetrized two-electron table) and
//      adj_u[m] A (factor columns).  Blocks whose conditioning certificate fails are listed.
//   3. careful_backward_kernel: listed blocks (uncertified: ill-conditioned or rank deficient)
//      take the derivative of the exact cofactor polynomial, evaluated in the frame of the
//      block's singular value decomposition (products of singular values only, no inverse;
//      see svd_frame_adjoint).
// The two contractions over the R factor columns (adj_u . l_m at each packed pair, and the
// factor-column adjoint sum_t adj_u (x) A-scatter) run on the FP64 tensor cores (dgemm.cu) over
// chunks of records around the backward kernel, which walks left-string work items like the forward
// kernel and accumulates the two-electron table per left string in shared memory.  The host
// then maps the two-electron table and factor-column adjoints onto the packed integrals
// (full-rank pair kernel) or onto caller-supplied RI factors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "device_algebra.cuh"
#include "internal.h"
#include "kernels.h"
#include "pair_value.cuh"
#include "plan.h"

namespace vbcore {
namespace {


__device__ __forceinline__ int occ_byte(const uint64_t* row, int i) {
    const uint64_t w = row[i >> 3];
    return (int)((w >> (8 * (i & 7))) & 0xFFu);
}

// Row-major upper-triangle index t -> (u, v), u <= v, of an N x N table.
__device__ __forceinline__ void upper_decode(long long t, long long N, long long* u, long long* v) {
    const double b = 2.0 * (double)N + 1.0;
    long long uu = (long long)floor((b - sqrt(fmax(b * b - 8.0 * (double)t, 0.0))) * 0.5);
    if (uu < 0) uu = 0;
    if (uu > N - 1) uu = N - 1;
    while (uu > 0 && uu * N - uu * (uu - 1) / 2 > t) --uu;
    while (uu + 1 < N && (uu + 1) * N - (uu + 1) * uu / 2 <= t) ++uu;
    *u = uu;
    *v = uu + (t - (uu * N - uu * (uu - 1) / 2));
}

__global__ void det_weights_kernel(long long n_det, const int64_t* __restrict__ off, const int* __restrict__ str,
                                   const double* __restrict__ coef, const double* __restrict__ c, double* __restrict__ w) {
    for (long long d = blockIdx.x * (long long)blockDim.x + threadIdx.x; d < n_det; d += (long long)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (long long t = off[d]; t < off[d + 1]; ++t) acc = fma(coef[t], c[str[t]], acc);
        w[d] = acc;
    }
}

struct AdjArgs {
    FullPairArgs f;
    const double* w;
    double lambda;
    double* adj_a;
    double* adj_b;
    int adj_stride;  // R + 2: [u adjoint (R)], adj(det), adj(H)
};

// With shared alpha/beta string tables and a spin-flip symmetric determinant list (the flipped
// determinant carries the same structure terms, so w(flip d) = w(d)), the beta-side scatter of a
// pair {d, e} equals the alpha-side scatter of {flip d, flip e} into the same record, so the
// record adjoint is twice the alpha-side sum.  That sum is grouped by alpha record (i <= j): over
// d in D_i, e in D_j (D_i: determinants with alpha string i), weight 2 w_d w_e for i < j and all
// ordered pairs with weight w_d w_e for i = j.  One warp per record, lanes over the factor
// columns (m = lane + 32 q, q < 4: R <= 128), one write per record, no atomics.
__global__ void __launch_bounds__(256) det_pair_adjoint_flip_kernel(AdjArgs a, const int* __restrict__ aoff,
                                                                    const int* __restrict__ adets) {
    const int R = a.f.R;
    const long long Na = a.f.Na;
    const long long n_rec = Na * (Na + 1) / 2;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < n_rec; t += nwarps) {
        long long i, j;
        upper_decode(t, Na, &i, &j);
        const int i0 = __ldg(aoff + i), i1 = __ldg(aoff + i + 1);
        const int j0 = __ldg(aoff + j), j1 = __ldg(aoff + j + 1);
        const double pair_w = i == j ? 1.0 : 2.0;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        double acc_det = 0.0, acc_h = 0.0;
        // 32 determinants of each side at a time: lanes load their indices, weights and beta
        // strings together, then the warp walks the pairs with shuffled operands, so the record
        // loads of consecutive pairs do not wait on one another
        for (int qc = j0; qc < j1; qc += 32) {
            const int nq = min(32, j1 - qc);
            int be_l = 0;
            double we_l = 0.0;
            if (lane < nq) {
                const int e = __ldg(adets + qc + lane);
                we_l = __ldg(a.w + e);
                be_l = __ldg(a.f.det_beta + e);
            }
            for (int pc = i0; pc < i1; pc += 32) {
                const int np_ = min(32, i1 - pc);
                int bd_l = 0;
                double wd_l = 0.0;
                if (lane < np_) {
                    const int d = __ldg(adets + pc + lane);
                    wd_l = __ldg(a.w + d) * pair_w;
                    bd_l = __ldg(a.f.det_beta + d);
                }
                for (int pp = 0; pp < np_; ++pp) {
                    const double wd = __shfl_sync(0xffffffffu, wd_l, pp);
                    const int bd = __shfl_sync(0xffffffffu, bd_l, pp);
                    if (wd == 0.0) continue;
#pragma unroll 4
                    for (int qq = 0; qq < nq; ++qq) {
                        const double omega = wd * __shfl_sync(0xffffffffu, we_l, qq);
                        const int be = __shfl_sync(0xffffffffu, be_l, qq);
                        if (omega == 0.0) continue;
                        const double* rb =
                            a.f.rec_b + record_index(min(bd, be), max(bd, be), a.f.Nb) * a.f.stride_b;
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int m = lane + 32 * u;
                            if (m < R) acc[u] = fma(omega, m < a.f.r_pos ? __ldg(rb + m) : -__ldg(rb + m), acc[u]);
                        }
                        const double sb = __ldg(rb + R), hb = __ldg(rb + R + 1);
                        acc_det = fma(omega, hb - a.lambda * sb, acc_det);
                        acc_h = fma(omega, sb, acc_h);
                    }
                }
            }
        }
        double* adj = a.adj_a + t * a.adj_stride;
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) {
            const int m = lane + 32 * qq;
            if (m < R) adj[m] += 2.0 * acc[qq];
        }
        if (lane == 0) {
            adj[R] += 2.0 * acc_det;
            adj[R + 1] += 2.0 * acc_h;
        }
    }
}

// Determinant weights and beta strings in alpha-string order (the order of alpha_dets).
__global__ void alpha_order_kernel(long long n_det, const int* __restrict__ adets, const double* __restrict__ w,
                                   const int* __restrict__ det_beta, double* __restrict__ ws, int* __restrict__ bs) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n_det;
         k += (long long)gridDim.x * blockDim.x) {
        const int d = __ldg(adets + k);
        ws[k] = __ldg(w + d);
        bs[k] = __ldg(det_beta + d);
    }
}

// The record adjoint of det_pair_adjoint_flip_kernel in two stages per alpha string i, for plans
// whose alpha strings carry several determinants each (D = n_det / Na of them on average: the
// one-stage form gathers D^2 beta records per alpha record, this one about 2 D):
//   T_i[b][c] = sum_{d in D_i} w_d val_c(rec(beta_d, b))                for every beta string b,
//   adj[(i, j)][c] += 2 pair_w sum_{e in D_j} w_e T_i[beta_e][c]        for every j >= i,
// with val_m = s_m u[m] (m < R), val_R = H - lambda S, val_{R+1} = S.  T_i lives in shared
// memory; one CTA per (alpha string i, chunk of CC record components), every adjoint entry is
// written by one thread and every sum runs in a fixed order.  ws / bs: weights and beta strings in
// alpha_dets order (alpha_order_kernel).
template <int CC>
__global__ void __launch_bounds__(256) det_pair_adjoint_two_stage_kernel(AdjArgs a, const int* __restrict__ aoff,
                                                                         const double* __restrict__ ws,
                                                                         const int* __restrict__ bs) {
    extern __shared__ double sT[];  // Nb x CC
    const int i = blockIdx.x;
    const int c0 = blockIdx.y * CC;
    const int R = a.f.R, r_pos = a.f.r_pos;
    const int ncomp = R + 2;
    const int Nb = a.f.Nb;
    const int i0 = __ldg(aoff + i), i1 = __ldg(aoff + i + 1);
    if (i0 == i1) return;
    // the determinants of alpha string i (weights, beta strings) in shared memory when they fit, so
    // that the record gathers of consecutive determinants do not wait on index loads
    constexpr int kStaged = 512;
    __shared__ double s_w[kStaged];
    __shared__ int s_b[kStaged];
    const bool staged = i1 - i0 <= kStaged;
    if (staged)
        for (int q = threadIdx.x; q < i1 - i0; q += blockDim.x) {
            s_w[q] = __ldg(ws + i0 + q);
            s_b[q] = __ldg(bs + i0 + q);
        }
    __syncthreads();
    for (int t = threadIdx.x; t < Nb * CC; t += blockDim.x) {
        const int b = t / CC, c = c0 + t % CC;
        double acc = 0.0;
        if (c < ncomp) {
            const double sign = c < r_pos ? 1.0 : -1.0;
#pragma unroll 8
            for (int k = i0; k < i1; ++k) {
                const int bd = staged ? s_b[k - i0] : __ldg(bs + k);
                const double* rb = a.f.rec_b + record_index(min(bd, b), max(bd, b), Nb) * a.f.stride_b;
                double v;
                if (c < R)
                    v = sign * __ldg(rb + c);
                else if (c == R)
                    v = __ldg(rb + R + 1) - a.lambda * __ldg(rb + R);
                else
                    v = __ldg(rb + R);
                acc = fma(staged ? s_w[k - i0] : __ldg(ws + k), v, acc);
            }
        }
        sT[t] = acc;
    }
    __syncthreads();
    const long long Na = a.f.Na;
    const long long items = (Na - i) * CC;
    for (long long t = threadIdx.x; t < items; t += blockDim.x) {
        const int j = i + (int)(t / CC), cl = (int)(t % CC), c = c0 + cl;
        if (c >= ncomp) continue;
        const int j0 = __ldg(aoff + j), j1 = __ldg(aoff + j + 1);
        double acc = 0.0;
        for (int k = j0; k < j1; ++k) acc = fma(__ldg(ws + k), sT[__ldg(bs + k) * CC + cl], acc);
        const double pair_w = j == i ? 1.0 : 2.0;
        double* adj = a.adj_a + record_index(i, j, Na) * a.adj_stride;
        adj[c] += 2.0 * pair_w * acc;
    }
}

// Record-component chunk of the two-stage adjoint for Nb beta strings (shared memory Nb x CC
// doubles, at most 100 KB so that two CTAs share an SM), 0 when even 4 components do not fit.
int two_stage_chunk(long long Nb) {
    for (int cc : {16, 8, 4})
        if ((size_t)Nb * cc * sizeof(double) <= 100u * 1024u) return cc;
    return 0;
}

template <int CC>
cudaError_t launch_two_stage(const AdjArgs& a, const int* aoff, const double* ws, const int* bs, cudaStream_t s) {
    const size_t smem = sizeof(double) * (size_t)a.f.Nb * CC;
    cudaError_t err = allow_dynamic_smem((const void*)det_pair_adjoint_two_stage_kernel<CC>, smem);
    if (err != cudaSuccess) return err;
    const dim3 grid((unsigned)a.f.Na, (unsigned)((a.f.R + 2 + CC - 1) / CC));
    det_pair_adjoint_two_stage_kernel<CC><<<grid, 256, smem, s>>>(a, aoff, ws, bs);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256) det_pair_adjoint_kernel(AdjArgs a) {
    const long long n = a.f.n_det;
    const long long total = n * (n + 1) / 2;
    const int R = a.f.R;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        long long d, e;
        upper_decode(t, n, &d, &e);
        const double omega = __ldg(a.w + d) * __ldg(a.w + e) * (d == e ? 1.0 : 2.0);
        if (omega == 0.0) continue;
        double sa = 1.0, ha = 0.0, sb = 1.0, hb = 0.0;
        const double* ra = nullptr;
        const double* rb = nullptr;
        long long ta = -1, tb = -1;
        if (a.f.ka > 0) {
            const int i = __ldg(a.f.det_alpha + d), j = __ldg(a.f.det_alpha + e);
            ta = record_index(min(i, j), max(i, j), a.f.Na);
            ra = a.f.rec_a + ta * a.f.stride_a;
            sa = ra[R];
            ha = ra[R + 1];
        }
        if (a.f.kb > 0) {
            const int i = __ldg(a.f.det_beta + d), j = __ldg(a.f.det_beta + e);
            tb = record_index(min(i, j), max(i, j), a.f.Nb);
            rb = a.f.rec_b + tb * a.f.stride_b;
            sb = rb[R];
            hb = rb[R + 1];
        }
        if (ra) {
            double* adj = a.adj_a + ta * a.adj_stride;
            if (rb)
                for (int m = 0; m < R; ++m) atomicAdd(adj + m, omega * (m < a.f.r_pos ? rb[m] : -rb[m]));
            atomicAdd(adj + R, omega * (hb - a.lambda * sb));
            atomicAdd(adj + R + 1, omega * sb);
        }
        if (rb) {
            double* adj = a.adj_b + tb * a.adj_stride;
            if (ra)
                for (int m = 0; m < R; ++m) atomicAdd(adj + m, omega * (m < a.f.r_pos ? ra[m] : -ra[m]));
            atomicAdd(adj + R, omega * (ha - a.lambda * sa));
            atomicAdd(adj + R + 1, omega * sa);
        }
    }
}

struct BackArgs {
    int n, k, N;
    const uint64_t* occ;
    const double* S;
    const double* h;
    const double* eri;
    const double* gamma;
    int gd;
    const double* lf;
    int ld;
    int R;
    const double* adj;
    int adj_stride;
    double* gS;  // n x n (index as read: S[L_c n + R_r])
    double* gh;  // n x n
    double* gG;  // gd x gd, [anti(L pair) gd + anti(R pair)]
    double* gL;  // [pair q * ld + m]
    unsigned long long* careful_count;
    unsigned long long* careful_list;
    // chunked fast path: items [item_begin, item_end) own records [record_base, ...)
    const int2* items;
    int item_begin, item_end;
    long long record_base;
    const double* Q;  // [record - record_base][np]: adj_u . l_m at each packed pair
    double* Pout;     // [record - record_base][np]: A scattered onto packed pairs (zeroed)
};

template <int K>
__global__ void __launch_bounds__(128) spin_backward_kernel(BackArgs a) {
    // shared accumulators: gS, gh (n x n) and the two-electron table rows of the current left
    // string's orbital pairs (CP x gd); flushed to global memory when the left string changes
    extern __shared__ double acc_s[];
    constexpr int CP = K * (K - 1) / 2;
    const int n = a.n, gd = a.gd, np = a.ld;
    double* sgS = acc_s;
    double* sgh = acc_s + n * n;
    double* sgG = acc_s + 2 * n * n;
    __shared__ int sCp[CP > 0 ? CP : 1];
    for (int i = threadIdx.x; i < 2 * n * n + CP * gd; i += blockDim.x) acc_s[i] = 0.0;
    const long long N = a.N;
    const int per = (a.item_end - a.item_begin + gridDim.x - 1) / gridDim.x;
    const int ib = a.item_begin + blockIdx.x * per;
    const int ie = min(a.item_end, ib + per);
    long long cur_u = -1;
    auto flush_gamma = [&]() {
        __syncthreads();
        if (cur_u >= 0)
            for (int i = threadIdx.x; i < CP * gd; i += blockDim.x) {
                const double v = sgG[i];
                if (v != 0.0) atomicAdd(a.gG + (long long)sCp[i / gd] * gd + (i % gd), v);
                sgG[i] = 0.0;
            }
        __syncthreads();
    };
    for (int item = ib; item < ie; ++item) {
        const int2 it = a.items[item];
        const long long u = it.x;
        int L[K];
        {
            const uint64_t wl = __ldg(a.occ + 2 * u);
#pragma unroll
            for (int c = 0; c < K; ++c) L[c] = (int)((wl >> (8 * c)) & 0xFFu);
        }
        if (u != cur_u) {
            flush_gamma();
            if (threadIdx.x == 0) {
                int q = 0;
#pragma unroll
                for (int c2 = 1; c2 < K; ++c2)
#pragma unroll
                    for (int c1 = 0; c1 < c2; ++c1) sCp[c2 * (c2 - 1) / 2 + c1] = dev::anti_index(L[c1], L[c2]), ++q;
            }
            cur_u = u;
            __syncthreads();
        }
        const long long v = (long long)it.y + threadIdx.x;
        if (v >= N) continue;
        const long long t = record_index(u, v, N);
        const long long tl = t - a.record_base;
        const double* adj = a.adj + t * a.adj_stride;
        const double aS = adj[a.R], aH = adj[a.R + 1];
        int Rr[K];
        {
            const uint64_t wr = __ldg(a.occ + 2 * v);
#pragma unroll
            for (int c = 0; c < K; ++c) Rr[c] = (int)((wr >> (8 * c)) & 0xFFu);
        }
        double x[K][K];
        double nx2 = 0.0;
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
            for (int c = 0; c < K; ++c) {
                x[r][c] = __ldg(a.S + L[c] * n + Rr[r]);
                nx2 = fma(x[r][c], x[r][c], nx2);
            }
        // Gauss-Jordan with partial pivoting: x -> (P X)^-1, lab = row permutation
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
        if (!(isfinite(det) && det != 0.0 && nx2 * ni2 < kCertificate2)) {
            const unsigned long long slot = atomicAdd(a.careful_count, 1ull);
            a.careful_list[slot] = ((unsigned long long)u << 32) | (unsigned long long)v;
            continue;
        }
        // B[c][r] = X^-1[c][r]: X^-1 = C P with C = x, so X^-1[c][lab[j]] = x[c][j]
        double B[K][K];
#pragma unroll
        for (int c = 0; c < K; ++c)
#pragma unroll
            for (int r = 0; r < K; ++r) {
                double val = 0.0;
#pragma unroll
                for (int j = 0; j < K; ++j) val = lab[j] == r ? x[c][j] : val;
                B[c][r] = val;
            }
        // G_A[r][c] = aH h(R_r, L_c) + sum_m adj_u[m] l_m[pair(R_r, L_c)], the sum read from the
        // chunk's Q = adj_U L_f^T (in x, reused as storage)
        const double* qrow = a.Q + tl * np;
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
            for (int c = 0; c < K; ++c) {
                const int q = dev::pair_index(Rr[r], L[c]);
                x[r][c] = fma(aH, __ldg(a.h + L[c] * n + Rr[r]), qrow[q]);
            }
        double gsum = 0.0;
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
            for (int c = 0; c < K; ++c) gsum = fma(x[r][c], B[c][r], gsum);
        // same-spin two-electron form: q(B) and Q = dq/dB (added into M = G_A + aH Q^T)
        double qv = 0.0;
        if (K >= 2) {
#pragma unroll
            for (int c2 = 1; c2 < K; ++c2)
#pragma unroll
                for (int c1 = 0; c1 < c2; ++c1) {
                    const int cpl = c2 * (c2 - 1) / 2 + c1;
                    const double* grow = a.gamma + (long long)dev::anti_index(L[c1], L[c2]) * gd;
#pragma unroll
                    for (int r1 = 0; r1 < K; ++r1)
#pragma unroll
                        for (int r2 = r1 + 1; r2 < K; ++r2) {
                            const int rp = dev::anti_index(Rr[r1], Rr[r2]);
                            const double G = __ldg(grow + rp);
                            const double minor = B[c1][r1] * B[c2][r2] - B[c1][r2] * B[c2][r1];
                            qv = fma(G, minor, qv);
                            const double gA = aH * G;
                            x[r1][c1] = fma(gA, B[c2][r2], x[r1][c1]);
                            x[r2][c2] = fma(gA, B[c1][r1], x[r2][c2]);
                            x[r2][c1] = fma(-gA, B[c2][r1], x[r2][c1]);
                            x[r1][c2] = fma(-gA, B[c1][r2], x[r1][c2]);
                            if (aH != 0.0) atomicAdd(sgG + cpl * gd + rp, aH * det * minor);
                        }
                }
        }
        const double s = aS + gsum + aH * qv;
        double P[K][K];
#pragma unroll
        for (int r = 0; r < K; ++r)
#pragma unroll
            for (int i = 0; i < K; ++i) {
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c < K; ++c) acc = fma(x[r][c], B[c][i], acc);
                P[r][i] = acc;
            }
        double* prow = a.Pout + tl * np;
#pragma unroll
        for (int c = 0; c < K; ++c)
#pragma unroll
            for (int i = 0; i < K; ++i) {
                double bp = 0.0;
#pragma unroll
                for (int r = 0; r < K; ++r) bp = fma(B[c][r], P[r][i], bp);
                // adj_X[i][c] = d (s B[c][i] - (B M B)[c][i]); X[i][c] = S[L_c n + R_i]
                atomicAdd(sgS + L[c] * n + Rr[i], det * (s * B[c][i] - bp));
                const double A = det * B[c][i];
                if (aH != 0.0) atomicAdd(sgh + L[c] * n + Rr[i], aH * A);
                // A scattered onto the packed pairs: the chunk's P row (gL += adj_U^T P after);
                // two (i, c) can share a pair when both orbitals occur in both strings
                prow[dev::pair_index(Rr[i], L[c])] += A;
            }
    }
    flush_gamma();
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
        if (sgS[i] != 0.0) atomicAdd(a.gS + i, sgS[i]);
        if (sgh[i] != 0.0) atomicAdd(a.gh + i, sgh[i]);
    }
}

// Listed (uncertified) pairs [idx_begin, idx_end) of the careful list, or of all pairs.
__device__ __forceinline__ void careful_pair(const BackArgs& a, long long idx, int all_pairs, long long* u,
                                             long long* v) {
    if (all_pairs) {
        upper_decode(idx, a.N, u, v);
    } else {
        const unsigned long long w = a.careful_list[idx];
        *u = (long long)(w >> 32);
        *v = (long long)(w & 0xffffffffull);
    }
}

__global__ void gather_adjoint_kernel(BackArgs a, long long idx_begin, long long idx_end, int all_pairs,
                                      double* __restrict__ Ac) {
    const long long cnt = idx_end - idx_begin;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cnt * a.R;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / a.R;
        const int m = (int)(e % a.R);
        long long u, v;
        careful_pair(a, idx_begin + i, all_pairs, &u, &v);
        Ac[e] = a.adj[record_index(u, v, a.N) * a.adj_stride + m];
    }
}

// Product of the singular values outside the index set `skip` (bit mask).
template <int KM>
__device__ __forceinline__ double sv_product_except(int k, const double* sv, unsigned skip) {
    double p = 1.0;
    for (int l = 0; l < k; ++l)
        if (!((skip >> l) & 1u)) p *= sv[l];
    return p;
}

// Overlap adjoint of the exact cofactor polynomial of one block,
//   f(X) = aS det X + sum_{r,c} Aw[r][c] C_{r,c}(X) + sum_{r1<r2, c1<c2} Gw(r1 r2; c1 c2) C_{r1 r2; c1 c2}(X)
// (C: first- and second-order cofactors), at a block given by its singular value decomposition
// X = U diag(sv) V^T.  Cofactors are covariant under orthogonal changes of basis, so with
// X' = U^T X V, f(X) = det(U) det(V) F(X') where F carries the rotated weights A' = U^T Aw V and
// G' = C2(U)^T Gw C2(V) (C2: the matrix of 2 x 2 minors).  Every cofactor of a diagonal matrix,
// and every derivative of one, is a product of singular values, which gives
//   df/dX = det(U) det(V) U D' V^T,
//   D'(a,a) = aS D1_a + sum_{r != a} A'(r,r) D2_{ar} + sum_{p not containing a} G'(p,p) D3_{p+a},
//   D'(a,b) = -A'(b,a) D2_{ab} + sum_{m != a,b} (-1)^(1+[m>a]+[m>b]) G'({b,m},{a,m}) D3_{abm},
// with D_j the product of the singular values outside the j listed indices.  Nothing is divided
// by a singular value, so the result is the exact derivative at any nullity.
// Aw[r k + c]; gamma_row(c1, c2) returns the two-electron table row of the left pair (already
// scaled by the Hamiltonian adjoint through `scale`); gX[r k + c] receives df/dX[r][c].
template <int KM>
__device__ __forceinline__ void svd_frame_adjoint(int k, const double* U, const double* V, const double* sv, double parity,
                                  double aS, const double* Aw, double scale, const double* gamma, int gd,
                                  const int* L, const int* Rr, double* gX) {
    // U[r][s] = U[s k + r], V[c][s] = V[s k + c]
    double Ap[KM * KM], Dp[KM * KM], W[KM * KM];
    for (int r = 0; r < k; ++r)
        for (int t = 0; t < k; ++t) {
            double acc = 0.0;
            for (int c = 0; c < k; ++c) acc = fma(Aw[r * k + c], V[t * k + c], acc);
            W[r * k + t] = acc;
        }
    for (int s2 = 0; s2 < k; ++s2)
        for (int t = 0; t < k; ++t) {
            double acc = 0.0;
            for (int r = 0; r < k; ++r) acc = fma(U[s2 * k + r], W[r * k + t], acc);
            Ap[s2 * k + t] = acc;
        }
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) {
            if (a == b) {
                double d = aS * sv_product_except<KM>(k, sv, 1u << a);
                for (int r = 0; r < k; ++r)
                    if (r != a) d = fma(Ap[r * k + r], sv_product_except<KM>(k, sv, (1u << a) | (1u << r)), d);
                Dp[a * k + a] = d;
            } else {
                Dp[a * k + b] = -Ap[b * k + a] * sv_product_except<KM>(k, sv, (1u << a) | (1u << b));
            }
        }
    if (k >= 3 && scale != 0.0) {
        constexpr int KP = KM * (KM - 1) / 2;
        const int kp = k * (k - 1) / 2;
        int pi[KP], pj[KP];  // local pair t = j (j - 1) / 2 + i, i < j
        for (int j = 1, t = 0; j < k; ++j)
            for (int i = 0; i < j; ++i, ++t) {
                pi[t] = i;
                pj[t] = j;
            }
        int rowp[KP];  // table column of each right (row) pair
        for (int t = 0; t < kp; ++t) rowp[t] = dev::anti_index(Rr[pi[t]], Rr[pj[t]]);
        double Vq[KP], Tq[KP];
        for (int q = 0; q < kp; ++q) {
            const int q1 = pi[q], q2 = pj[q];
            for (int t = 0; t < kp; ++t) {
                const int c1 = pi[t], c2 = pj[t];
                Vq[t] = V[q1 * k + c1] * V[q2 * k + c2] - V[q2 * k + c1] * V[q1 * k + c2];
            }
            for (int t = 0; t < kp; ++t) Tq[t] = 0.0;
            for (int t = 0; t < kp; ++t) {
                const double vc = Vq[t];
                const double* grow = gamma + (long long)dev::anti_index(L[pi[t]], L[pj[t]]) * gd;
                for (int rp = 0; rp < kp; ++rp) Tq[rp] = fma(__ldg(grow + rowp[rp]), vc, Tq[rp]);
            }
            // G'(p, q) for a row pair p = (p1 < p2)
            auto gprime = [&](int p1, int p2) {
                double acc = 0.0;
                for (int rp = 0; rp < kp; ++rp) {
                    const int r1 = pi[rp], r2 = pj[rp];
                    acc = fma(U[p1 * k + r1] * U[p2 * k + r2] - U[p2 * k + r1] * U[p1 * k + r2], Tq[rp], acc);
                }
                return scale * acc;
            };
            const double gqq = gprime(q1, q2);
            for (int a = 0; a < k; ++a)
                if (a != q1 && a != q2)
                    Dp[a * k + a] = fma(gqq, sv_product_except<KM>(k, sv, (1u << q1) | (1u << q2) | (1u << a)),
                                        Dp[a * k + a]);
            for (int side = 0; side < 2; ++side) {
                const int a = side ? q2 : q1, m = side ? q1 : q2;
                for (int b = 0; b < k; ++b) {
                    if (b == a || b == m) continue;
                    const double g = b < m ? gprime(b, m) : gprime(m, b);
                    const int parity = 1 + (m > a) + (m > b);
                    const double d3 = sv_product_except<KM>(k, sv, (1u << a) | (1u << b) | (1u << m));
                    Dp[a * k + b] = fma((parity & 1) ? -g : g, d3, Dp[a * k + b]);
                }
            }
        }
    }
    // gX = parity U D' V^T
    for (int a = 0; a < k; ++a)
        for (int c = 0; c < k; ++c) {
            double acc = 0.0;
            for (int b = 0; b < k; ++b) acc = fma(Dp[a * k + b], V[b * k + c], acc);
            W[a * k + c] = acc;
        }
    for (int r = 0; r < k; ++r)
        for (int c = 0; c < k; ++c) {
            double acc = 0.0;
            for (int a = 0; a < k; ++a) acc = fma(U[a * k + r], W[a * k + c], acc);
            gX[r * k + c] = parity * acc;
        }
}

// One thread per listed (uncertified) pair.  The adjoints are those of the exact cofactor
// polynomial, evaluated in the frame of the block's singular value decomposition with the
// singular values as computed (no rank truncation): the overlap adjoint by svd_frame_adjoint, the
// first cofactors C = det(U) det(V) U diag(D1) V^T for the one-electron adjoint and the P row
// (row i = idx - idx_begin, for the factor-column GEMM adj_U P^T after the kernel), and the
// second cofactors det(U) det(V) C2(U) diag(D2) C2(V)^T for the two-electron table (accumulated
// per CTA in shared memory when it fits).  For a full-rank block this is the same derivative as
// the inverse-based one, without its loss of accuracy (relative kappa * eps) on ill-conditioned
// blocks; where the reference truncates singular values below 1e-12 the two functions differ by
// terms of that order.  adj_u . l_m at each packed pair is read from Q.
template <int KM, int KC>  // KC > 0: electrons per string fixed at compile time (== KM)
__global__ void __launch_bounds__(128) careful_backward_kernel(BackArgs a, long long idx_begin, long long idx_end,
                                                               int all_pairs, double* gpart) {
    // this block's slot: two-electron table (gd^2), then the S and h adjoints (n^2 each);
    // only the block's own threads add into it, no shared memory, no barrier
    constexpr int KP = KM * (KM - 1) / 2;
    const int k = KC > 0 ? KC : a.k, n = a.n, np = a.ld, gd = a.gd;
    const long long N = a.N;
    double* gG = gpart + (size_t)blockIdx.x * ((size_t)gd * gd + 2 * (size_t)n * n);
    double* gSb = gG + (size_t)gd * gd;
    double* ghb = gSb + (size_t)n * n;
    for (long long idx = idx_begin + blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < idx_end;
         idx += (long long)gridDim.x * blockDim.x) {
        if (k == 0) break;
        long long u, v;
        careful_pair(a, idx, all_pairs, &u, &v);
        const long long t = record_index(u, v, N);
        const long long row = idx - idx_begin;
        const double* adj = a.adj + t * a.adj_stride;
        const double aS = adj[a.R], aH = adj[a.R + 1];
        int L[KM], Rr[KM];
        for (int c = 0; c < k; ++c) {
            L[c] = occ_byte(a.occ + 2 * u, c);
            Rr[c] = occ_byte(a.occ + 2 * v, c);
        }
        double x[KM * KM];  // x[c k + r] = X[r][c]
        for (int c = 0; c < k; ++c)
            for (int r = 0; r < k; ++r) x[c * k + r] = __ldg(a.S + L[c] * n + Rr[r]);
        double U[KM * KM], V[KM * KM], sv[KM];
        dev::jacobi_svd<KM>(k, x, sv, U, V);
        const double parity = dev::orthogonal_det_sign<KM>(k, U) * dev::orthogonal_det_sign<KM>(k, V);
        const double* qrow = a.Q + row * np;
        double GA[KM * KM];  // GA[r k + c] = aH h[L_c][R_r] + adj_u . l_m at pair(R_r, L_c)
        for (int r = 0; r < k; ++r)
            for (int c = 0; c < k; ++c)
                GA[r * k + c] = fma(aH, __ldg(a.h + L[c] * n + Rr[r]), qrow[dev::pair_index(Rr[r], L[c])]);
        {
            double gX[KM * KM];
            svd_frame_adjoint<KM>(k, U, V, sv, parity, aS, GA, aH, a.gamma, gd, L, Rr, gX);
            for (int r = 0; r < k; ++r)
                for (int c = 0; c < k; ++c) atomicAdd(gSb + L[c] * n + Rr[r], gX[r * k + c]);
        }
        // first cofactors
        double d1[KM];
        for (int s2 = 0; s2 < k; ++s2) d1[s2] = parity * sv_product_except<KM>(k, sv, 1u << s2);
        double* prow = a.Pout + row * np;
        for (int r = 0; r < k; ++r)
            for (int c = 0; c < k; ++c) {
                double A = 0.0;
                for (int s2 = 0; s2 < k; ++s2) A = fma(U[s2 * k + r] * d1[s2], V[s2 * k + c], A);
                if (aH != 0.0) atomicAdd(ghb + L[c] * n + Rr[r], aH * A);
                prow[dev::pair_index(Rr[r], L[c])] += A;
            }
        // second cofactors into the two-electron table
        if (aH != 0.0 && k >= 2) {
            const int kp = k * (k - 1) / 2;
            int pi[KP], pj[KP];
            for (int j = 1, q = 0; j < k; ++j)
                for (int i = 0; i < j; ++i, ++q) {
                    pi[q] = i;
                    pj[q] = j;
                }
            double d2[KP];
            for (int q = 0; q < kp; ++q) d2[q] = aH * parity * sv_product_except<KM>(k, sv, (1u << pi[q]) | (1u << pj[q]));
            for (int rp = 0; rp < kp; ++rp) {
                const int r1 = pi[rp], r2 = pj[rp];
                double w[KP];
                for (int q = 0; q < kp; ++q) {
                    const int p1 = pi[q], p2 = pj[q];
                    w[q] = d2[q] * (U[p1 * k + r1] * U[p2 * k + r2] - U[p2 * k + r1] * U[p1 * k + r2]);
                }
                const int rcol = dev::anti_index(Rr[r1], Rr[r2]);
                for (int cp = 0; cp < kp; ++cp) {
                    const int c1 = pi[cp], c2 = pj[cp];
                    double acc = 0.0;
                    for (int q = 0; q < kp; ++q) {
                        const int p1 = pi[q], p2 = pj[q];
                        acc = fma(w[q], V[p1 * k + c1] * V[p2 * k + c2] - V[p2 * k + c1] * V[p1 * k + c2], acc);
                    }
                    if (acc != 0.0) atomicAdd(gG + (long long)dev::anti_index(L[c1], L[c2]) * gd + rcol, acc);
                }
            }
        }
    }
}

// Sums the block slots [gG (g2) | gS (n2) | gh (n2)] into the outputs.
__global__ void reduce_slots_kernel(const double* __restrict__ gpart, int slots, int g2, int n2, double* __restrict__ gG,
                                    double* __restrict__ gS, double* __restrict__ gh) {
    const int size = g2 + 2 * n2;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < slots; ++b) acc += gpart[(size_t)b * size + i];
        if (i < g2)
            gG[i] += acc;
        else if (i < g2 + n2)
            gS[i - g2] += acc;
        else
            gh[i - g2 - n2] += acc;
    }
}

template <int K>
cudaError_t launch_backward(const BackArgs& b, cudaStream_t s) {
    const size_t smem = sizeof(double) * (2 * b.n * b.n + (size_t)(K * (K - 1) / 2) * b.gd);
    if (smem > 48 * 1024) {
        cudaError_t err = allow_dynamic_smem((const void*)spin_backward_kernel<K>, (int)smem);
        if (err != cudaSuccess) return err;
    }
    const int items = b.item_end - b.item_begin;
    const int grid = std::max(1, std::min(148 * 4, items));
    spin_backward_kernel<K><<<grid, 128, smem, s>>>(b);
    return cudaGetLastError();
}

// The listed (or all) pairs in chunks: gather their u-adjoint rows Ac, Q = L_f^T Ac, the careful
// kernel (P rows), gL += Ac P^T.
vb_status careful_chunks(vb_context* ctx, BackArgs b, long long count, int all_pairs, double* partial) {
    if (count <= 0) return VB_OK;
    cudaStream_t s = ctx->stream;
    const int np = b.ld, R = b.R;
    // chunk buffers: up to 768 MB, at most half of what the context budget has left
    const size_t left = ctx->budget > ctx->current ? ctx->budget - ctx->current : 0;
    const size_t target = std::max<size_t>((size_t)16 << 20, std::min<size_t>((size_t)768 << 20, left / 2));
    const long long chunk = std::min<long long>(
        count, std::max<long long>(1024, (long long)(target / (8ULL * (2 * np + R + 1)))));
    // per-block slots (two-electron table, S and h adjoints), summed once after the last chunk
    const size_t slot_bytes = sizeof(double) * ((size_t)b.gd * b.gd + 2 * (size_t)b.n * b.n);
    auto kernel = b.k == 7 ? careful_backward_kernel<7, 7>
                           : (b.k <= 8 ? careful_backward_kernel<8, 0> : careful_backward_kernel<dev::KMAX, 0>);
    int per_sm = 4;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0) != cudaSuccess || per_sm < 1) per_sm = 4;
    const int grid = 148 * std::min(per_sm, 8);  // one wave of resident blocks
    DeviceBuffer acb, qb, pb, slots;
    vb_status st;
    if ((st = slots.allocate(ctx, slot_bytes * grid)) != VB_OK) return st;
    if (cudaMemsetAsync(slots.ptr, 0, slot_bytes * grid, s) != cudaSuccess)
        return set_error(ctx, VB_ERR_CUDA, "vb_hs_plan_gradient: memset failed");
    if ((st = acb.allocate(ctx, sizeof(double) * (size_t)chunk * std::max(R, 1))) != VB_OK) return st;
    if ((st = qb.allocate(ctx, sizeof(double) * (size_t)chunk * np)) != VB_OK) return st;
    if ((st = pb.allocate(ctx, sizeof(double) * (size_t)chunk * np)) != VB_OK) return st;
    b.Q = qb.as<double>();
    b.Pout = pb.as<double>();
    for (long long i0 = 0; i0 < count; i0 += chunk) {
        const long long i1 = std::min(count, i0 + chunk), cnt = i1 - i0;
        cudaError_t err = cudaMemsetAsync(pb.ptr, 0, sizeof(double) * (size_t)cnt * np, s);
        if (err == cudaSuccess && R > 0) {
            gather_adjoint_kernel<<<(unsigned)std::min<long long>(4096, (cnt * R + 255) / 256), 256, 0, s>>>(
                b, i0, i1, all_pairs, acb.as<double>());
            err = cudaGetLastError();
            if (err == cudaSuccess)
                err = launch_factor_project(np, R, b.lf, np, acb.as<double>(), R, cnt, qb.as<double>(), np, s);
        } else if (err == cudaSuccess) {
            err = cudaMemsetAsync(qb.ptr, 0, sizeof(double) * (size_t)cnt * np, s);
        }
        if (err == cudaSuccess) {
            kernel<<<grid, 128, 0, s>>>(b, i0, i1, all_pairs, slots.as<double>());
            err = cudaGetLastError();
        }
        if (err == cudaSuccess)
            err = launch_factor_outer(np, R, acb.as<double>(), R, pb.as<double>(), np, cnt, b.gL, np, partial, s);
        if (err != cudaSuccess) return cuda_error(ctx, err, "vb_hs_plan_gradient (exact path)");
    }
    {
        const int g2 = b.gd * b.gd, n2 = b.n * b.n;
        reduce_slots_kernel<<<std::max(1, std::min(148 * 4, (g2 + 2 * n2 + 127) / 128)), 128, 0, s>>>(
            slots.as<double>(), grid, g2, n2, b.gG, b.gS, b.gh);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return cuda_error(ctx, err, "vb_hs_plan_gradient (block slots)");
    }
    return VB_OK;
}

}  // namespace

// Largest per-thread stack frame among the exact-path gradient kernels (see the context).
size_t gradient_stack_bytes() {
    size_t m = 0;
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, careful_backward_kernel<8, 0>) == cudaSuccess) m = std::max(m, fa.localSizeBytes);
    if (cudaFuncGetAttributes(&fa, careful_backward_kernel<7, 7>) == cudaSuccess) m = std::max(m, fa.localSizeBytes);
    return m;
}

namespace {

// ---- host-side small dense algebra ---------------------------------------------------------

// Least squares min ||A X - Y|| for A (m x r, column-major, full column rank) by Householder QR;
// Y is m x p, X (r x p) returned column-major.
std::vector<double> least_squares(std::vector<double> A, int m, int r, std::vector<double> Y, int p) {
    std::vector<double> tau(r, 0.0);
    for (int j = 0; j < r; ++j) {
        double norm = 0.0;
        for (int i = j; i < m; ++i) norm += A[i + (size_t)j * m] * A[i + (size_t)j * m];
        norm = std::sqrt(norm);
        if (norm == 0.0) continue;
        const double alpha = A[j + (size_t)j * m] > 0 ? -norm : norm;
        std::vector<double> vh(m, 0.0);
        vh[j] = A[j + (size_t)j * m] - alpha;
        for (int i = j + 1; i < m; ++i) vh[i] = A[i + (size_t)j * m];
        double vv = 0.0;
        for (int i = j; i < m; ++i) vv += vh[i] * vh[i];
        if (vv == 0.0) continue;
        auto reflect = [&](double* col) {
            double dot = 0.0;
            for (int i = j; i < m; ++i) dot += vh[i] * col[i];
            const double f = 2.0 * dot / vv;
            for (int i = j; i < m; ++i) col[i] -= f * vh[i];
        };
        for (int c = j; c < r; ++c) reflect(&A[(size_t)c * m]);
        for (int c = 0; c < p; ++c) reflect(&Y[(size_t)c * m]);
    }
    std::vector<double> X((size_t)r * p, 0.0);
    for (int c = 0; c < p; ++c)
        for (int i = r - 1; i >= 0; --i) {
            double acc = Y[i + (size_t)c * m];
            for (int k2 = i + 1; k2 < r; ++k2) acc -= A[i + (size_t)k2 * m] * X[k2 + (size_t)c * r];
            const double d = A[i + (size_t)i * m];
            X[i + (size_t)c * r] = d != 0.0 ? acc / d : 0.0;
        }
    return X;
}

int host_pair(int a, int b) {
    const int hi = std::max(a, b), lo = std::min(a, b);
    return hi * (hi + 1) / 2 + lo;
}

}  // namespace
}  // namespace vbcore

using namespace vbcore;

extern "C" vb_status vb_hs_plan_gradient(vb_hs_plan* p, const double* S, const double* h, const double* eri,
                                         int mem_space, const double* structure_coefficients, double eigenvalue,
                                         double* dS_out, double* dh_out, double* deri_out, const double* ri_factors,
                                         int n_aux, double* dri_out) {
    if (!p) return VB_ERR_INVALID;
    vb_context* ctx = p->ctx;
    if (!S || !h || !eri || !structure_coefficients || !dS_out || !dh_out)
        return set_error(ctx, VB_ERR_INVALID, "vb_hs_plan_gradient: null pointer");
    if (mem_space != VB_MEM_HOST && mem_space != VB_MEM_DEVICE)
        return set_error(ctx, VB_ERR_INVALID, "bad memory space");
    if ((ri_factors == nullptr) != (dri_out == nullptr) || (ri_factors && n_aux < 1))
        return set_error(ctx, VB_ERR_INVALID, "vb_hs_plan_gradient: ri_factors and dri_out go together");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int launches = 0;
    const double *dS = nullptr, *dh = nullptr, *deri = nullptr;
    vb_status st = VB_OK;
    if (records_match(p, S, h, eri, mem_space)) {
        dS = p->S_in.as<double>();
        dh = p->h_in.as<double>();
        deri = p->eri_in.as<double>();
    } else if ((st = prepare_spin_records(p, S, h, eri, mem_space, &dS, &dh, &deri, &launches)) != VB_OK) {
        return st;
    }
    const int n = p->n, np = p->np, gd = p->gd, R = p->R;
    const int adj_stride = R + 2;
    // scratch: w, coefficients, adjoint records, gradient accumulators
    const size_t n_gS = (size_t)n * n, n_gG = (size_t)std::max(gd, 1) * std::max(gd, 1), n_gL = (size_t)np * np;
    const size_t acc_doubles = 2 * n_gS + n_gG + n_gL;
    // the two-stage record adjoint when alpha strings carry four or more determinants on average
    const bool flip_adjoint = p->has_flip && p->shared_tables && p->ka > 0 && p->R <= 128;
    const int chunk = flip_adjoint && p->n_det >= 4LL * p->Na ? two_stage_chunk(p->Nb) : 0;
    const size_t order_doubles = chunk ? (size_t)p->n_det + ((size_t)p->n_det + 1) / 2 : 0;
    if ((st = p->grad_acc.allocate(ctx, sizeof(double) * (acc_doubles + p->n_det + p->n_str + order_doubles))) !=
        VB_OK)
        return st;
    double* gS = p->grad_acc.as<double>();
    double* gh = gS + n_gS;
    double* gG = gh + n_gS;
    double* gL = gG + n_gG;
    double* w = gL + n_gL;
    double* cdev = w + p->n_det;
    double* ws = cdev + p->n_str;
    int* bs = reinterpret_cast<int*>(ws + p->n_det);
    const long long adj_a_n = std::max(1LL, p->npairs_a) * adj_stride;
    const long long adj_b_n = p->shared_tables ? 0 : std::max(1LL, p->npairs_b) * adj_stride;
    if ((st = p->adj_a.allocate(ctx, sizeof(double) * adj_a_n)) != VB_OK) return st;
    if (!p->shared_tables && p->kb > 0 && (st = p->adj_b.allocate(ctx, sizeof(double) * adj_b_n)) != VB_OK) return st;
    cudaError_t err = cudaMemsetAsync(gS, 0, sizeof(double) * acc_doubles, s);
    if (err == cudaSuccess) err = cudaMemsetAsync(p->adj_a.ptr, 0, sizeof(double) * adj_a_n, s);
    if (err == cudaSuccess && p->adj_b.ptr) err = cudaMemsetAsync(p->adj_b.ptr, 0, sizeof(double) * adj_b_n, s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(cdev, structure_coefficients, sizeof(double) * p->n_str,
                              mem_space == VB_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s);
    if (err == cudaSuccess) {
        det_weights_kernel<<<(unsigned)std::min<long long>(4096, (p->n_det + 255) / 256), 256, 0, s>>>(
            p->n_det, p->det_off.as<int64_t>(), p->det_str.as<int>(), p->det_coef.as<double>(), cdev, w);
        err = cudaGetLastError();
    }
    AdjArgs aa{};
    aa.f = full_args(p);
    aa.w = w;
    aa.lambda = eigenvalue;
    aa.adj_a = p->adj_a.as<double>();
    aa.adj_b = p->shared_tables ? p->adj_a.as<double>() : p->adj_b.as<double>();
    aa.adj_stride = adj_stride;
    if (err == cudaSuccess) {
        if (chunk) {
            alpha_order_kernel<<<(unsigned)std::min<long long>(4096, (p->n_det + 255) / 256), 256, 0, s>>>(
                p->n_det, p->alpha_dets.as<int>(), w, p->det_beta.as<int>(), ws, bs);
            err = cudaGetLastError();
            if (err == cudaSuccess) {
                const int* aoff = p->alpha_off.as<int>();
                err = chunk == 16 ? launch_two_stage<16>(aa, aoff, ws, bs, s)
                      : chunk == 8 ? launch_two_stage<8>(aa, aoff, ws, bs, s)
                                   : launch_two_stage<4>(aa, aoff, ws, bs, s);
            }
        } else {
            if (flip_adjoint)
                det_pair_adjoint_flip_kernel<<<148 * 8, 256, 0, s>>>(aa, p->alpha_off.as<int>(),
                                                                     p->alpha_dets.as<int>());
            else
                det_pair_adjoint_kernel<<<148 * 8, 256, 0, s>>>(aa);
            err = cudaGetLastError();
        }
    }
    // split-K partials of the factor-column adjoint (one R x np block per CTA of factor_outer)
    DeviceBuffer partial;
    if (err == cudaSuccess && (st = partial.allocate(ctx, sizeof(double) * kOuterMaxParts * (size_t)std::max(1, R) * np)) != VB_OK)
        return st;
    // backward through each distinct spin table
    for (int beta = 0; beta < 2 && err == cudaSuccess; ++beta) {
        const int k = beta ? p->kb : p->ka;
        if (k <= 0 || (beta && p->shared_tables)) continue;
        BackArgs b{};
        b.n = n;
        b.k = k;
        b.N = beta ? p->Nb : p->Na;
        b.occ = beta ? p->occ_b.as<uint64_t>() : p->occ_a.as<uint64_t>();
        b.S = dS;
        b.h = dh;
        b.eri = deri;
        b.gamma = p->gamma.as<double>();
        b.gd = gd;
        b.lf = p->lf.as<double>();
        b.ld = np;
        b.R = R;
        b.adj = beta ? p->adj_b.as<double>() : p->adj_a.as<double>();
        b.adj_stride = adj_stride;
        b.gS = gS;
        b.gh = gh;
        b.gG = gG;
        b.gL = gL;
        b.careful_count = p->counters.as<unsigned long long>() + 2 + beta;
        b.careful_list = beta ? p->list_b.as<unsigned long long>() : p->list_a.as<unsigned long long>();
        err = cudaMemsetAsync(b.careful_count, 0, sizeof(unsigned long long), s);
        if (err != cudaSuccess) break;
        const bool fast = k <= 8 && frame_spin_supported(n, k, R);
        if (fast) {
            // chunks of whole work items (left string u, right strings v0 .. v0 + 127): per chunk
            // Q = L_f^T adj_U (the u-adjoint contracted with every factor column at every packed
            // pair), the backward kernel (writes P = A scattered onto packed pairs), then
            // gL += adj_U P^T -- the two contractions over the R factor columns as FP64 GEMMs
            const long long NN = b.N;
            std::vector<int2> items;
            std::vector<long long> rec_off;  // first record of each item, then the total
            long long tot = 0;
            for (long long u = 0; u < NN; ++u)
                for (long long v0 = u; v0 < NN; v0 += kSpinBlock) {
                    items.push_back(make_int2((int)u, (int)v0));
                    rec_off.push_back(tot);
                    tot += std::min<long long>(kSpinBlock, NN - v0);
                }
            rec_off.push_back(tot);
            const long long cap = std::max<long long>(kSpinBlock, ((long long)256 << 20) / (8LL * np));
            DeviceBuffer ditems, qbuf, pbuf;
            if ((st = upload(ctx, ditems, items.data(), sizeof(int2) * items.size())) != VB_OK) return st;
            const long long rows_max = std::min<long long>(cap + kSpinBlock, tot);
            if ((st = qbuf.allocate(ctx, sizeof(double) * (size_t)np * rows_max)) != VB_OK) return st;
            if ((st = pbuf.allocate(ctx, sizeof(double) * (size_t)np * rows_max)) != VB_OK) return st;
            b.items = ditems.as<int2>();
            b.Q = qbuf.as<double>();
            b.Pout = pbuf.as<double>();
            for (size_t i0 = 0; i0 < items.size() && err == cudaSuccess;) {
                size_t i1 = i0;
                while (i1 < items.size() && rec_off[i1 + 1] - rec_off[i0] <= cap) ++i1;
                if (i1 == i0) ++i1;
                const long long tb = rec_off[i0], rows = rec_off[i1] - tb;
                const double* A = b.adj + tb * adj_stride;
                err = launch_factor_project(np, R, b.lf, np, A, adj_stride, rows, qbuf.as<double>(), np, s);
                if (err == cudaSuccess) err = cudaMemsetAsync(pbuf.ptr, 0, sizeof(double) * (size_t)np * rows, s);
                if (err != cudaSuccess) break;
                b.item_begin = (int)i0;
                b.item_end = (int)i1;
                b.record_base = tb;
                switch (k) {
                    case 1: err = launch_backward<1>(b, s); break;
                    case 2: err = launch_backward<2>(b, s); break;
                    case 3: err = launch_backward<3>(b, s); break;
                    case 4: err = launch_backward<4>(b, s); break;
                    case 5: err = launch_backward<5>(b, s); break;
                    case 6: err = launch_backward<6>(b, s); break;
                    case 7: err = launch_backward<7>(b, s); break;
                    case 8: err = launch_backward<8>(b, s); break;
                    default: break;
                }
                if (err != cudaSuccess) break;
                err = launch_factor_outer(np, R, A, adj_stride, pbuf.as<double>(), np, rows, gL, np,
                                          partial.as<double>(), s);
                if (err != cudaSuccess) break;
                i0 = i1;
            }
            if (err != cudaSuccess) break;
            unsigned long long listed = 0;
            err = cudaMemcpyAsync(&listed, b.careful_count, sizeof(listed), cudaMemcpyDeviceToHost, s);
            if (err == cudaSuccess) err = cudaStreamSynchronize(s);
            if (err != cudaSuccess) break;
            if ((st = careful_chunks(ctx, b, (long long)listed, 0, partial.as<double>())) != VB_OK) return st;
        } else {
            const long long NN = b.N;
            if ((st = careful_chunks(ctx, b, NN * (NN + 1) / 2, 1, partial.as<double>())) != VB_OK) return st;
        }
        err = cudaGetLastError();
    }
    std::vector<double> hS(n_gS), hh(n_gS), hG(n_gG), hL(n_gL), hlf((size_t)np * np);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hS.data(), gS, sizeof(double) * n_gS, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hh.data(), gh, sizeof(double) * n_gS, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hG.data(), gG, sizeof(double) * n_gG, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hL.data(), gL, sizeof(double) * n_gL, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(hlf.data(), p->lf.ptr, sizeof(double) * (size_t)np * np, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "vb_hs_plan_gradient");

    // symmetric gradients of S and h: dE = sum G_ij dS_ij for symmetric dS
    std::vector<double> outS(n_gS), outh(n_gS);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            outS[i + (size_t)j * n] = 0.5 * (hS[i + (size_t)j * n] + hS[j + (size_t)i * n]);
            outh[i + (size_t)j * n] = 0.5 * (hh[i + (size_t)j * n] + hh[j + (size_t)i * n]);
        }
    // factor-column adjoint G (np x R, G[q][m] = hL[q * np + m]) = Ksym L_f Sigma with
    // Ksym = dE/dK symmetrized; X = G Sigma, Ksym L_f = X
    std::vector<double> Xm((size_t)np * R), Lf((size_t)np * R);
    for (int q = 0; q < np; ++q)
        for (int m = 0; m < R; ++m) {
            Xm[q + (size_t)m * np] = hL[(size_t)q * np + m] * (m < p->r_pos ? 1.0 : -1.0);
            Lf[q + (size_t)m * np] = hlf[(size_t)q * np + m];
        }
    if (deri_out) {
        if (R != np)
            return set_error(ctx, VB_ERR_UNSUPPORTED,
                             "vb_hs_plan_gradient: the pair kernel has rank " + std::to_string(R) + " < " +
                                 std::to_string(np) +
                                 "; packed-integral gradients need a full-rank kernel (pass RI factors instead)");
        // Ksym = X L_f^-1  <=>  L_f^T Ksym^T = X^T
        std::vector<double> LfT((size_t)np * np), XT((size_t)np * np);
        for (int i = 0; i < np; ++i)
            for (int j = 0; j < np; ++j) {
                LfT[i + (size_t)j * np] = Lf[j + (size_t)i * np];
                XT[i + (size_t)j * np] = Xm[j + (size_t)i * np];
            }
        std::vector<double> KsT = least_squares(LfT, np, np, XT, np);  // = Ksym^T
        const long long ne = (long long)np * (np + 1) / 2;
        std::vector<double> outE(ne, 0.0);
        for (int a2 = 0; a2 < np; ++a2)
            for (int b2 = 0; b2 <= a2; ++b2) {
                const double ks = 0.5 * (KsT[a2 + (size_t)b2 * np] + KsT[b2 + (size_t)a2 * np]);
                outE[(size_t)a2 * (a2 + 1) / 2 + b2] += a2 == b2 ? 0.5 * ks : ks;
            }
        // same-spin table: Gamma[(i<k)][(j<l)] = (ij|kl) - (il|kj)
        for (int row = 0; row < gd; ++row) {
            int kk = 1;
            while ((kk + 1) * kk / 2 <= row) ++kk;
            const int i = row - kk * (kk - 1) / 2;
            for (int col = 0; col < gd; ++col) {
                const double g = hG[(size_t)row * gd + col];
                if (g == 0.0) continue;
                int l = 1;
                while ((l + 1) * l / 2 <= col) ++l;
                const int j = col - l * (l - 1) / 2;
                outE[host_pair(host_pair(i, j), host_pair(kk, l))] += g;
                outE[host_pair(host_pair(i, l), host_pair(kk, j))] -= g;
            }
        }
        if (mem_space == VB_MEM_HOST)
            std::copy(outE.begin(), outE.end(), deri_out);
        else if ((err = cudaMemcpyAsync(deri_out, outE.data(), sizeof(double) * ne, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return cuda_error(ctx, err, "vb_hs_plan_gradient");
    }
    if (ri_factors) {
        // dE/dF for K = F F^T with F (np x n_aux) spanning the factor space: Ksym F = X M, F = L_f M
        std::vector<double> F((size_t)np * n_aux);
        if (mem_space == VB_MEM_HOST)
            std::copy(ri_factors, ri_factors + F.size(), F.begin());
        else if ((err = cudaMemcpy(F.data(), ri_factors, sizeof(double) * F.size(), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_error(ctx, err, "vb_hs_plan_gradient");
        std::vector<double> M = least_squares(Lf, np, R, F, n_aux);  // R x n_aux
        std::vector<double> D((size_t)np * n_aux, 0.0);
        for (int q = 0; q < np; ++q)
            for (int c = 0; c < n_aux; ++c) {
                double acc = 0.0;
                for (int m = 0; m < R; ++m) acc += Xm[q + (size_t)m * np] * M[m + (size_t)c * R];
                D[q + (size_t)c * np] = acc;
            }
        // same-spin table through K: Gamma = K-entries difference; its adjoint maps onto the
        // packed integrals, which are F F^T entries: d(ij|kl) = dF_p F_q^T + F_p dF_q^T
        for (int row = 0; row < gd; ++row) {
            int kk = 1;
            while ((kk + 1) * kk / 2 <= row) ++kk;
            const int i = row - kk * (kk - 1) / 2;
            for (int col = 0; col < gd; ++col) {
                const double g = hG[(size_t)row * gd + col];
                if (g == 0.0) continue;
                int l = 1;
                while ((l + 1) * l / 2 <= col) ++l;
                const int j = col - l * (l - 1) / 2;
                const int p1 = host_pair(i, j), q1 = host_pair(kk, l), p2 = host_pair(i, l), q2 = host_pair(kk, j);
                for (int c = 0; c < n_aux; ++c) {
                    D[p1 + (size_t)c * np] += g * F[q1 + (size_t)c * np];
                    D[q1 + (size_t)c * np] += g * F[p1 + (size_t)c * np];
                    D[p2 + (size_t)c * np] -= g * F[q2 + (size_t)c * np];
                    D[q2 + (size_t)c * np] -= g * F[p2 + (size_t)c * np];
                }
            }
        }
        if (mem_space == VB_MEM_HOST)
            std::copy(D.begin(), D.end(), dri_out);
        else if ((err = cudaMemcpyAsync(dri_out, D.data(), sizeof(double) * D.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return cuda_error(ctx, err, "vb_hs_plan_gradient");
    }
    if (mem_space == VB_MEM_HOST) {
        std::copy(outS.begin(), outS.end(), dS_out);
        std::copy(outh.begin(), outh.end(), dh_out);
    } else {
        err = cudaMemcpyAsync(dS_out, outS.data(), sizeof(double) * n_gS, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(dh_out, outh.data(), sizeof(double) * n_gS, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) return cuda_error(ctx, err, "vb_hs_plan_gradient");
    }
    return VB_OK;
}
