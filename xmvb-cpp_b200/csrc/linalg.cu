// Dense FP64 metric linear algebra on the device.
//
//  * vb_metric_cholesky: upper Cholesky factor S = U^T U of a symmetric positive-definite
//    metric (overlap_upper, src/vbscf/orbitals/preparation/cholesky.hpp:10-15, Eigen::LLT).
//  * vb_generalized_eigh: H C = S C E with LAPACK dsygvd(itype 1, 'V', 'U') semantics
//    (GeneralizedEigensolver::solve_dense, src/linalg/eigensolver.cpp:365-388): only the upper
//    triangles of H and S are read, eigenvalues ascending, C^T S C = I, and info = n + i when
//    the leading minor of order i of S is not positive definite
//    (check_generalized_eigensolver_info, eigensolver.cpp:39-49).
//  * vb_generalized_eigh_batched: many independent problems, one CTA each.
//
// Method (one kernel): blocked right-looking Cholesky (32-column panels), blocked inverse of
// the triangular factor, A = U^-T H U^-1 and C = U^-1 Q as tiled GEMMs, and the symmetric
// eigenproblem of A by block Jacobi in round-robin (tournament) order over 16-index blocks:
// each round diagonalizes the 32 x 32 subproblems of m_b / 2 disjoint block pairs in shared
// memory and applies the resulting orthogonal 32 x 32 factors to A and the eigenvectors as
// small GEMMs.  Jacobi needs no tridiagonalization, is parallel within a round and converges
// quadratically.
//
// A single problem runs as a cooperative launch (one CTA per SM) whose phases are separated
// by a grid barrier with a bounded spin; a batch runs one problem per CTA with __syncthreads.
// Data written inside the kernel is read with __ldcg (L2), never through the incoherent L1
// or read-only paths.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace vbcore {
namespace {

constexpr int kThreads = 256;
constexpr int kTile = 32;
constexpr long long kBarrierSpinLimit = 1ll << 26;  // default: ~ seconds with 64 ns sleeps
constexpr int kMaxSweeps = 60;
constexpr int kSmallProblem = 96;  // single-problem calls at or below this size use one CTA

struct Control {
    unsigned bar_count;
    unsigned bar_gen;
    int err;       // 1: a grid barrier gave up waiting
    int info;      // Cholesky failure: order of the first non-positive leading minor
    unsigned rotations[3];
    int sweeps;
    double fro2;   // squared Frobenius norm of the reduced matrix
};

struct EighArgs {
    int n;
    int mode;            // 0: Cholesky only, 1: full generalized eigenproblem, 2: Cholesky + U^-1
    const double* H;     // n x n, column-major (upper triangle read)
    const double* S;     // n x n, column-major (upper triangle read)
    double* U;           // Cholesky factor (output for mode 0)
    double* Ui;          // U^-1 (zero-initialised)
    double* T;           // scratch n x n
    double* A0;          // ping-pong n x n
    double* A1;
    double* V;           // Jacobi rotations (zero-initialised)
    double* W;           // per block pair 32 x 32 subproblem rotations
    int* rank;           // n
    double* evals;       // n
    double* evecs;       // n x n
    Control* ctl;        // zero-initialised
    long long spin_limit;  // polls a grid-barrier wait makes before it gives up (ctl->err = 1)
};

struct BlockSync {
    __device__ __forceinline__ bool operator()() const {
        __syncthreads();
        return true;
    }
};

// Grid barrier whose waits are bounded: a CTA that polls `spin_limit` times without the barrier
// opening sets ctl->err and leaves; every other waiting CTA leaves as soon as it sees err, so the
// kernel always ends and the host reads VB_ERR_TIMEOUT.
struct GridSync {
    Control* ctl;
    unsigned nblocks;
    long long spin_limit;
    __device__ bool operator()() const {
        __syncthreads();
        if (threadIdx.x == 0) {
            volatile unsigned* gen = &ctl->bar_gen;
            const unsigned g = *gen;
            __threadfence();
            if (atomicAdd(&ctl->bar_count, 1u) == nblocks - 1) {
                atomicExch(&ctl->bar_count, 0u);
                __threadfence();
                atomicAdd(&ctl->bar_gen, 1u);
            } else {
                long long spins = 0;
                while (*gen == g) {
                    if (++spins > spin_limit) {
                        atomicExch(&ctl->err, 1);
                        break;
                    }
                    if (*(volatile int*)&ctl->err) break;
                    __nanosleep(64);
                }
            }
            __threadfence();
        }
        __syncthreads();
        return *(volatile int*)&ctl->err == 0;
    }
};

__device__ __forceinline__ double ld(const double* p) { return __ldcg(p); }

// Element (r, c) of the symmetric matrix whose upper triangle is stored column-major in M.
__device__ __forceinline__ double upper_elem(const double* M, int n, int r, int c) {
    return r <= c ? ld(M + r + (long long)c * n) : ld(M + c + (long long)r * n);
}

struct Shared {
    double a[kTile][kTile + 1];
    double b[kTile][kTile + 1];
    double d[kTile][kTile + 1];
    int flag;
};

// FP64 tensor-core step (mma.sync m8n8k4): this lane's fragment (row lane / 4, columns
// 2 (lane % 4) + {0, 1}) of the 8 x 8 output tile (mt, nt) of a 32 x 32 product, accumulated over
// k < 32 with A(r, k) = fa(r, k) and B(k, c) = fb(k, c).  Eight warps cover the 16 output tiles
// of a 32 x 32 tile two at a time (tiles warp and warp + 8).
__device__ __forceinline__ void dmma8(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

template <class FA, class FB>
__device__ __forceinline__ void mma_tile32(double (&acc)[2], FA fa, FB fb, int mt, int nt) {
    const int lane = threadIdx.x & 31, gr = lane >> 2, gc = lane & 3;
#pragma unroll
    for (int k0 = 0; k0 < kTile; k0 += 4) dmma8(acc, fa(8 * mt + gr, k0 + gc), fb(k0 + gc, 8 * nt + gr));
}

// ---------------------------------------------------------------------------------------
// Cholesky, S = U^T U (upper), right-looking with 32-column panels.
template <class Sync>
__device__ bool cholesky(const EighArgs& a, const Sync& sync, Shared& sh, int cta, int ncta) {
    const int n = a.n;
    const int tid = threadIdx.x;
    const long long gtid = (long long)cta * blockDim.x + tid, gstride = (long long)ncta * blockDim.x;
    double* U = a.U;
    for (long long e = gtid; e < (long long)n * n; e += gstride) {
        const int r = (int)(e % n), c = (int)(e / n);
        U[e] = r <= c ? ld(a.S + e) : 0.0;
    }
    if (!sync()) return false;
    for (int j0 = 0; j0 < n; j0 += kTile) {
        const int jb = min(kTile, n - j0);
        const int j1 = j0 + jb;
        // (1) factor the diagonal block
        if (cta == 0) {
            for (int e = tid; e < jb * jb; e += blockDim.x) {
                const int r = e % jb, c = e / jb;
                sh.d[r][c] = r <= c ? ld(U + (j0 + r) + (long long)(j0 + c) * n) : 0.0;
            }
            if (tid == 0) sh.flag = 0;
            __syncthreads();
            for (int k = 0; k < jb; ++k) {
                if (tid == 0) {
                    const double dk = sh.d[k][k];
                    if (!(dk > 0.0) || !isfinite(dk))
                        sh.flag = j0 + k + 1;
                    else
                        sh.d[k][k] = sqrt(dk);
                }
                __syncthreads();
                if (sh.flag) break;
                const double piv = sh.d[k][k];
                for (int c = k + 1 + tid; c < jb; c += blockDim.x) sh.d[k][c] /= piv;
                __syncthreads();
                const int w = jb - k - 1;
                for (int e = tid; e < w * w; e += blockDim.x) {
                    const int r = k + 1 + e % w, c = k + 1 + e / w;
                    if (r <= c) sh.d[r][c] = fma(-sh.d[k][r], sh.d[k][c], sh.d[r][c]);
                }
                __syncthreads();
            }
            if (sh.flag) {
                if (tid == 0) atomicExch(&a.ctl->info, sh.flag);
            } else {
                for (int e = tid; e < jb * jb; e += blockDim.x) {
                    const int r = e % jb, c = e / jb;
                    if (r <= c) U[(j0 + r) + (long long)(j0 + c) * n] = sh.d[r][c];
                }
            }
        }
        if (!sync()) return false;
        if (*(volatile int*)&a.ctl->info) return false;
        if (j1 >= n) break;
        // (2) panel row: U12 = U11^-T A12, one column per thread
        for (int e = tid; e < jb * jb; e += blockDim.x) {
            const int r = e % jb, c = e / jb;
            sh.d[r][c] = r <= c ? ld(U + (j0 + r) + (long long)(j0 + c) * n) : 0.0;
        }
        __syncthreads();
        for (long long c = j1 + gtid; c < n; c += gstride) {
            double x[kTile];
#pragma unroll
            for (int r = 0; r < kTile; ++r) x[r] = r < jb ? ld(U + (j0 + r) + c * n) : 0.0;
#pragma unroll
            for (int r = 0; r < kTile; ++r) {
                if (r < jb) {
                    double s = x[r];
#pragma unroll
                    for (int k = 0; k < r; ++k) s = fma(-sh.d[k][r], x[k], s);
                    x[r] = s / sh.d[r][r];
                }
            }
#pragma unroll
            for (int r = 0; r < kTile; ++r)
                if (r < jb) U[(j0 + r) + c * n] = x[r];
        }
        if (!sync()) return false;
        // (3) trailing update of the upper part: A22 -= U12^T U12, 32 x 32 tiles (ti <= tj)
        const int m = n - j1;
        const int nt = (m + kTile - 1) / kTile;
        const int ntiles = nt * (nt + 1) / 2;
        for (int t = cta; t < ntiles; t += ncta) {
            int tj = 0;
            while ((tj + 1) * (tj + 2) / 2 <= t) ++tj;
            const int ti = t - tj * (tj + 1) / 2;
            for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                const int k = e % kTile, i = e / kTile;
                const int ri = j1 + ti * kTile + i, cj = j1 + tj * kTile + i;
                sh.a[k][i] = (k < jb && ri < n) ? ld(U + (j0 + k) + (long long)ri * n) : 0.0;
                sh.b[k][i] = (k < jb && cj < n) ? ld(U + (j0 + k) + (long long)cj * n) : 0.0;
            }
            __syncthreads();
            // A22 tile -= U12(:, ti)^T U12(:, tj) on the FP64 tensor cores (rows of the panel past
            // jb are zero in sh.a / sh.b)
            const int warp = tid >> 5, lane = tid & 31;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int ot = warp + 8 * q, mt = ot & 3, nt = ot >> 2;
                double acc[2] = {0.0, 0.0};
                mma_tile32(
                    acc, [&](int r, int k) { return sh.a[k][r]; }, [&](int k, int c) { return sh.b[k][c]; }, mt, nt);
                const int r = j1 + ti * kTile + 8 * mt + (lane >> 2);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = j1 + tj * kTile + 8 * nt + 2 * (lane & 3) + h;
                    if (r < n && c < n && r <= c) U[r + (long long)c * n] -= acc[h];
                }
            }
            __syncthreads();
        }
        if (!sync()) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------------------
// Ui = U^-1 (upper), by 32 x 32 blocks: diagonal blocks first, then block diagonals
// Ui[I][J] = -Ui[I][I] sum_{K=I+1..J} U[I][K] Ui[K][J].
template <class Sync>
__device__ bool triangular_inverse(const EighArgs& a, const Sync& sync, Shared& sh, int cta, int ncta) {
    const int n = a.n;
    const int tid = threadIdx.x;
    const int nb = (n + kTile - 1) / kTile;
    const double* U = a.U;
    double* Ui = a.Ui;
    for (int I = cta; I < nb; I += ncta) {
        const int r0 = I * kTile, bi = min(kTile, n - r0);
        for (int e = tid; e < kTile * kTile; e += blockDim.x) {
            const int r = e % kTile, c = e / kTile;
            sh.d[r][c] = (r < bi && c < bi && r <= c) ? ld(U + (r0 + r) + (long long)(r0 + c) * n) : 0.0;
            sh.a[r][c] = 0.0;
        }
        __syncthreads();
        if (tid < bi) {
            const int j = tid;
            sh.a[j][j] = 1.0 / sh.d[j][j];
            for (int i = j - 1; i >= 0; --i) {
                double s = 0.0;
                for (int k = i + 1; k <= j; ++k) s = fma(sh.d[i][k], sh.a[k][j], s);
                sh.a[i][j] = -s / sh.d[i][i];
            }
        }
        __syncthreads();
        for (int e = tid; e < bi * bi; e += blockDim.x) {
            const int r = e % bi, c = e / bi;
            if (r <= c) Ui[(r0 + r) + (long long)(r0 + c) * n] = sh.a[r][c];
        }
        __syncthreads();
    }
    if (!sync()) return false;
    for (int dgl = 1; dgl < nb; ++dgl) {
        for (int I = cta; I + dgl < nb; I += ncta) {
            const int J = I + dgl;
            const int r0 = I * kTile, c0 = J * kTile;
            const int warp = tid >> 5, lane = tid & 31, gr = lane >> 2, gc = lane & 3;
            // P = sum_K U[I][K] Ui[K][J] and Ui[I][J] = -Ui[I][I] P on the FP64 tensor cores
            double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
            for (int K = I + 1; K <= J; ++K) {
                const int k0 = K * kTile;
                for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                    const int r = e % kTile, c = e / kTile;
                    sh.a[r][c] = (r0 + r < n && k0 + c < n) ? ld(U + (r0 + r) + (long long)(k0 + c) * n) : 0.0;
                    sh.b[r][c] = (k0 + r < n && c0 + c < n) ? ld(Ui + (k0 + r) + (long long)(c0 + c) * n) : 0.0;
                }
                __syncthreads();
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int ot = warp + 8 * q;
                    mma_tile32(
                        acc[q], [&](int r, int k) { return sh.a[r][k]; }, [&](int k, int c) { return sh.b[k][c]; },
                        ot & 3, ot >> 2);
                }
                __syncthreads();
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int ot = warp + 8 * q, mt = ot & 3, nt = ot >> 2;
#pragma unroll
                for (int h = 0; h < 2; ++h) sh.b[8 * mt + gr][8 * nt + 2 * gc + h] = acc[q][h];
            }
            for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                const int r = e % kTile, c = e / kTile;
                sh.a[r][c] = (r0 + r < n && r0 + c < n) ? ld(Ui + (r0 + r) + (long long)(r0 + c) * n) : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int ot = warp + 8 * q, mt = ot & 3, nt = ot >> 2;
                double out[2] = {0.0, 0.0};
                mma_tile32(
                    out, [&](int r, int k) { return sh.a[r][k]; }, [&](int k, int c) { return sh.b[k][c]; }, mt, nt);
                const int r = r0 + 8 * mt + gr;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = c0 + 8 * nt + 2 * gc + h;
                    if (r < n && c < n) Ui[r + (long long)c * n] = -out[h];
                }
            }
            __syncthreads();
        }
        if (!sync()) return false;
    }
    return true;
}

// C (n x n) = op_A * op_B with 32 x 32 output tiles; la(r, k), lb(k, c) return the operands.
template <class LA, class LB>
__device__ void gemm_tiles(int n, LA la, LB lb, double* C, Shared& sh, int cta, int ncta) {
    const int tid = threadIdx.x;
    const int tm = (n + kTile - 1) / kTile;
    for (int t = cta; t < tm * tm; t += ncta) {
        const int ti = t % tm, tj = t / tm;
        const int i = tid & 31, jq = tid >> 5;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k0 = 0; k0 < n; k0 += kTile) {
            for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                const int r = e % kTile, c = e / kTile;
                const int gr = ti * kTile + r, gk = k0 + c;
                sh.a[r][c] = (gr < n && gk < n) ? la(gr, gk) : 0.0;
                const int gk2 = k0 + r, gc = tj * kTile + c;
                sh.b[r][c] = (gk2 < n && gc < n) ? lb(gk2, gc) : 0.0;
            }
            __syncthreads();
#pragma unroll 8
            for (int k = 0; k < kTile; ++k) {
                const double av = sh.a[i][k];
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] = fma(av, sh.b[k][jq + 8 * q], acc[q]);
            }
            __syncthreads();
        }
        const int r = ti * kTile + i;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = tj * kTile + jq + 8 * q;
            if (r < n && c < n) C[r + (long long)c * n] = acc[q];
        }
    }
}

// Round-robin pairing: round r of m - 1 (m even), pair i of m / 2 -> (p, q), p < q.
__device__ __forceinline__ void round_pair(int m, int r, int i, int* p, int* q) {
    auto pos = [&](int k) { return k == 0 ? 0 : 1 + (k - 1 + r) % (m - 1); };
    int a = pos(i), b = pos(m - 1 - i);
    *p = min(a, b);
    *q = max(a, b);
}

// Block Jacobi.  Indices are grouped in blocks of kHalf = 16; block pairs (P, Q) meet in
// round-robin order, m_b - 1 rounds per sweep.  A round (1) diagonalizes every 32 x 32
// subproblem [[A_PP, A_PQ], [A_QP, A_QQ]] by one cyclic Jacobi sweep in shared memory, giving an
// orthogonal W per pair, and (2) applies them: A'[I_i, I_j] = W_i^T A[I_i, I_j] W_j for all pair
// combinations (ping-pong buffers) and V[:, I_i] <- V[:, I_i] W_i.  Rotations of the inner sweep
// use J = [[c, s], [-s, c]] annihilating g_pq in J^T G J (Golub & Van Loan, Algorithm 8.4.1) and
// are skipped when |g_pq| <= 1e-15 sqrt(|g_pp g_qq|) or <= 1e-14 ||A||_F (the rounding level of
// the blocked update); a sweep without an applied rotation ends the iteration.
constexpr int kHalf = 16;

__device__ __forceinline__ int sub_index(int P, int Q, int l, int n) {
    const int g = l < kHalf ? P * kHalf + l : Q * kHalf + (l - kHalf);
    return g < n ? g : -1;
}

template <class Sync>
__device__ bool jacobi(const EighArgs& a, const Sync& sync, Shared& sh, int cta, int ncta, double** A_final) {
    const int n = a.n;
    const int nbk = (n + kHalf - 1) / kHalf;
    const int mb = nbk + (nbk & 1);
    const int pairs = mb / 2;
    const int tid = threadIdx.x;
    const double fro = sqrt(ld(&a.ctl->fro2));
    const double skip_abs = 1.0e-14 * fro + 1.0e-300;
    double* Ain = a.A0;
    double* Aout = a.A1;
    double* Wg = a.W;
    __shared__ double rc[kHalf], rs[kHalf], rt[kHalf];
    __shared__ int rapplied, roff;
    __shared__ unsigned char inner_p[kTile - 1][kHalf], inner_q[kTile - 1][kHalf];
    for (int e = tid; e < (kTile - 1) * kHalf; e += blockDim.x) {
        int p, q;
        round_pair(kTile, e / kHalf, e % kHalf, &p, &q);
        inner_p[e / kHalf][e % kHalf] = (unsigned char)p;
        inner_q[e / kHalf][e % kHalf] = (unsigned char)q;
    }
    __syncthreads();
    for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
        if (cta == 0 && tid == 0) a.ctl->rotations[(sweep + 1) % 3] = 0u;
        for (int r = 0; r < mb - 1; ++r) {
            // (1) one Jacobi sweep on each 32 x 32 subproblem
            for (int i = cta; i < pairs; i += ncta) {
                int P, Q;
                round_pair(mb, r, i, &P, &Q);
                for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                    const int l = e % kTile, c = e / kTile;
                    const int gl = sub_index(P, Q, l, n), gc = sub_index(P, Q, c, n);
                    sh.a[l][c] = (gl >= 0 && gc >= 0) ? ld(Ain + gl + (long long)gc * n) : 0.0;
                    sh.b[l][c] = l == c ? 1.0 : 0.0;
                }
                if (tid == 0) {
                    rapplied = 0;
                    roff = 0;
                }
                __syncthreads();
                // a subproblem that is already diagonal to the thresholds keeps W = I
                for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                    const int l = e % kTile, c = e / kTile;
                    if (l < c) {
                        const double v = fabs(sh.a[l][c]);
                        if (v > skip_abs && v > 1.0e-15 * sqrt(fabs(sh.a[l][l]) * fabs(sh.a[c][c]))) roff = 1;
                    }
                }
                __syncthreads();
                for (int ir = 0; ir < kTile - 1 && roff; ++ir) {
                    if (tid < kHalf) {
                        const int p = inner_p[ir][tid], q = inner_q[ir][tid];
                        double c = 1.0, sn = 0.0, t = 0.0;
                        if (sub_index(P, Q, p, n) >= 0 && sub_index(P, Q, q, n) >= 0) {
                            const double app = sh.a[p][p], aqq = sh.a[q][q], apq = sh.a[p][q];
                            const double aapq = fabs(apq);
                            if (aapq > skip_abs && aapq > 1.0e-15 * sqrt(fabs(app) * fabs(aqq))) {
                                // t = tan of the rotation angle, |t| <= 1 (the smaller root)
                                const double d = aqq - app;
                                const double two = 2.0 * apq;
                                const double den = fabs(d) + sqrt(fma(d, d, two * two));
                                t = (d >= 0.0 ? two : -two) / den;
                                c = rsqrt(fma(t, t, 1.0));
                                sn = t * c;
                                atomicAdd(&rapplied, 1);
                            }
                        }
                        rc[tid] = c;
                        rs[tid] = sn;
                        rt[tid] = t;
                    }
                    __syncthreads();
                    {
                        // 2 x 2 block (bi, bj) of the subproblem, one per thread
                        const int bi = tid % kHalf, bj = tid / kHalf;
                        const int pi = inner_p[ir][bi], qi = inner_q[ir][bi];
                        const int pj = inner_p[ir][bj], qj = inner_q[ir][bj];
                        const double ci = rc[bi], si = rs[bi], cj = rc[bj], sj = rs[bj];
                        if (bi == bj) {
                            if (si != 0.0) {
                                const double apq = sh.a[pi][qi], ti = rt[bi];
                                sh.a[pi][pi] -= ti * apq;
                                sh.a[qi][qi] += ti * apq;
                                sh.a[pi][qi] = 0.0;
                                sh.a[qi][pi] = 0.0;
                            }
                        } else if (si != 0.0 || sj != 0.0) {
                            const double b00 = sh.a[pi][pj], b01 = sh.a[pi][qj];
                            const double b10 = sh.a[qi][pj], b11 = sh.a[qi][qj];
                            const double x00 = cj * b00 - sj * b01, x01 = sj * b00 + cj * b01;
                            const double x10 = cj * b10 - sj * b11, x11 = sj * b10 + cj * b11;
                            sh.a[pi][pj] = ci * x00 - si * x10;
                            sh.a[pi][qj] = ci * x01 - si * x11;
                            sh.a[qi][pj] = si * x00 + ci * x10;
                            sh.a[qi][qj] = si * x01 + ci * x11;
                        }
                        // W <- W J: rows x, pair k (two per thread)
                        for (int u = tid; u < kTile * kHalf; u += blockDim.x) {
                            const int x = u % kTile, k = u / kTile;
                            const double sk = rs[k];
                            if (sk == 0.0) continue;
                            const int p = inner_p[ir][k], q = inner_q[ir][k];
                            const double ck = rc[k];
                            const double wp = sh.b[x][p], wq = sh.b[x][q];
                            sh.b[x][p] = ck * wp - sk * wq;
                            sh.b[x][q] = sk * wp + ck * wq;
                        }
                    }
                    __syncthreads();
                }
                for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                    const int l = e % kTile, c = e / kTile;
                    Wg[(long long)i * kTile * kTile + l + c * kTile] = sh.b[l][c];
                }
                if (tid == 0 && rapplied) atomicAdd(&a.ctl->rotations[sweep % 3], (unsigned)rapplied);
                __syncthreads();
            }
            if (!sync()) return false;
            // (2) apply: A' = W_i^T A W_j per pair combination, V <- V W
            const int chunks = (n + kTile - 1) / kTile;
            const int a_tasks = pairs * pairs;
            for (int task = cta; task < a_tasks + chunks * pairs; task += ncta) {
                const int l = tid & 31, cq = tid >> 5;
                if (task < a_tasks) {
                    const int i = task % pairs, j = task / pairs;
                    int Pi, Qi, Pj, Qj;
                    round_pair(mb, r, i, &Pi, &Qi);
                    round_pair(mb, r, j, &Pj, &Qj);
                    for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                        const int x = e % kTile, c = e / kTile;
                        const int gx = sub_index(Pi, Qi, x, n), gc = sub_index(Pj, Qj, c, n);
                        sh.a[x][c] = (gx >= 0 && gc >= 0) ? ld(Ain + gx + (long long)gc * n) : 0.0;
                        sh.b[x][c] = ld(Wg + (long long)i * kTile * kTile + x + c * kTile);
                    }
                    __syncthreads();
                    double y[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
                    for (int k = 0; k < kTile; ++k) {
                        const double w = sh.b[k][l];
#pragma unroll
                        for (int q = 0; q < 4; ++q) y[q] = fma(w, sh.a[k][cq + 8 * q], y[q]);
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) sh.d[l][cq + 8 * q] = y[q];
                    __syncthreads();
                    for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                        const int x = e % kTile, c = e / kTile;
                        sh.a[x][c] = ld(Wg + (long long)j * kTile * kTile + x + c * kTile);
                    }
                    __syncthreads();
                    double z[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
                    for (int k = 0; k < kTile; ++k) {
                        const double yv = sh.d[l][k];
#pragma unroll
                        for (int q = 0; q < 4; ++q) z[q] = fma(yv, sh.a[k][cq + 8 * q], z[q]);
                    }
                    const int gl = sub_index(Pi, Qi, l, n);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int gc = sub_index(Pj, Qj, cq + 8 * q, n);
                        if (gl >= 0 && gc >= 0) Aout[gl + (long long)gc * n] = z[q];
                    }
                } else {
                    const int v = task - a_tasks;
                    const int chunk = v % chunks, j = v / chunks;
                    int Pj, Qj;
                    round_pair(mb, r, j, &Pj, &Qj);
                    for (int e = tid; e < kTile * kTile; e += blockDim.x) {
                        const int x = e % kTile, c = e / kTile;
                        const int gx = chunk * kTile + x, gc = sub_index(Pj, Qj, c, n);
                        sh.a[x][c] = (gx < n && gc >= 0) ? ld(a.V + gx + (long long)gc * n) : 0.0;
                        sh.b[x][c] = ld(Wg + (long long)j * kTile * kTile + x + c * kTile);
                    }
                    __syncthreads();
                    double z[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
                    for (int k = 0; k < kTile; ++k) {
                        const double xv = sh.a[l][k];
#pragma unroll
                        for (int q = 0; q < 4; ++q) z[q] = fma(xv, sh.b[k][cq + 8 * q], z[q]);
                    }
                    const int gx = chunk * kTile + l;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int gc = sub_index(Pj, Qj, cq + 8 * q, n);
                        if (gx < n && gc >= 0) a.V[gx + (long long)gc * n] = z[q];
                    }
                }
                __syncthreads();
            }
            double* tmp = Ain;
            Ain = Aout;
            Aout = tmp;
            if (!sync()) return false;
        }
        const unsigned count = *(volatile unsigned*)&a.ctl->rotations[sweep % 3];
        if (cta == 0 && tid == 0) a.ctl->sweeps = sweep + 1;
        if (count == 0u) break;
    }
    *A_final = Ain;
    return true;
}

template <class Sync>
__device__ void eigh_body(const EighArgs& a, const Sync& sync, Shared& sh, int cta, int ncta) {
    const int n = a.n;
    const int tid = threadIdx.x;
    const long long gtid = (long long)cta * blockDim.x + tid, gstride = (long long)ncta * blockDim.x;
    if (!cholesky(a, sync, sh, cta, ncta)) return;
    if (a.mode == 0) return;
    if (!triangular_inverse(a, sync, sh, cta, ncta)) return;
    if (a.mode == 2) return;
    // T = H Ui (H symmetric from its upper triangle; Ui upper)
    const double* H = a.H;
    const double* Ui = a.Ui;
    gemm_tiles(
        n, [&](int r, int k) { return upper_elem(H, n, r, k); },
        [&](int k, int c) { return k <= c ? ld(Ui + k + (long long)c * n) : 0.0; }, a.T, sh, cta, ncta);
    if (!sync()) return;
    // A1 = Ui^T T
    const double* T = a.T;
    gemm_tiles(
        n, [&](int r, int k) { return k <= r ? ld(Ui + k + (long long)r * n) : 0.0; },
        [&](int k, int c) { return ld(T + k + (long long)c * n); }, a.A1, sh, cta, ncta);
    if (!sync()) return;
    // A0 = (A1 + A1^T) / 2, V = I, Frobenius norm
    double part = 0.0;
    for (long long e = gtid; e < (long long)n * n; e += gstride) {
        const int r = (int)(e % n), c = (int)(e / n);
        const double v = 0.5 * (ld(a.A1 + e) + ld(a.A1 + c + (long long)r * n));
        a.A0[e] = v;
        part = fma(v, v, part);
        if (r == c) a.V[e] = 1.0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((tid & 31) == 0) atomicAdd(&a.ctl->fro2, part);
    if (!sync()) return;
    double* A = nullptr;
    if (!jacobi(a, sync, sh, cta, ncta, &A)) return;
    // C = Ui V
    const double* V = a.V;
    gemm_tiles(
        n, [&](int r, int k) { return r <= k ? ld(Ui + r + (long long)k * n) : 0.0; },
        [&](int k, int c) { return ld(V + k + (long long)c * n); }, a.T, sh, cta, ncta);
    // ascending order (stable for ties)
    for (long long i = gtid; i < n; i += gstride) {
        const double li = ld(A + i + i * (long long)n);
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double lj = ld(A + j + (long long)j * n);
            rank += (lj < li || (lj == li && j < i)) ? 1 : 0;
        }
        a.rank[i] = rank;
        a.evals[rank] = li;
    }
    if (!sync()) return;
    for (long long e = gtid; e < (long long)n * n; e += gstride) {
        const int r = (int)(e % n), c = (int)(e / n);
        a.evecs[r + (long long)__ldcg(a.rank + c) * n] = ld(a.T + e);
    }
}

// Small generalized eigenproblems (n <= kTinyProblem, the structure problems of small active
// spaces): one warp, everything in shared memory.  Cholesky S = U^T U (lane j owns column j),
// U^-1, A = U^-T H U^-1, cyclic Jacobi on A with the rotations accumulated in V (lane i updates
// row/column i of each rotation), then eigenvalues ascending and C = U^-1 V.  Same outputs and
// info semantics as the cooperative kernel (ctl->info = order of the first non-positive leading
// minor of S, ctl->sweeps).
constexpr int kTinyProblem = 32;

__global__ void __launch_bounds__(32) eigh_tiny_kernel(EighArgs a) {
    __shared__ double sU[kTinyProblem][kTinyProblem + 1];   // S, then U (upper), then U^-1
    __shared__ double sA[kTinyProblem][kTinyProblem + 1];   // H, then A
    __shared__ double sV[kTinyProblem][kTinyProblem + 1];
    __shared__ double sT[kTinyProblem][kTinyProblem + 1];
    __shared__ double sw[kTinyProblem];
    __shared__ int sorder[kTinyProblem];
    const int n = a.n, lane = threadIdx.x;
    for (int e = lane; e < n * n; e += 32) {
        const int r = e % n, c = e / n;
        sU[r][c] = r <= c ? a.S[e] : a.S[c + (long long)r * n];
        sA[r][c] = r <= c ? a.H[e] : a.H[c + (long long)r * n];
        sV[r][c] = r == c ? 1.0 : 0.0;
    }
    __syncwarp();
    // Cholesky, right-looking on the upper triangle
    for (int k = 0; k < n; ++k) {
        const double d = sU[k][k];
        if (!(d > 0.0) || !isfinite(d)) {
            if (lane == 0) a.ctl->info = k + 1;
            return;
        }
        const double u = sqrt(d);
        __syncwarp();
        if (lane == k) sU[k][k] = u;
        if (lane > k && lane < n) sU[k][lane] /= u;
        __syncwarp();
        if (lane > k && lane < n)
            for (int i = k + 1; i <= lane; ++i) sU[i][lane] = fma(-sU[k][i], sU[k][lane], sU[i][lane]);
        __syncwarp();
    }
    for (int e = lane; e < n * n; e += 32) {
        const int r = e % n, c = e / n;
        if (r > c) sU[r][c] = 0.0;
    }
    __syncwarp();
    // U^-1 by columns (lane j: column j, back substitution), into sT then back to sU
    if (lane < n) {
        const int j = lane;
        for (int i = n - 1; i >= 0; --i) {
            double x = i == j ? 1.0 : 0.0;
            for (int k = i + 1; k <= j; ++k) x = fma(-sU[i][k], sT[k][j], x);
            sT[i][j] = i <= j ? x / sU[i][i] : 0.0;
        }
    }
    __syncwarp();
    for (int e = lane; e < n * n; e += 32) sU[e % n][e / n] = sT[e % n][e / n];
    __syncwarp();
    // A = U^-T H U^-1 (T = H U^-1, then U^-T T), lane j: column j
    if (lane < n) {
        const int j = lane;
        for (int i = 0; i < n; ++i) {
            double x = 0.0;
            for (int k = 0; k <= j; ++k) x = fma(sA[i][k], sU[k][j], x);
            sT[i][j] = x;
        }
    }
    __syncwarp();
    if (lane < n) {
        const int j = lane;
        for (int i = 0; i < n; ++i) {
            double x = 0.0;
            for (int k = 0; k <= i; ++k) x = fma(sU[k][i], sT[k][j], x);
            sV[i][j] = x;  // A in sV for now
        }
    }
    __syncwarp();
    for (int e = lane; e < n * n; e += 32) {
        const int r = e % n, c = e / n;
        sA[r][c] = 0.5 * (sV[r][c] + sV[c][r]);
    }
    __syncwarp();
    for (int e = lane; e < n * n; e += 32) sV[e % n][e / n] = (e % n) == (e / n) ? 1.0 : 0.0;
    __syncwarp();
    // cyclic Jacobi
    // (an off-diagonal entry below eps sqrt|a_pp a_qq|, or below 1e-17 ||A||_F, is set to zero
    // instead of rotated; the iteration ends after a sweep without rotations)
    double fro = 0.0;
    for (int e = lane; e < n * n; e += 32) fro = fma(sA[e % n][e / n], sA[e % n][e / n], fro);
    for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, o);
    const double floor_abs = 1.0e-17 * sqrt(fro);
    int sweep = 0;
    for (; sweep < kMaxSweeps; ++sweep) {
        int rotations = 0;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = sA[p][q];
                const double app = sA[p][p], aqq = sA[q][q];
                if (fabs(apq) <= fmax(2.220446049250313e-16 * sqrt(fabs(app * aqq)), floor_abs)) {
                    __syncwarp();
                    if (lane == 0) sA[p][q] = sA[q][p] = 0.0;
                    __syncwarp();
                    continue;
                }
                ++rotations;
                const double tau = (aqq - app) / (2.0 * apq);
                const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double cs = 1.0 / sqrt(1.0 + t * t), sn = t * cs;
                __syncwarp();
                // columns p, q of A and V (lane i: row i)
                if (lane < n) {
                    const double aip = sA[lane][p], aiq = sA[lane][q];
                    sA[lane][p] = cs * aip - sn * aiq;
                    sA[lane][q] = sn * aip + cs * aiq;
                    const double vip = sV[lane][p], viq = sV[lane][q];
                    sV[lane][p] = cs * vip - sn * viq;
                    sV[lane][q] = sn * vip + cs * viq;
                }
                __syncwarp();
                // rows p, q of A (lane i: column i)
                if (lane < n) {
                    const double api = sA[p][lane], aqi = sA[q][lane];
                    sA[p][lane] = cs * api - sn * aqi;
                    sA[q][lane] = sn * api + cs * aqi;
                }
                __syncwarp();
            }
        if (rotations == 0) break;
    }
    if (lane == 0) a.ctl->sweeps = sweep;
    // eigenvalues ascending (rank by comparison, ties by index), C = U^-1 V
    if (lane < n) {
        const double li = sA[lane][lane];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double lj = sA[j][j];
            rank += (lj < li || (lj == li && j < lane)) ? 1 : 0;
        }
        sorder[rank] = lane;
        sw[rank] = li;
    }
    __syncwarp();
    if (lane < n) a.evals[lane] = sw[lane];
    for (int e = lane; e < n * n; e += 32) {
        const int r = e % n, c = e / n, src = sorder[c];
        double x = 0.0;
        for (int k = r; k < n; ++k) x = fma(sU[r][k], sV[k][src], x);
        a.evecs[r + (long long)c * n] = x;
    }
}

__global__ void __launch_bounds__(kThreads) eigh_grid_kernel(EighArgs a) {
    __shared__ Shared sh;
    GridSync sync{a.ctl, gridDim.x, a.spin_limit};
    eigh_body(a, sync, sh, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(kThreads) eigh_block_kernel(const EighArgs* __restrict__ args, int count) {
    __shared__ Shared sh;
    const int b = blockIdx.x;
    if (b >= count) return;
    const EighArgs a = args[b];
    BlockSync sync;
    eigh_body(a, sync, sh, 0, 1);
}

// Workspace of one problem (doubles / ints), all offsets 256-byte aligned.
struct Layout {
    size_t U, Ui, T, A0, A1, V, W, evals, evecs, H, S, rank, ctl, total;
};

size_t align_up(size_t x) { return (x + 255) / 256 * 256; }

Layout layout_for(int n, int mode, bool own_inputs, bool own_outputs) {
    Layout L{};
    const size_t m2 = sizeof(double) * (size_t)n * n;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off = align_up(off + bytes);
        return at;
    };
    L.U = take(m2);
    if (mode == 2) L.Ui = take(m2);
    if (mode == 1) {
        L.Ui = take(m2);
        L.T = take(m2);
        L.A0 = take(m2);
        L.A1 = take(m2);
        L.V = take(m2);
        const int nbk = (n + 15) / 16;
        L.W = take(sizeof(double) * 1024 * (size_t)((nbk + (nbk & 1)) / 2));
        L.rank = take(sizeof(int) * n);
        if (own_outputs) {
            L.evals = take(sizeof(double) * n);
            L.evecs = take(m2);
        }
        if (own_inputs) L.H = take(m2);
    }
    if (own_inputs) L.S = take(m2);
    L.ctl = take(sizeof(Control));
    L.total = off;
    return L;
}

// Bytes that must start at zero: Ui and V (mode 1) and the control block.
cudaError_t clear_workspace(unsigned char* base, const Layout& L, int n, int mode, cudaStream_t s) {
    const size_t m2 = sizeof(double) * (size_t)n * n;
    cudaError_t err = cudaMemsetAsync(base + L.ctl, 0, sizeof(Control), s);
    if (err == cudaSuccess && mode >= 1) err = cudaMemsetAsync(base + L.Ui, 0, m2, s);
    if (err == cudaSuccess && mode == 1) err = cudaMemsetAsync(base + L.V, 0, m2, s);
    return err;
}

EighArgs args_for(unsigned char* base, const Layout& L, int n, int mode, const double* H, const double* S,
                  double* evals, double* evecs, double* U_out) {
    EighArgs a{};
    a.n = n;
    a.mode = mode;
    a.H = H;
    a.S = S;
    a.U = U_out ? U_out : reinterpret_cast<double*>(base + L.U);
    if (mode == 2) a.Ui = reinterpret_cast<double*>(base + L.Ui);
    if (mode == 1) {
        a.Ui = reinterpret_cast<double*>(base + L.Ui);
        a.T = reinterpret_cast<double*>(base + L.T);
        a.A0 = reinterpret_cast<double*>(base + L.A0);
        a.A1 = reinterpret_cast<double*>(base + L.A1);
        a.V = reinterpret_cast<double*>(base + L.V);
        a.W = reinterpret_cast<double*>(base + L.W);
        a.rank = reinterpret_cast<int*>(base + L.rank);
        a.evals = evals;
        a.evecs = evecs;
    }
    a.ctl = reinterpret_cast<Control*>(base + L.ctl);
    a.spin_limit = kBarrierSpinLimit;
    return a;
}

// Multi-CTA cooperative launches are serialized across the process (they are held from launch
// to completion by the callers below): the grid barrier needs every CTA resident, and two
// grid-wide solves from different host threads must not compete for residency.
std::mutex g_cooperative;

cudaError_t launch_single(const EighArgs& a, cudaStream_t s, int* grid_out) {
    if (a.mode == 1 && a.n <= kTinyProblem) {
        *grid_out = 1;
        eigh_tiny_kernel<<<1, 32, 0, s>>>(a);
        return cudaGetLastError();
    }
    if (a.n <= kSmallProblem) {
        // one CTA: the grid barrier of a one-block launch never waits
        void* params[] = {const_cast<EighArgs*>(&a)};
        *grid_out = 1;
        return cudaLaunchCooperativeKernel((const void*)eigh_grid_kernel, dim3(1), dim3(kThreads), params, 0, s);
    }
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err == cudaSuccess) err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eigh_grid_kernel, kThreads, 0);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    const int grid = sms;  // one CTA per SM
    *grid_out = grid;
    void* params[] = {const_cast<EighArgs*>(&a)};
    return cudaLaunchCooperativeKernel((const void*)eigh_grid_kernel, dim3(grid), dim3(kThreads), params, 0, s);
}

}  // namespace
}  // namespace vbcore

using namespace vbcore;

namespace {

// Cholesky factor of a matrix above the one-CTA size: blocked panels, no grid barrier.
vb_status run_blocked_cholesky(vb_context* ctx, const double* S, int n, bool host, double* U_out, int* info,
                               const char* name) {
    cudaStream_t s = ctx->stream;
    const size_t m2 = sizeof(double) * (size_t)n * n;
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, (host ? 2 * m2 : 0) + blocked_cholesky_workspace(n, false));
    if (st != VB_OK) return st;
    unsigned char* base = static_cast<unsigned char*>(ws.ptr);
    const double* dS = S;
    double* dU = U_out;
    cudaError_t err = cudaSuccess;
    if (host) {
        err = cudaMemcpyAsync(base, S, m2, cudaMemcpyHostToDevice, s);
        dS = reinterpret_cast<const double*>(base);
        dU = reinterpret_cast<double*>(base + m2);
    }
    int bad = 0;
    if (err == cudaSuccess) err = blocked_cholesky(dS, n, dU, nullptr, base + (host ? 2 * m2 : 0), &bad, s);
    if (err == cudaSuccess && host && !bad) {
        err = cudaMemcpyAsync(U_out, dU, m2, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    }
    if (err != cudaSuccess) return cuda_error(ctx, err, name);
    if (bad) {
        if (info) *info = bad;
        return set_error(ctx, VB_ERR_NUMERIC,
                         std::string(name) + ": matrix is not positive definite (leading minor " +
                             std::to_string(bad) + ")");
    }
    return VB_OK;
}

vb_status run_single(vb_context* ctx, int mode, const double* H, const double* S, int n, int mem, double* evals,
                     double* evecs, double* U_out, int* info, const char* name) {
    if (!ctx) return VB_ERR_INVALID;
    if (info) *info = 0;
    if (n < 1 || !S || (mode == 1 && (!H || !evals || !evecs)) || (mode == 0 && !U_out))
        return set_error(ctx, VB_ERR_INVALID, std::string(name) + ": dimension must be positive and pointers non-null");
    if (mem != VB_MEM_HOST && mem != VB_MEM_DEVICE) return set_error(ctx, VB_ERR_INVALID, "bad memory space");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const bool host = mem == VB_MEM_HOST;
    if (mode == 0 && n > kSmallProblem) return run_blocked_cholesky(ctx, S, n, host, U_out, info, name);
    const Layout L = layout_for(n, mode, host, host);
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, L.total);
    if (st != VB_OK) return st;
    unsigned char* base = static_cast<unsigned char*>(ws.ptr);
    const size_t m2 = sizeof(double) * (size_t)n * n;
    cudaError_t err = cudaSuccess;
    const double* dS = S;
    const double* dH = H;
    double* dvals = evals;
    double* dvecs = evecs;
    double* dU = U_out;
    if (host) {
        err = cudaMemcpyAsync(base + L.S, S, m2, cudaMemcpyHostToDevice, s);
        dS = reinterpret_cast<double*>(base + L.S);
        if (mode == 1) {
            if (err == cudaSuccess) err = cudaMemcpyAsync(base + L.H, H, m2, cudaMemcpyHostToDevice, s);
            dH = reinterpret_cast<double*>(base + L.H);
            dvals = reinterpret_cast<double*>(base + L.evals);
            dvecs = reinterpret_cast<double*>(base + L.evecs);
        }
        dU = nullptr;
    }
    if (err == cudaSuccess) err = clear_workspace(base, L, n, mode, s);
    if (err != cudaSuccess) return cuda_error(ctx, err, name);
    EighArgs a = args_for(base, L, n, mode, dH, dS, dvals, dvecs, mode == 0 ? dU : nullptr);
    if (ctx->barrier_spin_limit > 0) a.spin_limit = ctx->barrier_spin_limit;
    int grid = 0;
    std::unique_lock<std::mutex> coop(g_cooperative, std::defer_lock);
    if (n > kSmallProblem) coop.lock();
    err = launch_single(a, s, &grid);
    if (err != cudaSuccess) return cuda_error(ctx, err, name);
    Control c{};
    err = cudaMemcpyAsync(&c, base + L.ctl, sizeof(Control), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess && host) {
        if (mode == 0)
            err = cudaMemcpyAsync(U_out, base + L.U, m2, cudaMemcpyDeviceToHost, s);
        else {
            err = cudaMemcpyAsync(evals, dvals, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
            if (err == cudaSuccess) err = cudaMemcpyAsync(evecs, dvecs, m2, cudaMemcpyDeviceToHost, s);
        }
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, name);
    if (c.err) return set_error(ctx, VB_ERR_TIMEOUT, std::string(name) + ": grid barrier timed out");
    if (c.info) {
        if (info) *info = mode == 1 ? n + c.info : c.info;
        return set_error(ctx, VB_ERR_NUMERIC,
                         mode == 1 ? std::string(name) + ": overlap_matrix is not positive definite (info=" +
                                         std::to_string(n + c.info) + ")"
                                   : std::string(name) + ": matrix is not positive definite (leading minor " +
                                         std::to_string(c.info) + ")");
    }
    if (mode == 1 && c.sweeps >= kMaxSweeps)
        return set_error(ctx, VB_ERR_NUMERIC, std::string(name) + ": Jacobi iteration did not converge");
    return VB_OK;
}

}  // namespace

namespace vbcore {

// U^-1 of the Cholesky factor of a device matrix (upper triangles read); *info = order of the
// first non-positive leading minor (0 on success).  Synchronizes the context stream.
vb_status factor_inverse_device(vb_context* ctx, const double* M, int n, double* Ui_out, int* info) {
    *info = 0;
    cudaStream_t s = ctx->stream;
    if (n > kSmallProblem) {
        // stream-ordered panels and tensor-core products, no grid barrier
        DeviceBuffer ws;
        const size_t u_bytes = sizeof(double) * (size_t)n * n;
        vb_status st = ws.allocate(ctx, u_bytes + blocked_cholesky_workspace(n, true));
        if (st != VB_OK) return st;
        unsigned char* base = static_cast<unsigned char*>(ws.ptr);
        const cudaError_t err =
            blocked_cholesky(M, n, reinterpret_cast<double*>(base), Ui_out, base + u_bytes, info, s);
        if (err != cudaSuccess) return cuda_error(ctx, err, "factor_inverse_device");
        return VB_OK;
    }
    const Layout L = layout_for(n, 2, false, false);
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, L.total);
    if (st != VB_OK) return st;
    unsigned char* base = static_cast<unsigned char*>(ws.ptr);
    cudaError_t err = clear_workspace(base, L, n, 2, s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "factor_inverse_device");
    EighArgs a = args_for(base, L, n, 2, nullptr, M, nullptr, nullptr, nullptr);
    if (ctx->barrier_spin_limit > 0) a.spin_limit = ctx->barrier_spin_limit;
    int grid = 0;
    std::unique_lock<std::mutex> coop(g_cooperative, std::defer_lock);
    if (n > kSmallProblem) coop.lock();
    err = launch_single(a, s, &grid);
    Control c{};
    if (err == cudaSuccess) err = cudaMemcpyAsync(&c, base + L.ctl, sizeof(Control), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(Ui_out, base + L.Ui, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "factor_inverse_device");
    if (c.err) return set_error(ctx, VB_ERR_TIMEOUT, "factor_inverse_device: grid barrier timed out");
    *info = c.info;
    return VB_OK;
}

}  // namespace vbcore

extern "C" {

vb_status vb_metric_cholesky(vb_context* ctx, const double* S, int n, int mem_space, double* upper_out, int* info) {
    return run_single(ctx, 0, nullptr, S, n, mem_space, nullptr, nullptr, upper_out, info, "vb_metric_cholesky");
}

vb_status vb_generalized_eigh(vb_context* ctx, const double* H, const double* S, int n, int mem_space,
                              double* eigenvalues, double* eigenvectors, int* info) {
    return run_single(ctx, 1, H, S, n, mem_space, eigenvalues, eigenvectors, nullptr, info, "vb_generalized_eigh");
}

vb_status vb_generalized_eigh_batched(vb_context* ctx, int count, const int* dims, const int64_t* offsets,
                                      const double* H, const double* S, int mem_space, double* eigenvalues,
                                      const int64_t* value_offsets, double* eigenvectors, int* info) {
    if (!ctx) return VB_ERR_INVALID;
    if (count < 0 || (count > 0 && (!dims || !offsets || !H || !S || !eigenvalues || !value_offsets ||
                                    !eigenvectors || !info)))
        return set_error(ctx, VB_ERR_INVALID, "vb_generalized_eigh_batched: bad arguments");
    if (mem_space != VB_MEM_DEVICE)
        return set_error(ctx, VB_ERR_INVALID, "vb_generalized_eigh_batched: device pointers only");
    if (count == 0) return VB_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    std::vector<Layout> layouts(count);
    std::vector<size_t> base_off(count);
    size_t total = 0;
    for (int b = 0; b < count; ++b) {
        if (dims[b] < 1) return set_error(ctx, VB_ERR_INVALID, "vb_generalized_eigh_batched: dimension must be positive");
        layouts[b] = layout_for(dims[b], 1, false, false);
        base_off[b] = total;
        total += layouts[b].total;
    }
    const size_t args_off = total;
    total = align_up(total + sizeof(EighArgs) * count);
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, total);
    if (st != VB_OK) return st;
    unsigned char* base = static_cast<unsigned char*>(ws.ptr);
    std::vector<EighArgs> args(count);
    cudaError_t err = cudaSuccess;
    for (int b = 0; b < count && err == cudaSuccess; ++b) {
        unsigned char* pb = base + base_off[b];
        err = clear_workspace(pb, layouts[b], dims[b], 1, s);
        args[b] = args_for(pb, layouts[b], dims[b], 1, H + offsets[b], S + offsets[b], eigenvalues + value_offsets[b],
                           eigenvectors + offsets[b], nullptr);
    }
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(base + args_off, args.data(), sizeof(EighArgs) * count, cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess) {
        eigh_block_kernel<<<count, kThreads, 0, s>>>(reinterpret_cast<const EighArgs*>(base + args_off), count);
        err = cudaGetLastError();
    }
    std::vector<Control> ctl(count);
    for (int b = 0; b < count && err == cudaSuccess; ++b)
        err = cudaMemcpyAsync(&ctl[b], base + base_off[b] + layouts[b].ctl, sizeof(Control), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "vb_generalized_eigh_batched");
    vb_status result = VB_OK;
    for (int b = 0; b < count; ++b) {
        info[b] = ctl[b].info ? dims[b] + ctl[b].info : (ctl[b].sweeps >= kMaxSweeps ? -1 : 0);
        if (info[b] != 0 && result == VB_OK)
            result = set_error(ctx, VB_ERR_NUMERIC,
                               "vb_generalized_eigh_batched: problem " + std::to_string(b) +
                                   (ctl[b].info ? " has an overlap matrix that is not positive definite"
                                                : " did not converge"));
    }
    return result;
}

}  // extern "C"
