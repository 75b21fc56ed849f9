// Lowest root of the dense structure problem H c = E S c by a generalized Davidson iteration
// on the device (the selected-root path of solve_structure_problem,
// src/vbscf/derivatives/gradient/active_space/evaluator.cpp:466-560, and
// GeneralizedEigensolver::solve_davidson, src/linalg/eigensolver.hpp:194-198, here on the
// materialized H and S).  For structure spaces too large for the dense all-root solver.
//
// Per iteration: one fused pass over H and S computes H t and S t for the newest basis vector
// (the HBM-bound step: 16 n^2 bytes), the projected problem (dimension <= kMaxSubspace) is
// solved on the host in FP64 by Cholesky + cyclic Jacobi, the Ritz vector and residual
// r = H x - theta S x are formed on the device, and the correction t = r / (theta S_ii - H_ii)
// is S-orthogonalized against the basis twice.  A full basis restarts from its 12 lowest Ritz
// vectors (thick restart).  Converged when ||r||_2 <= tol (||H x|| + |theta| ||S x||) (a
// backward-error criterion, attainable whatever the conditioning of S).  The diagonal
// preconditioner is weak on strongly coupled structure matrices, so after 24 iterations the
// Ritz value seeds a shift sigma below the lowest root (lowered until H - sigma S = U^T U is
// positive definite) and the correction becomes t = U^-1 U^-T r: the basis then grows along
// the Krylov space of the shift-inverted operator, whose lowest root is well separated.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "internal.h"

namespace vbcore {
namespace {

constexpr int kMaxSubspace = 48;
constexpr int kKeep = 12;  // Ritz vectors kept at a restart
constexpr int kDiagonalPhase = 24;  // iterations with the diagonal preconditioner
constexpr int kSplits = 64;  // column ranges of the matrix-vector partial sums (parallelism for the HBM stream)

// y_h = H x, y_s = S x (column-major n x n), partial sums over kSplits column ranges.
__global__ void __launch_bounds__(256) gemv2_partial_kernel(const double* __restrict__ H, const double* __restrict__ S,
                                                            int n, const double* __restrict__ x,
                                                            double* __restrict__ part_h, double* __restrict__ part_s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int split = blockIdx.y;
    const int chunk = (n + kSplits - 1) / kSplits;
    const int j0 = split * chunk, j1 = min(n, j0 + chunk);
    if (i >= n) return;
    double ah = 0.0, as = 0.0;
    for (int j = j0; j < j1; ++j) {
        const double xj = __ldg(x + j);
        ah = fma(__ldg(H + i + (long long)j * n), xj, ah);
        as = fma(__ldg(S + i + (long long)j * n), xj, as);
    }
    part_h[(long long)split * n + i] = ah;
    part_s[(long long)split * n + i] = as;
}

__global__ void gemv2_reduce_kernel(int n, const double* __restrict__ part_h, const double* __restrict__ part_s,
                                    double* __restrict__ yh, double* __restrict__ ys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ah = 0.0, as = 0.0;
    for (int sp = 0; sp < kSplits; ++sp) {
        ah += part_h[(long long)sp * n + i];
        as += part_s[(long long)sp * n + i];
    }
    yh[i] = ah;
    ys[i] = as;
}

// out[b] = sum_i A[i + c n] * y[i] with c = b for blocks b < k and, when y2 is given, c = b - k and
// y2 in place of y for blocks k .. 2k - 1; y == nullptr: column c with itself.  One CTA per dot,
// fixed reduction order.
__global__ void __launch_bounds__(256) multi_dot_kernel(const double* __restrict__ A, int n, int k,
                                                        const double* __restrict__ y, const double* __restrict__ y2,
                                                        double* __restrict__ out) {
    __shared__ double red[256];
    const int b = blockIdx.x;
    const int c = b < k ? b : b - k;
    const double* a = A + (long long)c * n;
    const double* v = b < k ? y : y2;
    if (!v) v = a;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc = fma(a[i], v[i], acc);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = red[0];
}

// y[i] = sum_c A[i + c n] coef[c] (+ beta * y[i]); grid row b (blockIdx.y) applies the same
// coefficients to A + b a_step into y + b y_step (the basis and its two images in one launch)
__global__ void combine_kernel(const double* __restrict__ A, int n, int k, const double* __restrict__ coef,
                               double beta, double* __restrict__ y, long long a_step = 0, long long y_step = 0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    A += blockIdx.y * a_step;
    y += blockIdx.y * y_step;
    double acc = beta == 0.0 ? 0.0 : beta * y[i];
    for (int c = 0; c < k; ++c) acc = fma(A[i + (long long)c * n], coef[c], acc);
    y[i] = acc;
}

// t = r / (theta s_ii - h_ii) (guarded), r = Hx - theta Sx
__global__ void residual_kernel(int n, const double* __restrict__ hx, const double* __restrict__ sx, double theta,
                                const double* __restrict__ hd, const double* __restrict__ sd, double* __restrict__ r,
                                double* __restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ri = hx[i] - theta * sx[i];
    r[i] = ri;
    double den = theta * sd[i] - hd[i];
    if (fabs(den) < 1.0e-8) den = den < 0.0 ? -1.0e-8 : 1.0e-8;
    t[i] = ri / den;
}

__global__ void diag_kernel(int n, const double* __restrict__ H, const double* __restrict__ S, double* hd, double* sd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    hd[i] = H[i + (long long)i * n];
    sd[i] = S[i + (long long)i * n];
}

// y = A^T x for upper-triangular A (one warp per column, coalesced down the column's rows <= col)
__global__ void __launch_bounds__(256) gemv_t_kernel(const double* __restrict__ A, int n, const double* __restrict__ x,
                                                     double* __restrict__ y) {
    const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (col >= n) return;
    const double* a = A + (long long)col * n;
    double acc = 0.0;
    for (int i = lane; i <= col; i += 32) acc = fma(__ldg(a + i), __ldg(x + i), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) y[col] = acc;
}

// y = A x for upper-triangular A, column-split partial sums (same scheme as gemv2; row i reads
// only its columns j >= i)
__global__ void __launch_bounds__(256) gemv_partial_kernel(const double* __restrict__ A, int n,
                                                           const double* __restrict__ x, double* __restrict__ part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int split = blockIdx.y;
    const int chunk = (n + kSplits - 1) / kSplits;
    const int j0 = split * chunk, j1 = min(n, j0 + chunk);
    if (i >= n) return;
    double acc = 0.0;
    for (int j = max(j0, i); j < j1; ++j) acc = fma(__ldg(A + i + (long long)j * n), __ldg(x + j), acc);
    part[(long long)split * n + i] = acc;
}

__global__ void reduce_splits_kernel(int n, const double* __restrict__ part, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0.0;
    for (int sp = 0; sp < kSplits; ++sp) acc += part[(long long)sp * n + i];
    y[i] = acc;
}

// M = H - sigma S
__global__ void shift_kernel(long long count, const double* __restrict__ H, const double* __restrict__ S, double sigma,
                             double* __restrict__ M) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count; e += (long long)gridDim.x * blockDim.x)
        M[e] = H[e] - sigma * S[e];
}

__global__ void scale_copy_kernel(int n, const double* __restrict__ x, double s, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = s * x[i];
}

// Small symmetric-definite problem on the host: A y = theta B y (k x k), all roots ascending.
bool small_eigs(int k, const std::vector<double>& A, const std::vector<double>& B, std::vector<double>* theta,
                std::vector<double>* y) {
    // B = L L^T
    std::vector<double> L(k * k, 0.0);
    for (int j = 0; j < k; ++j) {
        double d = B[j + j * k];
        for (int p = 0; p < j; ++p) d -= L[j + p * k] * L[j + p * k];
        if (!(d > 0.0)) return false;
        L[j + j * k] = std::sqrt(d);
        for (int i = j + 1; i < k; ++i) {
            double v = B[i + j * k];
            for (int p = 0; p < j; ++p) v -= L[i + p * k] * L[j + p * k];
            L[i + j * k] = v / L[j + j * k];
        }
    }
    // M = L^-1 A L^-T
    std::vector<double> Li(k * k, 0.0);
    for (int c = 0; c < k; ++c)
        for (int i = 0; i < k; ++i) {
            double v = i == c ? 1.0 : 0.0;
            for (int p = 0; p < i; ++p) v -= L[i + p * k] * Li[p + c * k];
            Li[i + c * k] = v / L[i + i * k];
        }
    std::vector<double> T(k * k, 0.0), M(k * k, 0.0);
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) {
            double v = 0.0;
            for (int p = 0; p < k; ++p) v += A[i + p * k] * Li[j + p * k];
            T[i + j * k] = v;
        }
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) {
            double v = 0.0;
            for (int p = 0; p < k; ++p) v += Li[i + p * k] * T[p + j * k];
            M[i + j * k] = v;
        }
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < i; ++j) M[i + j * k] = M[j + i * k] = 0.5 * (M[i + j * k] + M[j + i * k]);
    // cyclic Jacobi
    std::vector<double> V(k * k, 0.0);
    for (int i = 0; i < k; ++i) V[i + i * k] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) (i == j ? tot : off) += M[i + j * k] * M[i + j * k];
        if (off <= 1e-26 * (tot + off) || off == 0.0) break;
        for (int p = 0; p < k; ++p)
            for (int q = p + 1; q < k; ++q) {
                const double apq = M[p + q * k];
                if (apq == 0.0) continue;
                const double tau = (M[q + q * k] - M[p + p * k]) / (2.0 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::hypot(1.0, tau));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
                for (int r = 0; r < k; ++r) {
                    const double mp = M[r + p * k], mq = M[r + q * k];
                    M[r + p * k] = c * mp - s * mq;
                    M[r + q * k] = s * mp + c * mq;
                }
                for (int r = 0; r < k; ++r) {
                    const double mp = M[p + r * k], mq = M[q + r * k];
                    M[p + r * k] = c * mp - s * mq;
                    M[q + r * k] = s * mp + c * mq;
                }
                for (int r = 0; r < k; ++r) {
                    const double vp = V[r + p * k], vq = V[r + q * k];
                    V[r + p * k] = c * vp - s * vq;
                    V[r + q * k] = s * vp + c * vq;
                }
            }
    }
    std::vector<int> order(k);
    for (int i = 0; i < k; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return M[a + a * k] < M[b + b * k]; });
    theta->resize(k);
    y->assign((size_t)k * k, 0.0);
    // column j of Y = L^-T v_(j-th lowest): B-orthonormal Ritz coefficient vectors
    for (int j = 0; j < k; ++j) {
        const int src = order[j];
        (*theta)[j] = M[src + src * k];
        for (int i = 0; i < k; ++i) {
            double v = 0.0;
            for (int p = 0; p < k; ++p) v += Li[p + i * k] * V[p + src * k];
            (*y)[i + (size_t)j * k] = v;
        }
    }
    return true;
}

}  // namespace
}  // namespace vbcore

using namespace vbcore;

extern "C" vb_status vb_lowest_root(vb_context* ctx, const double* H, const double* S, int n, int mem_space,
                                    double tolerance, int max_iterations, double* eigenvalue, double* eigenvector,
                                    int* iterations) {
    if (!ctx) return VB_ERR_INVALID;
    if (n < 1 || !H || !S || !eigenvalue || !eigenvector)
        return set_error(ctx, VB_ERR_INVALID, "vb_lowest_root: bad arguments");
    if (mem_space != VB_MEM_HOST && mem_space != VB_MEM_DEVICE) return set_error(ctx, VB_ERR_INVALID, "bad memory space");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t m2 = sizeof(double) * (size_t)n * n, v1 = sizeof(double) * n;
    const bool host = mem_space == VB_MEM_HOST;
    const int kmax = std::min(kMaxSubspace, n);
    // workspace: [H S (host mode)] V HV SV (n x kmax) parts (2 x splits x n) vectors (8 n) coef
    const size_t ws_doubles = (host ? 2 * (size_t)n * n : 0) + 3 * (size_t)n * kmax + 2 * (size_t)kSplits * n +
                              8 * (size_t)n + 3 * kMaxSubspace + 3 * (size_t)kKeep * n;
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, sizeof(double) * ws_doubles);
    if (st != VB_OK) return st;
    double* base = ws.as<double>();
    const double* dH = H;
    const double* dS = S;
    cudaError_t err = cudaSuccess;
    if (host) {
        err = cudaMemcpyAsync(base, H, m2, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(base + (size_t)n * n, S, m2, cudaMemcpyHostToDevice, s);
        dH = base;
        dS = base + (size_t)n * n;
        base += 2 * (size_t)n * n;
    }
    double* V = base;
    double* HV = V + (size_t)n * kmax;
    double* SV = HV + (size_t)n * kmax;
    double* ph = SV + (size_t)n * kmax;
    double* ps = ph + (size_t)kSplits * n;
    double* hd = ps + (size_t)kSplits * n;
    double* sd = hd + n;
    double* x = sd + n;
    double* hx = x + n;
    double* sx = hx + n;
    double* r = sx + n;
    double* t = r + n;
    double* st_vec = t + n;
    double* coef = st_vec + n;
    double* dots = coef + kMaxSubspace;
    double* restart = dots + 2 * kMaxSubspace;  // 3 kKeep columns (dots: up to 2 kMaxSubspace)
    const int tb = 256, nb = (n + tb - 1) / tb;
    auto check = [&](const char* what) -> vb_status {
        if (err == cudaSuccess) err = cudaGetLastError();
        if (err != cudaSuccess) return cuda_error(ctx, err, what);
        return VB_OK;
    };
    auto gemv2 = [&](const double* in, double* yh, double* ys) {
        gemv2_partial_kernel<<<dim3(nb, kSplits), tb, 0, s>>>(dH, dS, n, in, ph, ps);
        gemv2_reduce_kernel<<<nb, tb, 0, s>>>(n, ph, ps, yh, ys);
    };
    // dots of the k columns of A with y (and, when y2 is given, then with y2; y == nullptr: each
    // column with itself), read back in one synchronization
    auto dots_of = [&](const double* A, int k, const double* y, std::vector<double>* out,
                       const double* y2 = nullptr) {
        const int m = y2 ? 2 * k : k;
        multi_dot_kernel<<<m, 256, 0, s>>>(A, n, k, y, y2, dots);
        out->resize(m);
        err = cudaMemcpyAsync(out->data(), dots, sizeof(double) * m, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    };
    diag_kernel<<<nb, tb, 0, s>>>(n, dH, dS, hd, sd);
    std::vector<double> hdh(n), sdh(n);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hdh.data(), hd, v1, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(sdh.data(), sd, v1, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if ((st = check("vb_lowest_root")) != VB_OK) return st;
    int start = 0;
    for (int i = 1; i < n; ++i)
        if (hdh[i] / sdh[i] < hdh[start] / sdh[start]) start = i;
    // v0 = e_start / sqrt(S_ss)
    std::vector<double> e0(n, 0.0);
    e0[start] = 1.0 / std::sqrt(sdh[start]);
    err = cudaMemcpyAsync(V, e0.data(), v1, cudaMemcpyHostToDevice, s);
    int k = 1;
    std::vector<double> Hs(kmax * kmax, 0.0), Ss(kmax * kmax, 0.0);
    double theta = 0.0;
    std::vector<double> y;
    double scale = 1.0;
    int it = 0;
    std::vector<double> ritz;  // lowest Ritz value of every iteration
    bool converged = false;
    // projected matrices are kept with the basis; column c is new (its H v and S v are computed
    // here unless the caller already stored them in HV and SV)
    auto add_column = [&](int c, bool have_images) -> vb_status {
        if (!have_images) gemv2(V + (size_t)c * n, HV + (size_t)c * n, SV + (size_t)c * n);
        std::vector<double> cols;
        dots_of(V, c + 1, HV + (size_t)c * n, &cols, SV + (size_t)c * n);
        if ((st = check("vb_lowest_root")) != VB_OK) return st;
        for (int i = 0; i <= c; ++i) {
            Hs[i + c * kmax] = Hs[c + i * kmax] = cols[i];
            Ss[i + c * kmax] = Ss[c + i * kmax] = cols[c + 1 + i];
        }
        return VB_OK;
    };
    if ((st = add_column(0, false)) != VB_OK) return st;
    DeviceBuffer mbuf, uibuf;
    double* Ui = nullptr;
    for (it = 0; it < max_iterations; ++it) {
        std::vector<double> A(k * k), Bm(k * k);
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) {
                A[i + j * k] = Hs[i + j * kmax];
                Bm[i + j * k] = Ss[i + j * kmax];
            }
        std::vector<double> thetas, Y;
        if (!small_eigs(k, A, Bm, &thetas, &Y))
            return set_error(ctx, VB_ERR_NUMERIC, "vb_lowest_root: projected overlap is not positive definite");
        theta = thetas[0];
        ritz.push_back(theta);
        y.assign(Y.begin(), Y.begin() + k);
        scale = std::max(1.0, std::fabs(theta));
        err = cudaMemcpyAsync(coef, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s);
        // x, hx, sx (consecutive vectors) from V, HV, SV (consecutive n x kmax blocks)
        combine_kernel<<<dim3(nb, 3), tb, 0, s>>>(V, n, k, coef, 0.0, x, (long long)n * kmax, n);
        residual_kernel<<<nb, tb, 0, s>>>(n, hx, sx, theta, hd, sd, r, t);
        // |H x|^2, |S x|^2, |r|^2 (hx, sx and r are consecutive vectors)
        std::vector<double> norms;
        dots_of(hx, 3, nullptr, &norms);
        if ((st = check("vb_lowest_root")) != VB_OK) return st;
        std::vector<double> rr{norms[2]};
        if (std::sqrt(rr[0]) <= tolerance * (std::sqrt(norms[0]) + std::fabs(theta) * std::sqrt(norms[1]))) {
            converged = true;
            break;
        }
        if (!Ui && it + 1 >= kDiagonalPhase) {
            // switch to the shift-invert preconditioner (H - sigma S)^-1 with sigma below the
            // lowest root: the factorization only holds (positive definite) there
            // shift below the root: by default from the residual, which overstates the distance to
            // the root by orders of magnitude on non-orthogonal structures (a shift far below it
            // leaves a weak preconditioner); when the Ritz values of the last eight iterations
            // decrease at a slowing rate, the root is estimated by Aitken's delta-squared
            // extrapolation of theta_{it-8}, theta_{it-4}, theta_it and the shift is 1.5 times the
            // estimated distance plus a tenth of the Ritz gap.  A shift that proves to lie above the
            // root fails the factorization and is widened below.
            double delta = std::max(1.0e-2 * scale, 10.0 * std::sqrt(rr[0]));
            const size_t nr = ritz.size();
            if (nr > 8) {
                const double d1 = ritz[nr - 5] - ritz[nr - 9], d2 = ritz[nr - 1] - ritz[nr - 5];
                if (d1 < 0.0 && d2 < 0.0 && d2 > d1) {
                    const double below = d2 * d2 / (d2 - d1);  // theta - estimated root
                    const double gap = thetas.size() > 1 ? thetas[1] - thetas[0] : 0.0;
                    delta = 1.5 * below + std::max(0.1 * gap, 1.0e-4 * scale);
                }
            }
            if ((st = mbuf.allocate(ctx, m2)) != VB_OK) return st;
            if ((st = uibuf.allocate(ctx, m2)) != VB_OK) return st;
            int info = 1;
            for (int attempt = 0; attempt < 16 && info != 0; ++attempt) {
                const long long count = (long long)n * n;
                shift_kernel<<<(unsigned)std::min<long long>(4096, (count + 255) / 256), 256, 0, s>>>(
                    count, dH, dS, theta - delta, mbuf.as<double>());
                if ((st = check("vb_lowest_root")) != VB_OK) return st;
                if ((st = factor_inverse_device(ctx, mbuf.as<double>(), n, uibuf.as<double>(), &info)) != VB_OK)
                    return st;
                if (info != 0) delta *= 4.0;
            }
            if (info != 0) return set_error(ctx, VB_ERR_NUMERIC, "vb_lowest_root: no positive-definite shift found");
            Ui = uibuf.as<double>();
        }
        if (Ui) {
            // t = U^-1 U^-T r
            gemv_t_kernel<<<(n * 32 + 255) / 256, 256, 0, s>>>(Ui, n, r, st_vec);
            gemv_partial_kernel<<<dim3(nb, kSplits), tb, 0, s>>>(Ui, n, st_vec, ph);
            reduce_splits_kernel<<<nb, tb, 0, s>>>(n, ph, t);
        }
        if (k == kmax) {
            // thick restart: the kKeep lowest Ritz vectors (S-orthonormal) and their images
            const int keep = std::min(kKeep, k);
            std::vector<double> nv((size_t)n * keep), nh((size_t)n * keep), ns((size_t)n * keep);
            for (int j = 0; j < keep; ++j) {
                err = cudaMemcpyAsync(coef, Y.data() + (size_t)j * k, sizeof(double) * k, cudaMemcpyHostToDevice, s);
                combine_kernel<<<dim3(nb, 3), tb, 0, s>>>(V, n, k, coef, 0.0, restart + (size_t)j * n,
                                                          (long long)n * kmax, (long long)keep * n);
                err = cudaStreamSynchronize(s);  // coef is reused by the next column
            }
            err = cudaMemcpyAsync(V, restart, v1 * keep, cudaMemcpyDeviceToDevice, s);
            if (err == cudaSuccess) err = cudaMemcpyAsync(HV, restart + (size_t)keep * n, v1 * keep, cudaMemcpyDeviceToDevice, s);
            if (err == cudaSuccess) err = cudaMemcpyAsync(SV, restart + (size_t)2 * keep * n, v1 * keep, cudaMemcpyDeviceToDevice, s);
            if ((st = check("vb_lowest_root")) != VB_OK) return st;
            for (int i = 0; i < keep; ++i)
                for (int j = 0; j < keep; ++j) {
                    Hs[i + j * kmax] = i == j ? thetas[i] : 0.0;
                    Ss[i + j * kmax] = i == j ? 1.0 : 0.0;
                }
            k = keep;
        }
        // S-orthogonalize the correction t against the basis, twice: V^T S t = (S V)^T t (S is
        // symmetric), so the coefficients come from the stored images S V without a pass over S
        for (int pass = 0; pass < 2; ++pass) {
            std::vector<double> c;
            dots_of(SV, k, t, &c);
            if ((st = check("vb_lowest_root")) != VB_OK) return st;
            for (double& v : c) v = -v;
            err = cudaMemcpyAsync(coef, c.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s);
            combine_kernel<<<nb, tb, 0, s>>>(V, n, k, coef, 1.0, t);
        }
        // one pass over H and S: H t and S t give the norm and, scaled, the new column's images
        gemv2(t, hx, st_vec);
        std::vector<double> nrm;
        dots_of(t, 1, st_vec, &nrm);
        if ((st = check("vb_lowest_root")) != VB_OK) return st;
        if (!(nrm[0] > 1e-28)) break;  // no new direction
        const double inv = 1.0 / std::sqrt(nrm[0]);
        scale_copy_kernel<<<nb, tb, 0, s>>>(n, t, inv, V + (size_t)k * n);
        scale_copy_kernel<<<nb, tb, 0, s>>>(n, hx, inv, HV + (size_t)k * n);
        scale_copy_kernel<<<nb, tb, 0, s>>>(n, st_vec, inv, SV + (size_t)k * n);
        ++k;
        if ((st = add_column(k - 1, true)) != VB_OK) return st;
    }
    if (iterations) *iterations = it;
    *eigenvalue = theta;
    if (host)
        err = cudaMemcpyAsync(eigenvector, x, v1, cudaMemcpyDeviceToHost, s);
    else
        err = cudaMemcpyAsync(eigenvector, x, v1, cudaMemcpyDeviceToDevice, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "vb_lowest_root");
    if (!converged) return set_error(ctx, VB_ERR_NUMERIC, "vb_lowest_root: no convergence within the iteration limit");
    return VB_OK;
}
