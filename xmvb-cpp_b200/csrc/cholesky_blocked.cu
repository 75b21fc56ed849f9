// Blocked FP64 Cholesky factorization and triangular inverse on the FP64 tensor cores, as
// stream-ordered launches with no grid barrier (vb_metric_cholesky and the Davidson shift-invert
// preconditioner above the one-CTA size).
//
// Factorization M = U^T U (upper triangle of M read; Eigen::LLT / LAPACK dpotrf semantics: the
// first non-positive or non-finite pivot stops it with info = its order), right-looking over
// 64-column panels:
//   1. bc_panel_kernel (one CTA): Cholesky of the updated diagonal block in shared memory and the
//      inverse of the resulting triangular block;
//   2. bc_panel_row_kernel: U_12 = U_11^-T A_12;
//   3. bc_trailing_kernel: A_22 -= U_12^T U_12 over the upper 64 x 64 tiles.
// Look-ahead: the trailing update's first tile (the next panel's diagonal block) runs first, then
// the next panel's factorization on a high-priority auxiliary stream while the remaining tiles run
// on the caller's stream.
// Inverse U^-1 (optional): the panel kernels leave U_JJ^-1 on the diagonal blocks; then for block
// sizes b = 64, 128, ... consecutive diagonal blocks are paired,
//   [[A, B], [0, C]]^-1 = [[A^-1, -A^-1 B C^-1], [0, C^-1]],
// every pair of a level at once: T = B C^-1 (bc_level_kernel<0>), then X = -A^-1 T
// (bc_level_kernel<1>).
// Products: 64 x 64 output tiles per CTA, 32-deep k-steps staged through shared memory (double
// buffered, the next step's loads in registers while the current one is multiplied), mma.sync
// m8n8k4 FP64.  Every launch first reads the status word and returns when a panel has failed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "internal.h"

namespace vbcore {
namespace {

constexpr int kNB = 64;         // panel width and output tile edge
constexpr int kKS = 32;         // k-step of a tile product
constexpr int kThreadsB = 256;  // eight warps: 16 x 32 of the output tile each
constexpr int kStrideKC = 36;   // [x][k] staging (k contiguous): 36 = 4 mod 16 doubles
constexpr int kStrideXC = 72;   // [k][x] staging (x contiguous): 72 = 8 mod 16 doubles
constexpr int kTileDoubles = kNB * kStrideKC;  // == kKS * kStrideXC
constexpr size_t kProductSmem = 4 * kTileDoubles * sizeof(double);

static_assert(kNB * kStrideKC == kKS * kStrideXC, "both staging layouts fill one tile buffer");

// Operand of a tile product: element (x, k) (x = row of A or column of B) at p[k + x ld] when the
// operand is k-contiguous, else at p[x + k ld]; x < xn and k < kn are read, the rest is zero.
struct Opnd {
    const double* p;
    long long ld;
    int xn, kn;
};

template <bool KC>
__device__ __forceinline__ void load_regs(const Opnd& o, int x0, int k0, double (&r)[8]) {
    const int t = threadIdx.x;
    if (KC) {
        const int k = k0 + (t & 31);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int x = x0 + (t >> 5) + 8 * i;
            r[i] = (x < o.xn && k < o.kn) ? o.p[k + (long long)x * o.ld] : 0.0;
        }
    } else {
        const int x = x0 + (t & 63);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int k = k0 + (t >> 6) + 4 * i;
            r[i] = (x < o.xn && k < o.kn) ? o.p[x + (long long)k * o.ld] : 0.0;
        }
    }
}

template <bool KC>
__device__ __forceinline__ void store_tile(double* s, const double (&r)[8]) {
    const int t = threadIdx.x;
    if (KC) {
        const int k = t & 31;
#pragma unroll
        for (int i = 0; i < 8; ++i) s[((t >> 5) + 8 * i) * kStrideKC + k] = r[i];
    } else {
        const int x = t & 63;
#pragma unroll
        for (int i = 0; i < 8; ++i) s[((t >> 6) + 4 * i) * kStrideXC + x] = r[i];
    }
}

template <bool KC>
__device__ __forceinline__ double frag(const double* s, int x, int k) {
    return KC ? s[x * kStrideKC + k] : s[k * kStrideXC + x];
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// acc += sum_{k in [kb, ke)} A(xa + r, k) B(k, xb + c) for the CTA's 64 x 64 output tile: warp w
// holds rows 16 (w % 4) .. + 15 and columns 32 (w / 4) .. + 31 as 2 x 4 fragments, lane element
// (row 8 i + lane / 4, column 8 j + 2 (lane % 4) + h) in acc[i][j][h].  kb < ke is uniform.
template <bool AKC, bool BKC>
__device__ void tile_product(Opnd A, Opnd B, int xa, int xb, int kb, int ke, double* smem,
                             double (&acc)[2][4][2]) {
    A.kn = min(A.kn, ke);
    B.kn = min(B.kn, ke);
    // buffers: A in [0, 2) and B in [2, 4) tile slots, alternating by k-step
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gr = lane >> 2, gc = lane & 3;
    const int wm = (warp & 3) * 16, wn = (warp >> 2) * 32;
    double ra[8], rb[8];
    load_regs<AKC>(A, xa, kb, ra);
    load_regs<BKC>(B, xb, kb, rb);
    store_tile<AKC>(smem, ra);
    store_tile<BKC>(smem + 2 * kTileDoubles, rb);
    __syncthreads();
    int buf = 0;
    for (int k0 = kb; k0 < ke; k0 += kKS) {
        const bool more = k0 + kKS < ke;
        if (more) {
            load_regs<AKC>(A, xa, k0 + kKS, ra);
            load_regs<BKC>(B, xb, k0 + kKS, rb);
        }
        const double* a = smem + buf * kTileDoubles;
        const double* b = smem + (2 + buf) * kTileDoubles;
#pragma unroll
        for (int kk = 0; kk < kKS; kk += 4) {
            double af[2], bf[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) af[i] = frag<AKC>(a, wm + 8 * i + gr, kk + gc);
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = frag<BKC>(b, wn + 8 * j + gr, kk + gc);
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j], af[i], bf[j]);
        }
        if (more) {
            store_tile<AKC>(smem + (buf ^ 1) * kTileDoubles, ra);
            store_tile<BKC>(smem + (2 + (buf ^ 1)) * kTileDoubles, rb);
        }
        __syncthreads();
        buf ^= 1;
    }
}

// Output element (row, column) within the tile of acc[i][j][h].
__device__ __forceinline__ int out_row(int i) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    return (warp & 3) * 16 + 8 * i + (lane >> 2);
}
__device__ __forceinline__ int out_col(int j, int h) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    return (warp >> 2) * 32 + 8 * j + 2 * (lane & 3) + h;
}

__device__ __forceinline__ bool failed(const int* status) { return *(const volatile int*)status != 0; }

__global__ void bc_init_kernel(const double* __restrict__ M, double* __restrict__ U, int n) {
    const long long total = (long long)n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long r = e % n, c = e / n;
        U[e] = r <= c ? M[e] : 0.0;
    }
}

// Panel j0: Cholesky of the (updated) diagonal block, rows beyond the matrix padded with the
// identity.  Thread (g, c) keeps rows 16 g .. 16 g + 15 of column c in registers.  Pivot k is
// published through a double-buffered row in shared memory (one barrier per pivot): entries
// a[k][c] for c > k (zeros elsewhere), 1 / p_k and p_k, so the update a[r][c] -= a[k][r] a[k][c] / p_k
// needs no row or column test (rows r <= k and columns c <= k see zeros; the lower triangle takes
// values that are never read and is cleared at the end).  Row r is divided by sqrt(p_r) at the
// end.  The inverse of the triangular block follows the same way, pivots from the last up
// (X = I; X[k, :] /= u_kk; X[r, :] -= u_rk X[k, :] for r < k), with u held transposed in shared
// memory so that a thread's 16 entries of column k are 8 vector loads.  Writes U_JJ into U, its
// inverse into Ub (64 x 64, column-major) and, when Ui is given, onto Ui's diagonal block.
constexpr int kPanelRows = kNB / (kThreadsB / kNB);  // rows per thread (16)
constexpr int kUtStride = kNB + 2;                   // even: rows of the transposed factor stay 16-byte aligned
constexpr int kPrStride = kNB + 2;                   // published row: kNB entries, 1 / p, p
constexpr size_t kPanelSmem = sizeof(double) * (kNB * kUtStride + 2 * kPrStride + kNB);

// v[kk] by a tree of selects on the bits of kk (depth 4, no dynamic register index)
__device__ __forceinline__ double pick(const double (&v)[kPanelRows], int kk) {
    static_assert(kPanelRows == 16, "four select levels");
    double l1[8], l2[4], l3[2];
#pragma unroll
    for (int i = 0; i < 8; ++i) l1[i] = (kk & 1) ? v[2 * i + 1] : v[2 * i];
#pragma unroll
    for (int i = 0; i < 4; ++i) l2[i] = (kk & 2) ? l1[2 * i + 1] : l1[2 * i];
#pragma unroll
    for (int i = 0; i < 2; ++i) l3[i] = (kk & 4) ? l2[2 * i + 1] : l2[2 * i];
    return (kk & 8) ? l3[1] : l3[0];
}

__global__ void __launch_bounds__(kThreadsB) bc_panel_kernel(double* __restrict__ U, double* __restrict__ Ub,
                                                             double* __restrict__ Ui, int n, int j0, int* status) {
    extern __shared__ __align__(16) double psm[];
    double* ut = psm;                          // ut[c * kUtStride + r] = u[r][c]
    double* prow = psm + kNB * kUtStride;      // 2 x kPrStride
    double* piv = prow + 2 * kPrStride;        // pivots p_k
    if (failed(status)) return;
    const int t = threadIdx.x, c = t & (kNB - 1), g = t / kNB;
    const int jb = min(kNB, n - j0);
    double v[kPanelRows];
#pragma unroll
    for (int i = 0; i < kPanelRows; ++i) {
        const int r = kPanelRows * g + i;
        double x = 0.0;
        if (r < jb && c < jb) {
            if (r <= c) x = U[(j0 + r) + (long long)(j0 + c) * n];
        } else if (r == c) {
            x = 1.0;
        }
        v[i] = x;
    }
    // the pivot loops stay rolled (a short body that stays in the instruction cache); a thread's
    // row k % kPanelRows is picked from its registers by selects, not by a dynamic index
#pragma unroll 1
    for (int k = 0; k < kNB; ++k) {
        double* pr = prow + (k & 1) * kPrStride;
        if (g == k / kPanelRows) {
            const double x = pick(v, k % kPanelRows);  // a[k][c]
            pr[c] = c > k ? x : 0.0;
            if (c == k) {
                pr[kNB] = 1.0 / x;
                pr[kNB + 1] = x;
            }
        }
        __syncthreads();
        const double p = pr[kNB + 1];
        if (k < jb && (!(p > 0.0) || !isfinite(p))) {  // the same decision in every thread
            if (t == 0) atomicCAS(status, 0, j0 + k + 1);
            return;
        }
        if (t == 0) piv[k] = p;
        const double f = pr[c] * pr[kNB];
        const double2* q2 = reinterpret_cast<const double2*>(pr + kPanelRows * g);
#pragma unroll
        for (int i = 0; i < kPanelRows / 2; ++i) {
            const double2 q = q2[i];
            v[2 * i] = fma(-q.x, f, v[2 * i]);
            v[2 * i + 1] = fma(-q.y, f, v[2 * i + 1]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kPanelRows; ++i) {
        const int r = kPanelRows * g + i;
        const double d = sqrt(piv[r]);
        v[i] = r < c ? v[i] / d : (r == c ? d : 0.0);
        ut[c * kUtStride + r] = v[i];
        if (r <= c && c < jb) U[(j0 + r) + (long long)(j0 + c) * n] = v[i];
    }
    __syncthreads();
    if (t < kNB) piv[t] = 1.0 / ut[t * kUtStride + t];  // 1 / u_kk, off the pivot chain
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kPanelRows; ++i) v[i] = (kPanelRows * g + i == c) ? 1.0 : 0.0;
#pragma unroll 1
    for (int k = kNB - 1; k >= 0; --k) {
        double* pr = prow + (k & 1) * kPrStride;
        const bool owner = g == k / kPanelRows;
        const int kk = k % kPanelRows;
        double own = 0.0;
        if (owner) {
            own = pick(v, kk) * piv[k];
            pr[c] = own;
        }
        __syncthreads();
        const double xk = pr[c];
        const double2* u2 = reinterpret_cast<const double2*>(ut + k * kUtStride + kPanelRows * g);  // u[r][k]
#pragma unroll
        for (int i = 0; i < kPanelRows / 2; ++i) {
            const double2 q = u2[i];
            v[2 * i] = fma(-q.x, xk, v[2 * i]);
            v[2 * i + 1] = fma(-q.y, xk, v[2 * i + 1]);
        }
        if (owner) {
#pragma unroll
            for (int i = 0; i < kPanelRows; ++i) v[i] = i == kk ? own : v[i];
        }
    }
#pragma unroll
    for (int i = 0; i < kPanelRows; ++i) {
        const int r = kPanelRows * g + i;
        Ub[r + kNB * c] = v[i];
        if (Ui && r <= c && c < jb) Ui[(j0 + r) + (long long)(j0 + c) * n] = v[i];
    }
}

// U_12 = U_11^-T A_12 in place, 64 columns per CTA: A(i, k) = Ub[k + 64 i], B(k, c) = U[j0 + k + c n].
__global__ void __launch_bounds__(kThreadsB) bc_panel_row_kernel(double* __restrict__ U, const double* __restrict__ Ub,
                                                                 int n, int j0, const int* status) {
    extern __shared__ double smem[];
    if (failed(status)) return;
    const int jb = min(kNB, n - j0), j1 = j0 + jb;
    const int c0 = j1 + blockIdx.x * kNB;
    double acc[2][4][2] = {};
    tile_product<true, true>(Opnd{Ub, kNB, jb, jb}, Opnd{U + j0, n, n, jb}, 0, c0, 0, jb, smem, acc);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = out_row(i), c = c0 + out_col(j, h);
                if (r < jb && c < n) U[(j0 + r) + (long long)c * n] = acc[i][j][h];
            }
}

// A_22 -= U_12^T U_12 on the upper 64 x 64 tiles (ti <= tj) of the trailing matrix.
// Tiles first .. first + gridDim.x - 1 of the upper-tile enumeration (t = tj (tj + 1) / 2 + ti).
__global__ void __launch_bounds__(kThreadsB, 2) bc_trailing_kernel(double* __restrict__ U, int n, int j0,
                                                                   const int* status, int first) {
    extern __shared__ double smem[];
    if (failed(status)) return;
    const int jb = min(kNB, n - j0), j1 = j0 + jb;
    const long long b = (long long)blockIdx.x + first;
    int tj = (int)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while ((long long)tj * (tj + 1) / 2 > b) --tj;
    while ((long long)(tj + 1) * (tj + 2) / 2 <= b) ++tj;
    const int ti = (int)(b - (long long)tj * (tj + 1) / 2);
    const int r0 = j1 + kNB * ti, c0 = j1 + kNB * tj;
    const Opnd P{U + j0, n, n, jb};
    // the tile's current entries are loaded first, so that their latency overlaps the product
    double cur[2][4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = r0 + out_row(i), c = c0 + out_col(j, h);
                cur[i][j][h] = (r <= c && c < n) ? U[r + (long long)c * n] : 0.0;
            }
    double acc[2][4][2] = {};
    tile_product<true, true>(P, P, r0, c0, 0, jb, smem, acc);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = r0 + out_row(i), c = c0 + out_col(j, h);
                if (r <= c && c < n) U[r + (long long)c * n] = cur[i][j][h] - acc[i][j][h];
            }
}

// One level of the pairwise inverse: pair p has A = Ui block at rows/columns [r0, r0 + b), C at
// [c0, c0 + cs) with c0 = r0 + b, and B = U[r0 .., c0 ..].  STAGE 0: T = B C^-1 (k <= column:
// C^-1 is upper triangular); STAGE 1: Ui[r0 .., c0 ..] = -A^-1 T (k >= row).
template <int STAGE>
__global__ void __launch_bounds__(kThreadsB) bc_level_kernel(const double* __restrict__ U, double* __restrict__ Ui,
                                                             double* __restrict__ T, int n, int b, const int* status) {
    extern __shared__ double smem[];
    if (failed(status)) return;
    const int r0 = 2 * b * blockIdx.y, c0 = r0 + b;
    if (c0 >= n) return;
    const int cs = min(b, n - c0);
    const int tr = b / kNB;
    const int ti = blockIdx.x % tr, tj = blockIdx.x / tr;
    if (kNB * tj >= cs) return;
    const long long ln = n;
    double acc[2][4][2] = {};
    if (STAGE == 0) {
        const int ke = min(cs, kNB * tj + kNB);
        tile_product<false, true>(Opnd{U + r0 + c0 * ln, ln, b, cs}, Opnd{Ui + c0 + c0 * ln, ln, cs, cs}, kNB * ti,
                                  kNB * tj, 0, ke, smem, acc);
    } else {
        tile_product<false, true>(Opnd{Ui + r0 + r0 * ln, ln, b, b}, Opnd{T + r0 + c0 * ln, ln, cs, b}, kNB * ti,
                                  kNB * tj, kNB * ti, b, smem, acc);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = kNB * ti + out_row(i), c = kNB * tj + out_col(j, h);
                if (r < b && c < cs) {
                    const long long at = (r0 + r) + (c0 + c) * ln;
                    if (STAGE == 0)
                        T[at] = acc[i][j][h];
                    else
                        Ui[at] = -acc[i][j][h];
                }
            }
}

}  // namespace

size_t blocked_cholesky_workspace(int n, bool inverse) {
    const size_t t = inverse ? sizeof(double) * (size_t)n * n : 0;
    return t + sizeof(double) * kNB * kNB + 256;
}

// U (n x n, device, column-major; the lower triangle is written with zeros) and, when Ui is not
// null, U^-1 (same layout) of the device matrix M; `work` holds blocked_cholesky_workspace(n, Ui)
// bytes.  *info: order of the first failing pivot, 0 on success.  Synchronizes the stream.
namespace {

// High-priority auxiliary streams (with their two events) for the look-ahead panels, pooled per
// device: a call takes one for its duration, so concurrent calls from several host threads never
// share one.
struct AuxStream {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t block_ready = nullptr, panel_done = nullptr;
};
std::mutex g_aux_mutex;
std::vector<AuxStream> g_aux_free;

cudaError_t acquire_aux(AuxStream* out) {
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    {
        std::lock_guard<std::mutex> lock(g_aux_mutex);
        for (size_t i = 0; i < g_aux_free.size(); ++i)
            if (g_aux_free[i].device == device) {
                *out = g_aux_free[i];
                g_aux_free.erase(g_aux_free.begin() + (long)i);
                return cudaSuccess;
            }
    }
    AuxStream a;
    a.device = device;
    int least = 0, greatest = 0;
    err = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (err == cudaSuccess) err = cudaStreamCreateWithPriority(&a.stream, cudaStreamNonBlocking, greatest);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&a.block_ready, cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&a.panel_done, cudaEventDisableTiming);
    if (err != cudaSuccess) return err;
    // a fresh event counts as complete, so the first waits on it return at once
    *out = a;
    return cudaSuccess;
}

void release_aux(const AuxStream& a) {
    std::lock_guard<std::mutex> lock(g_aux_mutex);
    g_aux_free.push_back(a);
}

}  // namespace

cudaError_t blocked_cholesky(const double* M, int n, double* U, double* Ui, void* work, int* info,
                             cudaStream_t s) {
    *info = 0;
    unsigned char* w = static_cast<unsigned char*>(work);
    double* T = Ui ? reinterpret_cast<double*>(w) : nullptr;
    double* Ub = reinterpret_cast<double*>(w + (Ui ? sizeof(double) * (size_t)n * n : 0));
    int* status = reinterpret_cast<int*>(Ub + kNB * kNB);
    cudaError_t err = allow_dynamic_smem((const void*)bc_panel_kernel, kPanelSmem);
    if (err == cudaSuccess) err = allow_dynamic_smem((const void*)bc_panel_row_kernel, kProductSmem);
    if (err == cudaSuccess) err = allow_dynamic_smem((const void*)bc_trailing_kernel, kProductSmem);
    if (err == cudaSuccess) err = allow_dynamic_smem((const void*)bc_level_kernel<0>, kProductSmem);
    if (err == cudaSuccess) err = allow_dynamic_smem((const void*)bc_level_kernel<1>, kProductSmem);
    if (err == cudaSuccess) err = cudaMemsetAsync(status, 0, sizeof(int), s);
    if (err == cudaSuccess && Ui) err = cudaMemsetAsync(Ui, 0, sizeof(double) * (size_t)n * n, s);
    if (err != cudaSuccess) return err;
    const long long total = (long long)n * n;
    bc_init_kernel<<<(unsigned)std::min<long long>(4096, (total + 255) / 256), 256, 0, s>>>(M, U, n);
    // Look-ahead: after the panel row, the trailing update's first tile (the next panel's
    // diagonal block) runs alone, then the next panel's factorization goes to a high-priority
    // auxiliary stream while the other tiles run on s, so that the one-CTA panel takes an SM as
    // soon as a trailing CTA retires; the next panel row waits for it.
    AuxStream aux;
    if ((err = acquire_aux(&aux)) != cudaSuccess) return err;
    bc_panel_kernel<<<1, kThreadsB, kPanelSmem, s>>>(U, Ub, Ui, n, 0, status);
    for (int j0 = 0; j0 < n && err == cudaSuccess; j0 += kNB) {
        const int j1 = std::min(n, j0 + kNB);
        if (j1 >= n) break;
        const int m = n - j1, nt = (m + kNB - 1) / kNB;
        const long long tiles = (long long)nt * (nt + 1) / 2;
        if (j0 > 0 && (err = cudaStreamWaitEvent(s, aux.panel_done, 0)) != cudaSuccess) break;
        bc_panel_row_kernel<<<nt, kThreadsB, kProductSmem, s>>>(U, Ub, n, j0, status);
        bc_trailing_kernel<<<1, kThreadsB, kProductSmem, s>>>(U, n, j0, status, 0);
        if ((err = cudaEventRecord(aux.block_ready, s)) != cudaSuccess) break;
        if ((err = cudaStreamWaitEvent(aux.stream, aux.block_ready, 0)) != cudaSuccess) break;
        bc_panel_kernel<<<1, kThreadsB, kPanelSmem, aux.stream>>>(U, Ub, Ui, n, j1, status);
        if ((err = cudaEventRecord(aux.panel_done, aux.stream)) != cudaSuccess) break;
        if (tiles > 1)
            bc_trailing_kernel<<<(unsigned)(tiles - 1), kThreadsB, kProductSmem, s>>>(U, n, j0, status, 1);
        err = cudaGetLastError();
    }
    // join: the last panel on the auxiliary stream precedes the rest of s
    const cudaError_t join = cudaStreamWaitEvent(s, aux.panel_done, 0);
    if (err == cudaSuccess) err = join;
    release_aux(aux);
    if (Ui) {
        for (int b = kNB; b < n && err == cudaSuccess; b *= 2) {
            const int pairs = (n + 2 * b - 1) / (2 * b);
            const int tr = b / kNB;
            const dim3 grid((unsigned)(tr * tr), (unsigned)pairs);
            bc_level_kernel<0><<<grid, kThreadsB, kProductSmem, s>>>(U, Ui, T, n, b, status);
            bc_level_kernel<1><<<grid, kThreadsB, kProductSmem, s>>>(U, Ui, T, n, b, status);
            err = cudaGetLastError();
        }
    }
    int h = 0;
    if (err == cudaSuccess) err = cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err == cudaSuccess) *info = h;
    return err;
}

}  // namespace vbcore
