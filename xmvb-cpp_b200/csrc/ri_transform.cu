// RI AO -> active-space transform of the metric-whitened three-index factors, FP64
// (transform_ri_active_integrals, src/integrals/active/ri.cpp:33-96;
//  transform_ri_one_index, src/integrals/ao/ri_transform.cpp:10-37;
//  pack_ri_active_integrals, src/integrals/active/ri.cpp:13-31), and its adjoint.
//
// Layouts (column-major, as the reference's Eigen matrices):
//   B  [n_aux x NP], NP = n_bf (n_bf + 1) / 2, B[P + pair(mu, nu) n_aux]
//   C  [n_bf x n_act]
//   T  one-index factors [(n_act n_aux) x n_bf], T[(a n_aux + P) + mu n_act n_aux]
//        = sum_nu B_P(mu, nu) C(nu, a)                                     (ri_one_index_factors)
//   L  [n_aux x n_act (n_act + 1) / 2], L[P + pair(a, b) n_aux] = sum_mu T[a, P, mu] C(mu, b)
//   K  packed, K[pair(p, q)] = sum_P L[P, p] L[P, q]
//
// The one-index step carries the flops (2 n_aux n_bf^2 n_act): lanes own 4 auxiliary rows each
// (128 per warp) and accumulate T[a, P, mu] for all n_act orbitals in registers (64 FP64
// accumulators per lane), streaming the AO-pair columns pair(mu, nu) of B (1 KB coalesced per
// column) against rows of C.  Each packed column is needed by two AO indices (mu and nu).
//
// Split precision (VB_PRECISION_BF16X3): the one-index step on the tensor cores.  Every operand
// x (FP64, rounded to FP32) is split into three BF16 parts x = x0 + x1 + x2 (about 24 mantissa
// bits); the products of order <= 2 (a0 c0; a0 c1 + a1 c0; a0 c2 + a1 c1 + a2 c0) run as BF16
// mma.sync m16n8k16 tiles with FP32 accumulation, the leading order in its own accumulator that
// is flushed into FP64 every few K steps, the recombination in FP64 (compensated).  A warp owns
// 16 auxiliary rows of one AO index mu (one M tile; the two N tiles cover 16 active orbitals)
// and streams K = nu in steps of 16 straight from the packed columns (each column read is one
// aligned 128-byte line of 16 rows), one step prefetched in registers; the coefficient
// fragments (three splits, fragment order) are built once and staged in shared memory.  The
// kernel reads B once per (mu, nu) use like the FP64 kernel; with mu fastest in the grid, the
// second use of a packed column is normally an L2 hit.  The second index and the packing stay
// FP64.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "internal.h"

namespace vbcore {
namespace {

constexpr int kMaxActive = 16;
constexpr int kRowsPerLane = 4;
constexpr int kAuxTile = 32 * kRowsPerLane;  // auxiliary rows per warp
constexpr int kWarpsPerCta = 4;              // AO indices per CTA
constexpr int kNuChunk = 256;                // C rows staged per shared-memory chunk

__device__ __forceinline__ long long ao_pair(int a, int b) {
    const long long hi = a > b ? a : b, lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

// T[a, P, mu] = sum_nu B[P, pair(mu, nu)] C(nu, a).  grid.x = AO-index groups (fastest),
// grid.y = auxiliary tiles.
__global__ void __launch_bounds__(32 * kWarpsPerCta) one_index_kernel(const double* __restrict__ B, int n_aux, int n_bf,
                                                                      const double* __restrict__ C, int n_act,
                                                                      double* __restrict__ T) {
    __shared__ __align__(16) double sC[kNuChunk][kMaxActive];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mu = blockIdx.x * kWarpsPerCta + warp;
    const int aux0 = blockIdx.y * kAuxTile;
    double acc[kRowsPerLane][kMaxActive];
#pragma unroll
    for (int i = 0; i < kRowsPerLane; ++i)
#pragma unroll
        for (int a = 0; a < kMaxActive; ++a) acc[i][a] = 0.0;
    bool row_ok[kRowsPerLane];
#pragma unroll
    for (int i = 0; i < kRowsPerLane; ++i) row_ok[i] = aux0 + lane + 32 * i < n_aux;
    for (int nu0 = 0; nu0 < n_bf; nu0 += kNuChunk) {
        const int cnt = min(kNuChunk, n_bf - nu0);
        __syncthreads();
        for (int e = threadIdx.x; e < cnt * kMaxActive; e += blockDim.x) {
            const int a = e / cnt, nu = e % cnt;
            sC[nu][a] = a < n_act ? __ldg(C + nu0 + nu + (long long)a * n_bf) : 0.0;
        }
        __syncthreads();
        if (mu < n_bf) {
            const double* base = B + aux0 + lane;
#pragma unroll 2
            for (int nu = 0; nu < cnt; ++nu) {
                const double* col = base + ao_pair(mu, nu0 + nu) * n_aux;
                double b[kRowsPerLane];
#pragma unroll
                for (int i = 0; i < kRowsPerLane; ++i) b[i] = row_ok[i] ? __ldg(col + 32 * i) : 0.0;
                const double2* c2 = reinterpret_cast<const double2*>(&sC[nu][0]);
#pragma unroll
                for (int h = 0; h < kMaxActive / 2; ++h) {
                    const double2 c = c2[h];
#pragma unroll
                    for (int i = 0; i < kRowsPerLane; ++i) {
                        acc[i][2 * h] = fma(b[i], c.x, acc[i][2 * h]);
                        acc[i][2 * h + 1] = fma(b[i], c.y, acc[i][2 * h + 1]);
                    }
                }
            }
        }
    }
    if (mu >= n_bf) return;
    const long long ld = (long long)n_act * n_aux;
#pragma unroll
    for (int i = 0; i < kRowsPerLane; ++i) {
        const int P = aux0 + lane + 32 * i;
        if (!row_ok[i]) continue;
#pragma unroll
        for (int a = 0; a < kMaxActive; ++a)
            if (a < n_act) T[(long long)a * n_aux + P + (long long)mu * ld] = acc[i][a];
    }
}

// Pipelined variant for even n_aux (16-byte aligned columns) and n_bf <= kPipelinedMaxBf: a
// warp per AO index mu (six per CTA), each streaming its columns pair(mu, nu) of B through a
// private 3-stage cp.async ring in shared memory (no registers held by loads in flight), the
// rows of C staged once per CTA in shared memory (warp-uniform broadcast reads).  Two CTAs
// (12 warps) per SM: the 64 FP64 accumulators per lane cap residency at 12 warps anyway.
constexpr int kStages = 3;
constexpr int kNuStage = 2;
constexpr int kPipeWarps = 6;
constexpr int kPipelinedMaxBf = 1024;

size_t pipelined_smem_bytes(int n_bf) {
    return sizeof(double) * ((size_t)n_bf * kMaxActive + (size_t)kPipeWarps * kStages * kNuStage * kAuxTile);
}

__global__ void transpose_coefficients_kernel(const double* __restrict__ C, int n_bf, int n_act,
                                              double* __restrict__ Ct) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_bf * kMaxActive) return;
    const int nu = e / kMaxActive, a = e % kMaxActive;
    Ct[e] = a < n_act ? C[nu + (long long)a * n_bf] : 0.0;
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src, int src_bytes) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(gmem_src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(32 * kPipeWarps, 2) one_index_pipelined_kernel(const double* __restrict__ B,
                                                                                 int n_aux, int n_bf,
                                                                                 const double* __restrict__ Ct,
                                                                                 int n_act, double* __restrict__ T) {
    extern __shared__ __align__(16) double smem[];
    double* sCt = smem;                                    // [n_bf][16]
    double* ring_all = smem + (size_t)n_bf * kMaxActive;   // [warp][stage][nu][128]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mu = blockIdx.x * kPipeWarps + warp;
    const int aux0 = blockIdx.y * kAuxTile;
    for (int e = threadIdx.x; e < n_bf * kMaxActive / 2; e += blockDim.x)
        reinterpret_cast<double2*>(sCt)[e] = __ldg(reinterpret_cast<const double2*>(Ct) + e);
    __syncthreads();
    if (mu >= n_bf) return;  // warp-private pipeline below: no CTA-wide barrier after this point
    const int n_steps = (n_bf + kNuStage - 1) / kNuStage;
    double* ring = ring_all + (size_t)warp * kStages * kNuStage * kAuxTile;
    auto issue = [&](int step) {
        if (step < n_steps) {
            const int stage = step % kStages;
#pragma unroll
            for (int v = 0; v < kNuStage; ++v) {
                const int nu = step * kNuStage + v;
                const double* col = nu < n_bf ? B + ao_pair(mu, nu) * n_aux + aux0 : B;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int j = lane + 32 * h;  // 16-byte chunk: rows 2j, 2j + 1 of the tile
                    const bool ok = nu < n_bf && aux0 + 2 * j < n_aux;
                    cp_async16(ring + (stage * kNuStage + v) * kAuxTile + 2 * j, ok ? col + 2 * j : B, ok ? 16 : 0);
                }
            }
        }
        cp_async_commit();  // empty groups keep the group count uniform
    };
#pragma unroll
    for (int st = 0; st < kStages - 1; ++st) issue(st);
    double acc[kRowsPerLane][kMaxActive];
#pragma unroll
    for (int i = 0; i < kRowsPerLane; ++i)
#pragma unroll
        for (int a = 0; a < kMaxActive; ++a) acc[i][a] = 0.0;
    for (int step = 0; step < n_steps; ++step) {
        issue(step + kStages - 1);
        cp_async_wait<kStages - 1>();
        __syncwarp();
        const int stage = step % kStages;
#pragma unroll
        for (int v = 0; v < kNuStage; ++v) {
            const int nu = step * kNuStage + v;
            if (nu >= n_bf) break;
            const double* tile = ring + (stage * kNuStage + v) * kAuxTile + lane;
            double b[kRowsPerLane];
#pragma unroll
            for (int i = 0; i < kRowsPerLane; ++i) b[i] = tile[32 * i];
            const double2* c2 = reinterpret_cast<const double2*>(sCt + (size_t)nu * kMaxActive);
#pragma unroll
            for (int h = 0; h < kMaxActive / 2; ++h) {
                const double2 c = c2[h];
#pragma unroll
                for (int i = 0; i < kRowsPerLane; ++i) {
                    acc[i][2 * h] = fma(b[i], c.x, acc[i][2 * h]);
                    acc[i][2 * h + 1] = fma(b[i], c.y, acc[i][2 * h + 1]);
                }
            }
        }
        __syncwarp();
    }
    cp_async_wait<0>();
    const long long ld = (long long)n_act * n_aux;
#pragma unroll
    for (int i = 0; i < kRowsPerLane; ++i) {
        const int P = aux0 + lane + 32 * i;
        if (P >= n_aux) continue;
#pragma unroll
        for (int a = 0; a < kMaxActive; ++a)
            if (a < n_act) T[(long long)a * n_aux + P + (long long)mu * ld] = acc[i][a];
    }
}

// FP64 tensor-core variant (mma.sync m8n8k4, the FP64 tensor path of sm_100a) for even n_aux
// and n_bf <= kDmmaMaxBf: T_mu[P, a] = sum_nu B[P, pair(mu, nu)] C[nu, a] is, per AO index mu,
// a (64 auxiliary rows) x (16 active) x (n_bf) product.  Persistent CTAs of eight warps stage C
// once ([nu][20], padded so the B-fragment loads are conflict-free) and loop over (8 AO indices,
// 64 auxiliary rows) items; each warp streams its mu's columns through a private 3-stage
// cp.async ring of 8 columns x 64 rows (row stride 68: conflict-free A-fragment loads) and keeps
// 8 x 2 accumulator tiles in registers.  Items run with the auxiliary tile fastest, so the
// CTAs resident together read whole packed columns.  The sum over nu runs in a fixed order.
constexpr int kDmmaWarps = 8;
constexpr int kDmmaRows = 64;      // auxiliary rows per item (8 M tiles)
constexpr int kDmmaNu = 8;         // columns per ring stage (two k-steps)
constexpr int kDmmaStages = 3;
constexpr int kDmmaRing = 68;      // ring row stride (doubles; = 4 mod 16)
constexpr int kDmmaCt = 20;        // staged C stride (doubles; = 4 mod 16)
constexpr int kDmmaMaxBf = 768;   // shared memory: C staging plus the rings

size_t dmma_smem_bytes(int n_bf) {
    return sizeof(double) * ((size_t)n_bf * kDmmaCt + (size_t)kDmmaWarps * kDmmaStages * kDmmaNu * kDmmaRing);
}

__device__ __forceinline__ void dmma_f64(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(32 * kDmmaWarps, 1) one_index_dmma_kernel(const double* __restrict__ B, int n_aux,
                                                                            int n_bf, const double* __restrict__ Ct,
                                                                            int n_act, double* __restrict__ T) {
    extern __shared__ __align__(16) double smem[];
    double* sC = smem;                                       // [n_bf][kDmmaCt]
    double* ring_all = smem + (size_t)n_bf * kDmmaCt;       // [warp][stage][nu][kDmmaRing]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gr = lane >> 2, gc = lane & 3;
    for (int e = threadIdx.x; e < n_bf * kDmmaCt; e += blockDim.x) {
        const int nu = e / kDmmaCt, a = e % kDmmaCt;
        sC[e] = a < kMaxActive ? __ldg(Ct + (size_t)nu * kMaxActive + a) : 0.0;
    }
    __syncthreads();
    double* ring = ring_all + (size_t)warp * kDmmaStages * kDmmaNu * kDmmaRing;
    const int mu_blocks = (n_bf + kDmmaWarps - 1) / kDmmaWarps;
    const int aux_tiles = (n_aux + kDmmaRows - 1) / kDmmaRows;
    const int n_steps = (n_bf + kDmmaNu - 1) / kDmmaNu;
    const long long ld = (long long)n_act * n_aux;
    for (long long item = blockIdx.x; item < (long long)mu_blocks * aux_tiles; item += gridDim.x) {
        const int mu = (int)(item / aux_tiles) * kDmmaWarps + warp;
        const int aux0 = (int)(item % aux_tiles) * kDmmaRows;
        if (mu >= n_bf) continue;  // warp-private work below: no CTA-wide barrier
        auto issue = [&](int step) {
            if (step < n_steps) {
                double* stage = ring + (step % kDmmaStages) * kDmmaNu * kDmmaRing;
#pragma unroll
                for (int h = 0; h < kDmmaNu; ++h) {
                    // lane's 16-byte chunk: column h of the stage, rows 2 lane and 2 lane + 1
                    const int nu = step * kDmmaNu + h, r = 2 * lane;
                    const bool ok = nu < n_bf && aux0 + r < n_aux;
                    const double* src = ok ? B + ao_pair(mu, nu) * n_aux + aux0 + r : B;
                    cp_async16(stage + h * kDmmaRing + r, src, ok ? 16 : 0);
                }
            }
            cp_async_commit();
        };
#pragma unroll
        for (int st = 0; st < kDmmaStages - 1; ++st) issue(st);
        double acc[8][2][2];
#pragma unroll
        for (int m = 0; m < 8; ++m)
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) acc[m][nt][0] = acc[m][nt][1] = 0.0;
        for (int step = 0; step < n_steps; ++step) {
            issue(step + kDmmaStages - 1);
            cp_async_wait<kDmmaStages - 1>();
            __syncwarp();
            const double* stage = ring + (step % kDmmaStages) * kDmmaNu * kDmmaRing;
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                const int v = 4 * ks + gc;  // column of this lane's A (and row of its B) element
                const int nu = step * kDmmaNu + v;
                const double* cb = sC + (size_t)(nu < n_bf ? nu : 0) * kDmmaCt + gr;
                const double b0 = nu < n_bf ? cb[0] : 0.0, b1 = nu < n_bf ? cb[8] : 0.0;
#pragma unroll
                for (int m = 0; m < 8; ++m) {
                    const double a = stage[v * kDmmaRing + 8 * m + gr];
                    dmma_f64(acc[m][0], a, b0);
                    dmma_f64(acc[m][1], a, b1);
                }
            }
            __syncwarp();
        }
        cp_async_wait<0>();
        __syncwarp();
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int P = aux0 + 8 * m + gr;
            if (P >= n_aux) continue;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int a = 8 * nt + 2 * gc + h;
                    if (a < n_act) T[(long long)a * n_aux + P + (long long)mu * ld] = acc[m][nt][h];
                }
        }
    }
}

constexpr int kSplitWarps = 8;   // AO indices per CTA
constexpr int kSplitRows = 16;   // auxiliary rows per warp (one M tile)
constexpr int kSplitFlush = 4;   // K steps between flushes of the leading-order FP32 accumulator
constexpr int kSplitMaxSteps = 96;  // shared-memory coefficient fragments: n_bf <= 1536

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// Two FP32 values (x0: lower column / K index) as three BF16x2 words, x = w0 + w1 + w2.
__device__ __forceinline__ void split3(float x0, float x1, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    const float r0 = x0 - __low2float(h), r1 = x1 - __high2float(h);
    const __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
    const float s0 = r0 - __low2float(m), s1 = r1 - __high2float(m);
    const __nv_bfloat162 l = __floats2bfloat162_rn(s0, s1);
    w0 = bf16x2_bits(h);
    w1 = bf16x2_bits(m);
    w2 = bf16x2_bits(l);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Coefficient fragments for the m16n8k16 B operand: entry (step s, lane) holds, per split z,
// uint4 {b0 (N tile 0), b1 (N tile 0), b0 (N tile 1), b1 (N tile 1)} with
// b0 = C(16 s + 2 q + {0, 1}, a), b1 = C(16 s + 2 q + 8 + {0, 1}, a), a = 8 j + g (g = lane / 4,
// q = lane % 4); zero beyond n_bf and n_act.
__global__ void split_coefficients_kernel(const double* __restrict__ C, int n_bf, int n_act, int n_steps,
                                          uint4* __restrict__ Cf) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_steps * 32) return;
    const int st = e >> 5, lane = e & 31, g = lane >> 2, q = lane & 3;
    uint32_t w[3][2][2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int a = 8 * j + g;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int nu = 16 * st + 2 * q + 8 * r;
            const float c0 = (a < n_act && nu < n_bf) ? (float)C[nu + (long long)a * n_bf] : 0.0f;
            const float c1 = (a < n_act && nu + 1 < n_bf) ? (float)C[nu + 1 + (long long)a * n_bf] : 0.0f;
            split3(c0, c1, w[0][j][r], w[1][j][r], w[2][j][r]);
        }
    }
#pragma unroll
    for (int z = 0; z < 3; ++z) Cf[(size_t)e * 3 + z] = make_uint4(w[z][0][0], w[z][0][1], w[z][1][0], w[z][1][1]);
}

// T[a, P, mu] = sum_nu B[P, pair(mu, nu)] C(nu, a) by split-BF16 tensor-core tiles.
// grid.x = groups of kSplitWarps AO indices (fastest), grid.y = tiles of 16 auxiliary rows.
__global__ void __launch_bounds__(32 * kSplitWarps, 2) one_index_split_kernel(const double* __restrict__ B, int n_aux,
                                                                              int n_bf, int n_steps,
                                                                              const uint4* __restrict__ Cf, int n_act,
                                                                              double* __restrict__ T) {
    extern __shared__ uint4 sCf[];  // [n_steps][32][3]
    for (int e = threadIdx.x; e < n_steps * 32 * 3; e += blockDim.x) sCf[e] = __ldg(Cf + e);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mu = blockIdx.x * kSplitWarps + warp;
    if (mu >= n_bf) return;  // no CTA barrier below
    const int g = lane >> 2, q = lane & 3;
    const int P0 = blockIdx.y * kSplitRows;
    const int row0 = P0 + g, row1 = P0 + g + 8;
    const bool ok0 = row0 < n_aux, ok1 = row1 < n_aux;
    // x[2 ci + h]: column ci of {2q, 2q + 1, 2q + 8, 2q + 9}, row h of {g, g + 8}
    auto load = [&](int st, double(&x)[8]) {
#pragma unroll
        for (int ci = 0; ci < 4; ++ci) {
            const int nu = 16 * st + 2 * q + (ci & 1) + 8 * (ci >> 1);
            const bool nok = nu < n_bf;
            const double* col = B + ao_pair(mu, nok ? nu : 0) * n_aux;
            x[2 * ci] = (nok && ok0) ? __ldg(col + row0) : 0.0;
            x[2 * ci + 1] = (nok && ok1) ? __ldg(col + row1) : 0.0;
        }
    };
    float acc0[2][4], acc12[2][4];
    double accd[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            acc0[j][i] = 0.0f;
            acc12[j][i] = 0.0f;
            accd[j][i] = 0.0;
        }
    auto step = [&](int st, const double(&x)[8]) {
        // A fragments: reg0 (g, 2q..2q+1), reg1 (g+8, 2q..), reg2 (g, 2q+8..), reg3 (g+8, 2q+8..)
        uint32_t A0[4], A1[4], A2[4];
        split3((float)x[0], (float)x[2], A0[0], A1[0], A2[0]);
        split3((float)x[1], (float)x[3], A0[1], A1[1], A2[1]);
        split3((float)x[4], (float)x[6], A0[2], A1[2], A2[2]);
        split3((float)x[5], (float)x[7], A0[3], A1[3], A2[3]);
        const uint4* cf = sCf + ((size_t)st * 32 + lane) * 3;
        const uint4 c0 = cf[0], c1 = cf[1], c2 = cf[2];
        mma_bf16(acc0[0], A0, c0.x, c0.y);
        mma_bf16(acc0[1], A0, c0.z, c0.w);
        mma_bf16(acc12[0], A0, c1.x, c1.y);
        mma_bf16(acc12[1], A0, c1.z, c1.w);
        mma_bf16(acc12[0], A1, c0.x, c0.y);
        mma_bf16(acc12[1], A1, c0.z, c0.w);
        mma_bf16(acc12[0], A0, c2.x, c2.y);
        mma_bf16(acc12[1], A0, c2.z, c2.w);
        mma_bf16(acc12[0], A1, c1.x, c1.y);
        mma_bf16(acc12[1], A1, c1.z, c1.w);
        mma_bf16(acc12[0], A2, c0.x, c0.y);
        mma_bf16(acc12[1], A2, c0.z, c0.w);
        if ((st + 1) % kSplitFlush == 0) {
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    accd[j][i] += (double)acc0[j][i];
                    acc0[j][i] = 0.0f;
                }
        }
    };
    double xa[8], xb[8];
    load(0, xa);
    for (int st = 0; st < n_steps; st += 2) {
        if (st + 1 < n_steps) load(st + 1, xb);
        step(st, xa);
        if (st + 2 < n_steps) load(st + 2, xa);
        if (st + 1 < n_steps) step(st + 1, xb);
    }
    const long long ld = (long long)n_act * n_aux;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int P = (i < 2) ? row0 : row1;
            const int a = 8 * j + 2 * q + (i & 1);
            if (P < n_aux && a < n_act)
                T[(long long)a * n_aux + P + (long long)mu * ld] = accd[j][i] + (double)acc0[j][i] + (double)acc12[j][i];
        }
}

// Pipelined split kernel (even n_aux, 16-byte aligned B): each warp streams its 16 x 16 tiles
// of B through a private kSplitStages-deep cp.async ring in shared memory.  A tile is stored
// column by column (16 rows = eight 16-byte chunks); chunk j of column c sits at chunk
// position j ^ (c & 7), so the 8-byte fragment reads of a quarter warp hit distinct banks.
constexpr int kSplitStages = 4;

size_t split_pipelined_smem_bytes(int n_steps) {
    return sizeof(uint4) * (size_t)n_steps * 32 * 3 + sizeof(double) * (size_t)kSplitWarps * kSplitStages * 256;
}

__global__ void __launch_bounds__(32 * kSplitWarps, 2) one_index_split_pipelined_kernel(
    const double* __restrict__ B, int n_aux, int n_bf, int n_steps, const uint4* __restrict__ Cf, int n_act,
    double* __restrict__ T) {
    extern __shared__ uint4 sCf[];  // [n_steps][32][3], then the rings
    for (int e = threadIdx.x; e < n_steps * 32 * 3; e += blockDim.x) sCf[e] = __ldg(Cf + e);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mu = blockIdx.x * kSplitWarps + warp;
    if (mu >= n_bf) return;  // warp-private pipeline below: no CTA-wide barrier after this point
    double* ring = reinterpret_cast<double*>(sCf + (size_t)n_steps * 32 * 3) + (size_t)warp * kSplitStages * 256;
    const int g = lane >> 2, q = lane & 3;
    const int P0 = blockIdx.y * kSplitRows;
    // copy side: this lane moves chunk jc (rows 2 jc, 2 jc + 1) of columns cc + 4 t
    const int jc = lane & 7, cc = lane >> 3;
    const bool row_ok = P0 + 2 * jc < n_aux;
    const double* bsrc = B + P0 + 2 * jc;
    const int mu_tri = mu * (mu + 1) / 2;
    auto issue = [&](int st) {
        if (st < n_steps) {
            double* tile = ring + (st % kSplitStages) * 256;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int c = cc + 4 * t;
                const int nu = 16 * st + c;
                const bool ok = row_ok && nu < n_bf;
                const int pair = nu <= mu ? mu_tri + nu : nu * (nu + 1) / 2 + mu;
                const double* src = ok ? bsrc + (long long)pair * n_aux : B;
                cp_async16(tile + c * 16 + 2 * (jc ^ (c & 7)), src, ok ? 16 : 0);
            }
        }
        cp_async_commit();  // empty groups keep the group count uniform
    };
    // read side: fragment rows g and g + 8 are auxiliary rows 2g and 2g + 1 (one 16-byte chunk,
    // chunk g of a column); fragment columns 2q, 2q + 1, 2q + 8, 2q + 9 are nu offsets
    int roff[4];
#pragma unroll
    for (int ci = 0; ci < 4; ++ci) {
        const int c = 2 * q + (ci & 1) + 8 * (ci >> 1);
        roff[ci] = c * 16 + 2 * (g ^ (c & 7));
    }
#pragma unroll
    for (int st = 0; st < kSplitStages - 1; ++st) issue(st);
    float acc0[2][4], acc12[2][4];
    double accd[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            acc0[j][i] = 0.0f;
            acc12[j][i] = 0.0f;
            accd[j][i] = 0.0;
        }
    for (int st = 0; st < n_steps; ++st) {
        issue(st + kSplitStages - 1);
        cp_async_wait<kSplitStages - 1>();
        __syncwarp();
        const double* tile = ring + (st % kSplitStages) * 256;
        double2 v[4];  // v[ci] = (aux row 2g, aux row 2g + 1) of fragment column ci
#pragma unroll
        for (int ci = 0; ci < 4; ++ci) v[ci] = *reinterpret_cast<const double2*>(tile + roff[ci]);
        __syncwarp();  // the stage may be refilled by the next issue
        uint32_t A0[4], A1[4], A2[4];
        split3((float)v[0].x, (float)v[1].x, A0[0], A1[0], A2[0]);
        split3((float)v[0].y, (float)v[1].y, A0[1], A1[1], A2[1]);
        split3((float)v[2].x, (float)v[3].x, A0[2], A1[2], A2[2]);
        split3((float)v[2].y, (float)v[3].y, A0[3], A1[3], A2[3]);
        const uint4* cf = sCf + ((size_t)st * 32 + lane) * 3;
        const uint4 c0 = cf[0], c1 = cf[1], c2 = cf[2];
        mma_bf16(acc0[0], A0, c0.x, c0.y);
        mma_bf16(acc0[1], A0, c0.z, c0.w);
        mma_bf16(acc12[0], A0, c1.x, c1.y);
        mma_bf16(acc12[1], A0, c1.z, c1.w);
        mma_bf16(acc12[0], A1, c0.x, c0.y);
        mma_bf16(acc12[1], A1, c0.z, c0.w);
        mma_bf16(acc12[0], A0, c2.x, c2.y);
        mma_bf16(acc12[1], A0, c2.z, c2.w);
        mma_bf16(acc12[0], A1, c1.x, c1.y);
        mma_bf16(acc12[1], A1, c1.z, c1.w);
        mma_bf16(acc12[0], A2, c0.x, c0.y);
        mma_bf16(acc12[1], A2, c0.z, c0.w);
        if ((st + 1) % kSplitFlush == 0) {
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    accd[j][i] += (double)acc0[j][i];
                    acc0[j][i] = 0.0f;
                }
        }
    }
    cp_async_wait<0>();
    const long long ld = (long long)n_act * n_aux;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int P = P0 + 2 * g + ((i < 2) ? 0 : 1);
            const int a = 8 * j + 2 * q + (i & 1);
            if (P < n_aux && a < n_act)
                T[(long long)a * n_aux + P + (long long)mu * ld] = accd[j][i] + (double)acc0[j][i] + (double)acc12[j][i];
        }
}

// L[P, pair(a, b)] = sum_mu T[a, P, mu] C(mu, b) for b <= a.  CTA = (32 auxiliary rows, one
// orbital a); its four warps split the mu range (lane = auxiliary row, 16 accumulators for b)
// and reduce through shared memory.
__global__ void __launch_bounds__(128) second_index_kernel(const double* __restrict__ T, int n_aux, int n_bf,
                                                           const double* __restrict__ C, int n_act,
                                                           double* __restrict__ L) {
    __shared__ double red[4][kMaxActive][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int P = blockIdx.x * 32 + lane;
    const int a = blockIdx.y;
    const long long ld = (long long)n_act * n_aux;
    double acc[kMaxActive];
#pragma unroll
    for (int b = 0; b < kMaxActive; ++b) acc[b] = 0.0;
    const int chunk = (n_bf + 3) / 4;
    const int m0 = warp * chunk, m1 = min(n_bf, m0 + chunk);
    if (P < n_aux) {
        const double* t = T + (long long)a * n_aux + P;
#pragma unroll 4
        for (int m = m0; m < m1; ++m) {
            const double tv = __ldg(t + (long long)m * ld);
#pragma unroll
            for (int b = 0; b < kMaxActive; ++b)
                if (b <= a) acc[b] = fma(tv, __ldg(C + m + (long long)b * n_bf), acc[b]);
        }
    }
#pragma unroll
    for (int b = 0; b < kMaxActive; ++b) red[warp][b][lane] = acc[b];
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * kMaxActive; e += blockDim.x) {
        const int l = e % 32, b = e / 32;
        const int PP = blockIdx.x * 32 + l;
        if (b > a || PP >= n_aux) continue;
        L[PP + ao_pair(a, b) * n_aux] = red[0][b][l] + red[1][b][l] + red[2][b][l] + red[3][b][l];
    }
}

// K[pair(p, q)] = sum_P L[P, p] L[P, q] (q <= p): one warp per packed element.
__global__ void __launch_bounds__(256) pack_kernel(const double* __restrict__ L, int n_aux, int npair,
                                                   double* __restrict__ K) {
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long total = (long long)npair * (npair + 1) / 2;
    if (w >= total) return;
    int p = (int)((sqrt(8.0 * (double)w + 1.0) - 1.0) / 2.0);
    while ((long long)p * (p + 1) / 2 > w) --p;
    while ((long long)(p + 1) * (p + 2) / 2 <= w) ++p;
    const int q = (int)(w - (long long)p * (p + 1) / 2);
    const double* lp = L + (long long)p * n_aux;
    const double* lq = L + (long long)q * n_aux;
    double acc = 0.0;
    for (int P = lane; P < n_aux; P += 32) acc = fma(__ldg(lp + P), __ldg(lq + P), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) K[w] = acc;
}

// Adjoint.  With G = dE/dL and Gs[P, c, b] = G[P, pair(c, b)] (1 + delta_cb):
//   dE/dC(kappa, c) = sum_{P, b} Gs[P, c, b] T[b, P, kappa].
// adjoint_kernel: one CTA per (AO tile of 32, slice of the (b, P) range); partial sums go to
// a [slices x n_bf x n_act] buffer reduced in a fixed order by adjoint_reduce_kernel.
constexpr int kAdjSlices = 16;

__global__ void __launch_bounds__(256) adjoint_kernel(const double* __restrict__ T, const double* __restrict__ G,
                                                      int n_aux, int n_bf, int n_act, double* __restrict__ partial) {
    __shared__ double sT[32][33];   // [kappa local][k local]
    __shared__ double sG[32][kMaxActive + 1];  // [k local][c]
    const int k0_tile = blockIdx.x * 32;
    const int slice = blockIdx.y;
    const long long Ktot = (long long)n_act * n_aux;
    const long long per = (Ktot + kAdjSlices - 1) / kAdjSlices;
    const long long kb = slice * per, ke = min(Ktot, kb + per);
    const int tid = threadIdx.x;
    const int kl = tid & 31, cg = tid >> 5;  // thread: kappa local kl, c in {cg, cg + 8}
    double acc0 = 0.0, acc1 = 0.0;
    for (long long k0 = kb; k0 < ke; k0 += 32) {
        __syncthreads();
        for (int e = tid; e < 32 * 32; e += blockDim.x) {
            const int kk = e % 32, r = e / 32;
            const long long k = k0 + kk;
            const int kappa = k0_tile + r;
            sT[r][kk] = (k < ke && kappa < n_bf) ? __ldg(T + k + (long long)kappa * Ktot) : 0.0;
        }
        for (int e = tid; e < 32 * kMaxActive; e += blockDim.x) {
            const int kk = e % 32, c = e / 32;
            const long long k = k0 + kk;
            double g = 0.0;
            if (k < ke && c < n_act) {
                const int b = (int)(k / n_aux), P = (int)(k % n_aux);
                g = __ldg(G + P + ao_pair(c, b) * n_aux) * (c == b ? 2.0 : 1.0);
            }
            sG[kk][c] = g;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < 32; ++kk) {
            const double t = sT[kl][kk];
            acc0 = fma(t, sG[kk][cg], acc0);
            acc1 = fma(t, sG[kk][cg + 8], acc1);
        }
    }
    const int kappa = k0_tile + kl;
    if (kappa < n_bf) {
        double* out = partial + (long long)slice * n_bf * kMaxActive;
        out[(long long)kappa * kMaxActive + cg] = acc0;
        out[(long long)kappa * kMaxActive + cg + 8] = acc1;
    }
}

__global__ void adjoint_reduce_kernel(const double* __restrict__ partial, int n_bf, int n_act, double* __restrict__ dC) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_bf * n_act) return;
    const int kappa = e % n_bf, c = e / n_bf;
    double s = 0.0;
    for (int sl = 0; sl < kAdjSlices; ++sl) s += partial[(long long)sl * n_bf * kMaxActive + (long long)kappa * kMaxActive + c];
    dC[kappa + (long long)c * n_bf] = s;
}

size_t align_up(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace
}  // namespace vbcore

using namespace vbcore;

extern "C" {

vb_status vb_active_transform_ri(vb_context* ctx, const double* B_packed, int n_aux, int n_bf, const double* C,
                                 int n_act, int mem_space, double* one_index, double* L, double* K_packed) {
    return vb_active_transform_ri_precision(ctx, B_packed, n_aux, n_bf, C, n_act, VB_PRECISION_FP64, mem_space,
                                            one_index, L, K_packed);
}

vb_status vb_active_transform_ri_precision(vb_context* ctx, const double* B_packed, int n_aux, int n_bf,
                                           const double* C, int n_act, int precision, int mem_space,
                                           double* one_index, double* L, double* K_packed) {
    if (!ctx) return VB_ERR_INVALID;
    if (precision != VB_PRECISION_FP64 && precision != VB_PRECISION_BF16X3)
        return set_error(ctx, VB_ERR_INVALID, "vb_active_transform_ri: unknown precision");
    const bool split = precision == VB_PRECISION_BF16X3;
    const int split_steps = (n_bf + 15) / 16;
    if (split && split_steps > kSplitMaxSteps)
        return set_error(ctx, VB_ERR_UNSUPPORTED, "vb_active_transform_ri: split precision supports n_bf <= 1536");
    if (n_aux < 1 || n_bf < 1 || n_act < 1 || !B_packed || !C || !L)
        return set_error(ctx, VB_ERR_INVALID, "vb_active_transform_ri: dimensions must be positive, B, C and L non-null");
    if (n_act > kMaxActive)
        return set_error(ctx, VB_ERR_UNSUPPORTED, "vb_active_transform_ri: at most 16 active orbitals");
    if (mem_space != VB_MEM_HOST && mem_space != VB_MEM_DEVICE)
        return set_error(ctx, VB_ERR_INVALID, "bad memory space");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const bool host = mem_space == VB_MEM_HOST;
    const long long NP = (long long)n_bf * (n_bf + 1) / 2;
    const int npair = n_act * (n_act + 1) / 2;
    const size_t bB = sizeof(double) * (size_t)n_aux * NP, bC = sizeof(double) * (size_t)n_bf * n_act;
    const size_t bT = sizeof(double) * (size_t)n_act * n_aux * n_bf, bL = sizeof(double) * (size_t)n_aux * npair;
    const size_t bK = sizeof(double) * (size_t)npair * (npair + 1) / 2;
    size_t off = 0;
    auto take = [&](size_t bytes, bool need) {
        const size_t at = off;
        if (need) off = align_up(off + bytes);
        return at;
    };
    const size_t oB = take(bB, host), oC = take(bC, host), oT = take(bT, host || !one_index);
    const size_t oL = take(bL, host), oK = take(bK, host && K_packed);
    const bool pipelined = !split && n_aux % 2 == 0 && n_bf <= kPipelinedMaxBf &&
                           (host || reinterpret_cast<uintptr_t>(B_packed) % 16 == 0);
    const size_t oCt = take(sizeof(double) * (size_t)n_bf * kMaxActive, pipelined);
    const size_t oCf = take(sizeof(uint4) * (size_t)split_steps * 32 * 3, split);
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, off);
    if (st != VB_OK) return st;
    unsigned char* base = static_cast<unsigned char*>(ws.ptr);
    const double* dB = host ? reinterpret_cast<double*>(base + oB) : B_packed;
    const double* dC = host ? reinterpret_cast<double*>(base + oC) : C;
    double* dT = (host || !one_index) ? reinterpret_cast<double*>(base + oT) : one_index;
    double* dL = host ? reinterpret_cast<double*>(base + oL) : L;
    double* dK = host ? reinterpret_cast<double*>(base + oK) : K_packed;
    cudaError_t err = cudaSuccess;
    if (host) {
        err = cudaMemcpyAsync(const_cast<double*>(dB), B_packed, bB, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(const_cast<double*>(dC), C, bC, cudaMemcpyHostToDevice, s);
    }
    if (err == cudaSuccess) {
        const dim3 grid((n_bf + kWarpsPerCta - 1) / kWarpsPerCta, (n_aux + kAuxTile - 1) / kAuxTile);
        if (split) {
            uint4* Cf = reinterpret_cast<uint4*>(base + oCf);
            split_coefficients_kernel<<<(split_steps * 32 + 127) / 128, 128, 0, s>>>(dC, n_bf, n_act, split_steps, Cf);
            err = cudaGetLastError();
            const dim3 sgrid((n_bf + kSplitWarps - 1) / kSplitWarps, (n_aux + kSplitRows - 1) / kSplitRows);
            const bool ring = n_aux % 2 == 0 && (host || reinterpret_cast<uintptr_t>(B_packed) % 16 == 0);
            if (ring) {
                const size_t smem = split_pipelined_smem_bytes(split_steps);
                if (err == cudaSuccess) err = allow_dynamic_smem((const void*)one_index_split_pipelined_kernel, smem);
                if (err == cudaSuccess) {
                    one_index_split_pipelined_kernel<<<sgrid, 32 * kSplitWarps, smem, s>>>(dB, n_aux, n_bf, split_steps,
                                                                                          Cf, n_act, dT);
                    err = cudaGetLastError();
                }
            } else {
                const size_t smem = sizeof(uint4) * (size_t)split_steps * 32 * 3;
                if (err == cudaSuccess) err = allow_dynamic_smem((const void*)one_index_split_kernel, smem);
                if (err == cudaSuccess) {
                    one_index_split_kernel<<<sgrid, 32 * kSplitWarps, smem, s>>>(dB, n_aux, n_bf, split_steps, Cf,
                                                                                n_act, dT);
                    err = cudaGetLastError();
                }
            }
        } else if (pipelined) {
            double* Ct = reinterpret_cast<double*>(base + oCt);
            transpose_coefficients_kernel<<<(n_bf * kMaxActive + 255) / 256, 256, 0, s>>>(dC, n_bf, n_act, Ct);
            err = cudaGetLastError();
            const size_t smem = pipelined_smem_bytes(n_bf);
            if (n_bf <= kDmmaMaxBf) {
                // FP64 tensor cores, persistent CTAs (one per SM)
                const size_t dsmem = dmma_smem_bytes(n_bf);
                if (err == cudaSuccess) err = allow_dynamic_smem((const void*)one_index_dmma_kernel, (int)dsmem);
                int dev = 0, sms = 0;
                if (err == cudaSuccess) err = cudaGetDevice(&dev);
                if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                const long long items = (long long)((n_bf + kDmmaWarps - 1) / kDmmaWarps) *
                                        ((n_aux + kDmmaRows - 1) / kDmmaRows);
                const long long grid = items < sms ? items : sms;
                if (err == cudaSuccess) {
                    one_index_dmma_kernel<<<(unsigned)grid, 32 * kDmmaWarps, dsmem, s>>>(dB, n_aux, n_bf, Ct, n_act, dT);
                    err = cudaGetLastError();
                }
            } else {
            if (err == cudaSuccess)
                err = allow_dynamic_smem((const void*)one_index_pipelined_kernel, (int)smem);
            if (err == cudaSuccess) {
                const dim3 pgrid((n_bf + kPipeWarps - 1) / kPipeWarps, (n_aux + kAuxTile - 1) / kAuxTile);
                one_index_pipelined_kernel<<<pgrid, 32 * kPipeWarps, smem, s>>>(dB, n_aux, n_bf, Ct, n_act, dT);
                err = cudaGetLastError();
            }
            }
        } else {
            one_index_kernel<<<grid, 32 * kWarpsPerCta, 0, s>>>(dB, n_aux, n_bf, dC, n_act, dT);
            err = cudaGetLastError();
        }
    }
    if (err == cudaSuccess) {
        second_index_kernel<<<dim3((n_aux + 31) / 32, n_act), 128, 0, s>>>(dT, n_aux, n_bf, dC, n_act, dL);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess && K_packed) {
        const long long warps = (long long)npair * (npair + 1) / 2;
        pack_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(dL, n_aux, npair, dK);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess && host) {
        err = cudaMemcpyAsync(L, dL, bL, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess && K_packed) err = cudaMemcpyAsync(K_packed, dK, bK, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess && one_index) err = cudaMemcpyAsync(one_index, dT, bT, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    }
    if (err != cudaSuccess) return cuda_error(ctx, err, "vb_active_transform_ri");
    return VB_OK;  // device mode: stream-ordered (the workspace is freed in stream order)
}

vb_status vb_active_transform_ri_adjoint(vb_context* ctx, const double* one_index, const double* dL, int n_aux,
                                         int n_bf, int n_act, int mem_space, double* dC) {
    if (!ctx) return VB_ERR_INVALID;
    if (n_aux < 1 || n_bf < 1 || n_act < 1 || !one_index || !dL || !dC)
        return set_error(ctx, VB_ERR_INVALID, "vb_active_transform_ri_adjoint: bad arguments");
    if (n_act > kMaxActive)
        return set_error(ctx, VB_ERR_UNSUPPORTED, "vb_active_transform_ri_adjoint: at most 16 active orbitals");
    if (mem_space != VB_MEM_HOST && mem_space != VB_MEM_DEVICE)
        return set_error(ctx, VB_ERR_INVALID, "bad memory space");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const bool host = mem_space == VB_MEM_HOST;
    const int npair = n_act * (n_act + 1) / 2;
    const size_t bT = sizeof(double) * (size_t)n_act * n_aux * n_bf, bG = sizeof(double) * (size_t)n_aux * npair;
    const size_t bD = sizeof(double) * (size_t)n_bf * n_act;
    const size_t bP = sizeof(double) * (size_t)kAdjSlices * n_bf * kMaxActive;
    size_t off = 0;
    auto take = [&](size_t bytes, bool need) {
        const size_t at = off;
        if (need) off = align_up(off + bytes);
        return at;
    };
    const size_t oT = take(bT, host), oG = take(bG, host), oD = take(bD, host), oP = take(bP, true);
    DeviceBuffer ws;
    vb_status st = ws.allocate(ctx, off);
    if (st != VB_OK) return st;
    unsigned char* base = static_cast<unsigned char*>(ws.ptr);
    const double* dT = host ? reinterpret_cast<double*>(base + oT) : one_index;
    const double* dG = host ? reinterpret_cast<double*>(base + oG) : dL;
    double* dOut = host ? reinterpret_cast<double*>(base + oD) : dC;
    double* partial = reinterpret_cast<double*>(base + oP);
    cudaError_t err = cudaSuccess;
    if (host) {
        err = cudaMemcpyAsync(const_cast<double*>(dT), one_index, bT, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(const_cast<double*>(dG), dL, bG, cudaMemcpyHostToDevice, s);
    }
    if (err == cudaSuccess) {
        adjoint_kernel<<<dim3((n_bf + 31) / 32, kAdjSlices), 256, 0, s>>>(dT, dG, n_aux, n_bf, n_act, partial);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) {
        adjoint_reduce_kernel<<<(n_bf * n_act + 255) / 256, 256, 0, s>>>(partial, n_bf, n_act, dOut);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess && host) err = cudaMemcpyAsync(dC, dOut, bD, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess && host) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "vb_active_transform_ri_adjoint");
    return VB_OK;
}

}  // extern "C"
