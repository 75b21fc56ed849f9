// Structure H/S assembly as HBM streams (sm_100a).
//
// The reference accumulates H_IJ = sum_{d in I, e in J} c_dI c_eJ H_de for left <= right
// structure pairs and mirrors the upper triangle (hamiltonian_overlap.cpp:437-450, 890-1022).
// Here the determinant matrix is symmetric and only its upper triangle is produced, in bands
// of columns, already weighted by the determinant-pair kernel (U' = upper triangle with halved
// diagonal, folded over the spin-flip symmetry when present), so that H_d = U' + U'^T and
//   Z  = T^T U'          (n_str x n_det; one streaming pass over every band, band_reduce)
//   W  = Z T             (n_str x n_str; structure_reduce)
//   H  = W + W^T         (symmetrize)
// Every sum runs in a fixed order (no atomics), so results are bitwise reproducible.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"
#include "kernels.h"

namespace vbcore {
namespace {

constexpr int kTileBytes = kBandTileRows * kBandColumns * 8;  // one band tile (H or S)
constexpr long long kDrainPolls = 1ll << 22;  // bound on waiting for copies in flight (~seconds)
constexpr int kZPad = kBandColumns + 1;

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// One poll of the phase with the given parity; the thread may sleep up to ~1 us inside it.
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n selp.u32 %0, 1, 0, "
        "p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase of `bar` with the given parity: false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_test(bar, parity)) return true;
    return false;
}

// TMA: a [kBandTileRows x kBandColumns] box of the band at (column x, row y); rows past n_det
// and columns past the band width arrive as zeros.
__device__ __forceinline__ void tma_band_tile(void* dst, const CUtensorMap* map, int x, int y,
                                              unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Contiguous bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// One CTA per (32 band columns, structure group of kBandGroup), heaviest column blocks first
// (a column block needs the band rows d <= its last column).  The rows stream through two
// shared-memory stages, each filled by TMA (the H and S tiles) and bulk copies (the tile's
// terms of this structure group), completion tracked by one mbarrier per stage.  Lane l owns
// band column l; warp w accumulates the kBandSlots structures s * kBandWarps + w of the group in
// registers, walking each structure's terms of the tile in determinant order, two per step.
// Tiles that reach below the diagonal have their entries d > e zeroed in shared memory first,
// so the term loop carries no mask.  The accumulators then pass through shared memory so that
// Z is written in coalesced runs of structures.
__global__ void __launch_bounds__(kBandWarps * 32, 3)
    band_reduce_kernel(const __grid_constant__ CUtensorMap map_h, const __grid_constant__ CUtensorMap map_s,
                       BandReduceArgs a, int stage_bytes) {
    extern __shared__ __align__(1024) unsigned char bsm_raw[];
    __shared__ __align__(8) unsigned long long full[2];
    // stages start on 1024-byte boundaries (TMA destinations; the launch adds the slack)
    unsigned char* bsm = bsm_raw + ((1024u - (smem_addr(bsm_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int G = a.n_groups;
    const long long nb = (a.width + kBandColumns - 1) / kBandColumns;
    const long long b = nb - 1 - (long long)blockIdx.x / G;
    const int g = (int)(blockIdx.x % G);
    const long long col0 = b * kBandColumns;
    long long rows = a.e0 + col0 + kBandColumns;
    if (rows > a.n_det) rows = a.n_det;
    const int ntiles = (int)((rows + kBandTileRows - 1) / kBandTileRows);
    const int seg_max = a.seg_max;
    // the group's row tiles with terms (ascending), up to the last one this column block reaches
    const int* tl = a.seg_tiles + a.seg_tile_off[g];
    int nt = a.seg_tile_off[g + 1] - a.seg_tile_off[g];
    {
        int lo = 0, hi = nt;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (tl[mid] < ntiles)
                lo = mid + 1;
            else
                hi = mid;
        }
        nt = lo;
    }

    // stage st <- the i-th listed tile
    auto issue = [&](int i, int st) {
        const int t = tl[i];
        unsigned char* base = bsm + (size_t)st * stage_bytes;
        const long long seg = (long long)g * a.n_tiles + t;
        const long long o0 = a.seg_off[seg];
        const unsigned len = (unsigned)(a.seg_off[seg + 1] - o0);
        mbar_expect_tx(&full[st], 2u * kTileBytes + 9u * len + kBandMetaBytes);
        tma_band_tile(base, &map_h, (int)col0, t * kBandTileRows, &full[st]);
        tma_band_tile(base + kTileBytes, &map_s, (int)col0, t * kBandTileRows, &full[st]);
        if (len) {
            bulk_load(base + 2 * kTileBytes, a.term_c + o0, 8u * len, &full[st]);
            bulk_load(base + 2 * kTileBytes + 8 * seg_max, a.term_d + o0, len, &full[st]);
        }
        bulk_load(base + 2 * kTileBytes + 9 * seg_max, a.seg_meta + seg * kBandMetaBytes, kBandMetaBytes, &full[st]);
    };

    if (tid == 0) {
        mbar_init(&full[0]);
        mbar_init(&full[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = 0;  // tiles issued so far (thread 0)
    if (tid == 0 && nt > 0) {
        issue(0, 0);
        if (nt > 1) issue(1, 1);
        issued = nt > 1 ? 2 : 1;
    }
    double acc_h[kBandSlots], acc_s[kBandSlots];
#pragma unroll
    for (int s = 0; s < kBandSlots; ++s) acc_h[s] = acc_s[s] = 0.0;

    // One barrier per tile: after computing tile t every thread waits for tile t + 1, and the
    // barrier then both releases stage t & 1 for refilling and confirms tile t + 1 landed.
    // polls of up to ~1 us each (0 when the context's limit is below 16: the first wait gives up
    // at once, which is how the timeout path is exercised)
    const long long limit = a.spin_limit / 16;
    bool ok = nt == 0 || __syncthreads_and(mbar_wait(&full[0], 0u, limit)) != 0;
    int i = 0;
    for (; ok && i < nt; ++i) {
        const int st = i & 1;
        unsigned char* base = bsm + (size_t)st * stage_bytes;
        const long long r0 = (long long)tl[i] * kBandTileRows;
        if (r0 + kBandTileRows - 1 > a.e0 + col0) {
            // rows below the diagonal of this column block hold no data: zero them
            double* zH = reinterpret_cast<double*>(base);
            double* zS = zH + kBandTileRows * kBandColumns;
            for (int i = tid; i < kBandTileRows * kBandColumns; i += blockDim.x) {
                const int dl = i / kBandColumns, l = i % kBandColumns;
                if (r0 + dl > a.e0 + col0 + l) {
                    zH[i] = 0.0;
                    zS[i] = 0.0;
                }
            }
            // these generic-proxy writes precede the stage's next TMA fill
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        }
        const double* tH = reinterpret_cast<const double*>(base);
        const double* tS = reinterpret_cast<const double*>(base + kTileBytes);
        const double* tc = reinterpret_cast<const double*>(base + 2 * kTileBytes);
        const unsigned char* td = base + 2 * kTileBytes + 8 * seg_max;
        const unsigned char* cnt = td + seg_max;
        int q = reinterpret_cast<const unsigned short*>(cnt + kBandWarps * kBandSlots)[warp];
#pragma unroll
        for (int s = 0; s < kBandSlots; ++s) {
            const int n = cnt[warp * kBandSlots + s];
            for (int i = 0; i < n; i += 2, q += 2) {
                const bool two = i + 1 < n;
                const int d0 = td[q], d1 = two ? td[q + 1] : d0;
                const double c0 = tc[q], c1 = two ? tc[q + 1] : 0.0;
                const double h0 = tH[d0 * kBandColumns + lane], h1 = tH[d1 * kBandColumns + lane];
                const double s0 = tS[d0 * kBandColumns + lane], s1 = tS[d1 * kBandColumns + lane];
                acc_h[s] = fma(c1, h1, fma(c0, h0, acc_h[s]));
                acc_s[s] = fma(c1, s1, fma(c0, s0, acc_s[s]));
            }
            q -= (n & 1);
        }
        const bool next = i + 1 >= nt || mbar_wait(&full[st ^ 1], (unsigned)((i + 1) >> 1) & 1u, limit);
        ok = __syncthreads_and(next) != 0;
        if (ok && tid == 0 && i + 2 < nt) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(i + 2, st);
            ++issued;
        }
    }
    if (!ok) {
        // a tile never landed: flag it, let the copies still in flight land (a generous bound of
        // its own: no copy may outlive the CTA), and leave
        if (tid == 0) {
            atomicExch(a.error, 1);
            for (int u = i; u < issued; ++u) mbar_wait(&full[u & 1], (unsigned)(u >> 1) & 1u, kDrainPolls);
        }
        __syncthreads();
        return;
    }
    double* zh = reinterpret_cast<double*>(bsm);
    double* zs = zh + kBandGroup * kZPad;
#pragma unroll
    for (int s = 0; s < kBandSlots; ++s) {
        const int li = s * kBandWarps + warp;
        zh[li * kZPad + lane] = acc_h[s];
        zs[li * kZPad + lane] = acc_s[s];
    }
    __syncthreads();
    const int gbegin = g * kBandGroup;
    const int gcount = min(kBandGroup, a.n_str - gbegin);
    for (int i = tid; i < gcount * kBandColumns; i += blockDim.x) {
        const int l = i / gcount, li = i - l * gcount;
        if (col0 + l >= a.width) break;
        const long long col = a.e0 + col0 + l;
        a.Zh[col * a.n_str + gbegin + li] = zh[li * kZPad + l];
        a.Zs[col * a.n_str + gbegin + li] = zs[li * kZPad + l];
    }
}

// W[I, J] = sum_{(e, c) in J} c Z[I, e]; one CTA per J, threads over I.  The terms of J are
// staged in shared memory 256 at a time, and each thread keeps eight Z loads in flight.
constexpr int kReduceTerms = 256;

__global__ void __launch_bounds__(512) structure_reduce_kernel(StructureReduceArgs a) {
    __shared__ long long se[kReduceTerms];
    __shared__ double sc[kReduceTerms];
    const int J = blockIdx.x;
    const long long t0 = a.str_off[J], t1 = a.str_off[J + 1];
    for (int I0 = 0; I0 < a.n_str; I0 += blockDim.x) {
        const int I = I0 + threadIdx.x;
        const bool valid = I < a.n_str;
        double wh0 = 0.0, wh1 = 0.0, ws0 = 0.0, ws1 = 0.0;
        for (long long c0 = t0; c0 < t1; c0 += kReduceTerms) {
            const int n = (int)(t1 - c0 < kReduceTerms ? t1 - c0 : kReduceTerms);
            __syncthreads();
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                se[q] = __ldg(a.str_det + c0 + q) * a.n_str;
                sc[q] = __ldg(a.str_coef + c0 + q);
            }
            __syncthreads();
            if (!valid) continue;
            int q = 0;
            for (; q + 8 <= n; q += 8) {
                double zh[8], zs[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    zh[u] = __ldg(a.Zh + se[q + u] + I);
                    zs[u] = __ldg(a.Zs + se[q + u] + I);
                }
#pragma unroll
                for (int u = 0; u < 8; u += 2) {
                    wh0 = fma(sc[q + u], zh[u], wh0);
                    ws0 = fma(sc[q + u], zs[u], ws0);
                    wh1 = fma(sc[q + u + 1], zh[u + 1], wh1);
                    ws1 = fma(sc[q + u + 1], zs[u + 1], ws1);
                }
            }
            for (; q < n; ++q) {
                wh0 = fma(sc[q], __ldg(a.Zh + se[q] + I), wh0);
                ws0 = fma(sc[q], __ldg(a.Zs + se[q] + I), ws0);
            }
        }
        if (valid) {
            a.Wh[(long long)J * a.n_str + I] = wh0 + wh1;
            a.Ws[(long long)J * a.n_str + I] = ws0 + ws1;
        }
    }
}

__global__ void symmetrize_kernel(int n, const double* __restrict__ Wh, const double* __restrict__ Ws,
                                  double* __restrict__ H, double* __restrict__ S) {
    const long long total = (long long)n * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long J = t / n, I = t % n;
        H[t] = Wh[t] + Wh[I * n + J];
        S[t] = Ws[t] + Ws[I * n + J];
    }
}

}  // namespace

static int band_stage_bytes(int seg_max) { return (2 * kTileBytes + 9 * seg_max + kBandMetaBytes + 1023) / 1024 * 1024; }

size_t band_reduce_smem_bytes(int seg_max) {
    const size_t stages = 2 * (size_t)band_stage_bytes(seg_max);
    const size_t z = 2 * sizeof(double) * kBandGroup * kZPad;
    return (stages > z ? stages : z) + 1024;  // + alignment slack
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

bool band_tensor_map(CUtensorMap* map, const double* band, long long width, long long n_det, long long ldb) {
    auto encode = tensor_map_encoder();
    if (!encode) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)n_det};
    const cuuint64_t strides[1] = {(cuuint64_t)ldb * sizeof(double)};
    const cuuint32_t box[2] = {(cuuint32_t)kBandColumns, (cuuint32_t)kBandTileRows};
    const cuuint32_t elem[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(band), dims, strides, box, elem,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

cudaError_t launch_band_reduce(const BandReduceArgs& a, cudaStream_t stream, int* launches) {
    if (a.width <= 0 || a.n_str <= 0) return cudaSuccess;
    if (a.ldb % 2 != 0 || (reinterpret_cast<uintptr_t>(a.Hb) & 15) || (reinterpret_cast<uintptr_t>(a.Sb) & 15))
        return cudaErrorInvalidValue;
    CUtensorMap mh, ms;
    if (!band_tensor_map(&mh, a.Hb, a.width, a.n_det, a.ldb) || !band_tensor_map(&ms, a.Sb, a.width, a.n_det, a.ldb))
        return cudaErrorInvalidValue;
    const size_t smem = band_reduce_smem_bytes(a.seg_max);
    cudaError_t err = allow_dynamic_smem((const void*)band_reduce_kernel, smem);
    if (err != cudaSuccess) return err;
    const long long blocks = (a.width + kBandColumns - 1) / kBandColumns * a.n_groups;
    band_reduce_kernel<<<(unsigned)blocks, kBandWarps * 32, smem, stream>>>(mh, ms, a, band_stage_bytes(a.seg_max));
    ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_structure_reduce(const StructureReduceArgs& a, double* H, double* S, cudaStream_t stream,
                                    int* launches) {
    int threads = (a.n_str + 31) / 32 * 32;
    threads = threads > 512 ? 512 : threads;
    structure_reduce_kernel<<<a.n_str, threads, 0, stream>>>(a);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    const long long total = (long long)a.n_str * a.n_str;
    long long blocks = (total + 255) / 256;
    if (blocks > 2048) blocks = 2048;
    symmetrize_kernel<<<(unsigned)blocks, 256, 0, stream>>>(a.n_str, a.Wh, a.Ws, H, S);
    *launches += 2;
    return cudaGetLastError();
}

}  // namespace vbcore
