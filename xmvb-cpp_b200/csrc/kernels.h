// Kernel argument blocks and launchers (pair_kernels.cu, assembly.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vbcore {

// One spin-string table and its unordered spin-pair records.
// Record of pair (u <= v), left = string u, right = string v, stride rec_stride doubles:
//   [r * k + c] first-order cofactor A(r, c) (rows = right), r, c < k (zero for nullity >= 2)
//   [k*k + 0] overlap determinant, [+1] same-spin H (1e + 2e), [+2] one-electron part,
//   [+3] nullity.
struct SpinTableArgs {
    int n;          // active orbitals
    int k;          // electrons of this spin
    int n_strings;  // N
    const uint64_t* occ;  // N x 2 words; byte i = i-th occupied orbital (ascending), 0xFF unused
    long long n_pairs;    // N (N + 1) / 2
    const double* S;      // n x n active overlap
    const double* h;      // n x n one-electron integrals
    const double* gamma;  // gd x gd antisymmetrized two-electron table (k >= 2)
    const double* eri;    // packed (ij|kl)
    int gamma_dim;        // n (n - 1) / 2
    double* records;
    int rec_stride;
    unsigned long long* careful_count;
    long long* careful_list;
    int all_careful;  // 1: every pair takes the exact path (list is implicit 0..n_pairs-1)
};

struct FullPairArgs {
    int n, ka, kb, np;  // np = n (n + 1) / 2
    long long n_det;
    const int* det_alpha;
    const int* det_beta;
    const uint64_t* occ_a;
    const uint64_t* occ_b;
    const double* rec_a;
    const double* rec_b;
    int stride_a, stride_b;
    const double* kfull;  // np x np unpacked pair kernel
    int kfull_in_smem;
    long long e0, e1;     // band columns [e0, e1)
    long long n_items;    // determinant pairs (d <= e) in the band
    double* Hb;           // band, row-major: Hb[d * (e1 - e0) + (e - e0)], valid for d <= e
    double* Sb;
};

struct BandReduceArgs {
    long long n_det;
    int n_str;
    long long e0, width;      // band columns
    const double* Hb;
    const double* Sb;
    const long long* woff;    // per (warp bucket, determinant) CSR offsets of this structure chunk
    const int* wstruct;
    const double* wcoef;
    int struct_begin, struct_count;
    double* Zh;  // n_str x n_det column-major: Z[e * n_str + I]
    double* Zs;
};

struct StructureReduceArgs {
    int n_str;
    long long n_det;
    const long long* str_off;  // CSC by structure
    const long long* str_det;
    const double* str_coef;
    const double* Zh;
    const double* Zs;
    double* Wh;  // n_str x n_str column-major
    double* Ws;
};

constexpr int kBandReduceWarps = 8;
constexpr int kBandReduceColumns = 32;

cudaError_t launch_prepare_tables(int n, const double* eri, double* gamma, double* kfull, cudaStream_t stream);
cudaError_t launch_spin_pairs(const SpinTableArgs& a, cudaStream_t stream, int* launches);
cudaError_t launch_full_pairs(const FullPairArgs& a, cudaStream_t stream, int* launches);
cudaError_t launch_band_reduce(const BandReduceArgs& a, cudaStream_t stream, int* launches);
cudaError_t launch_structure_reduce(const StructureReduceArgs& a, double* H, double* S, cudaStream_t stream,
                                    int* launches);
cudaError_t launch_listed_pairs(const FullPairArgs& a, long long n_pairs, const long long* pairs, double* h_out,
                                double* s_out, cudaStream_t stream);
cudaError_t launch_resolve_blocks(int k, long long batch, const double* blocks, double* det, int* nullity,
                                  double* cof, cudaStream_t stream);
cudaError_t launch_same_spin_list(int n, int k, long long batch, const int* occ_left, const int* occ_right,
                                  const double* S, const double* h, const double* eri, double* scalars, double* cof,
                                  cudaStream_t stream);
size_t band_reduce_smem_bytes(int struct_count);
int band_reduce_max_structures();

}  // namespace vbcore
