// Kernel argument blocks and launchers (pair_kernels.cu, spin_frame.cu, assembly.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vbcore {

// Opposite-spin factorization of the pair kernel: K[p][q] = (p|q) over packed orbital pairs is
// written K = sum_m sigma_m l_m l_m^T (pivoted LDL^T, sigma = +1 for the first r_pos columns,
// -1 for the next r_neg), so the opposite-spin energy of a determinant pair
// sum A_a(r,c) A_b(r',c') (R_r L_c | R'_r' L'_c') becomes sum_m sigma_m u_a[m] u_b[m] with
// u[m] = sum_{r,c} A(r,c) l_m[pair(R_r, L_c)] computed once per spin pair.
//
// Spin-pair record of the unordered pair (u <= v) of one string table, left = string u, right =
// string v, at index u N - u (u - 1) / 2 + (v - u), stride rec_stride doubles:
//   [m] u-vector (m < R), [R + 0] overlap determinant, [R + 1] same-spin H (1e + 2e),
//   [R + 2] one-electron part, [R + 3] nullity.
struct SpinTableArgs {
    int n;          // active orbitals
    int k;          // electrons of this spin
    int n_strings;  // N
    const uint64_t* occ;  // N x 2 words; byte i = i-th occupied orbital (ascending), 0xFF unused
    long long n_pairs;    // N (N + 1) / 2
    const double* S;      // n x n active overlap
    const double* h;      // n x n one-electron integrals
    const double* gamma;  // gd x gd antisymmetrized table: gamma[rp * gd + cp] = (ij|kl) - (il|kj)
    const double* eri;    // packed (ij|kl)
    int gamma_dim;        // n (n - 1) / 2
    const double* lf;     // pair-kernel factor, lf[q * ld + m]
    int ld;               // leading dimension of lf (>= R)
    int R;                // number of factor columns
    double* records;
    int rec_stride;
    unsigned long long* careful_count;
    unsigned long long* careful_list;  // (u << 32) | v
    const int2* items;                 // fast-kernel work items: (left string u, first right string v0)
    int n_items;
    int all_careful;  // 1: every pair takes the exact path
    int r_pos;        // factor columns with sign +1 (the first r_pos of R)
    // frame kernel: right strings v >= u of each left string u at rlist[record_index(u, u)], bucketed
    // by hole set (excitation level first); ebound[u (k + 2) + e] = first position of level e
    const int* rlist;
    const unsigned* rdesc;  // per rlist entry: hole mask | particle mask << 8 | sign parity << 16
    const int* ebound;
    unsigned long long* task_counter;  // zero before the launch: left strings handed out so far
};

struct FullPairArgs {
    int ka, kb;
    long long n_det;
    const int* det_alpha;
    const int* det_beta;
    int Na, Nb;  // strings per table
    const double* rec_a;
    const double* rec_b;
    int stride_a, stride_b;
    int R, r_pos;         // factor columns, positive-sign columns
    long long e0, e1;     // band columns [e0, e1)
    long long n_items;    // determinant pairs (d <= e) in the band
    long long ldb;        // band row stride (elements, even: rows start on 16-byte boundaries)
    double* Hb;           // band, row-major: Hb[d * ldb + (e - e0)], valid for d <= e
    double* Sb;
    const int* flip;      // spin-flip permutation of determinants (nullptr: no folding)
};

// Band reduction Z = T^T U' (structure-major weights T, band U' upper triangle).  Rows of the
// band are streamed in tiles of kBandTileRows; for every (structure group g, row tile t) the plan
// holds one segment of (row-in-tile, coefficient) terms ordered by (warp, slot, determinant):
// seg_off[g T + t] (a multiple of 16) indexes term_c / term_d, and seg_meta holds kBandMetaBytes
// per segment: the term count of each (warp, slot) (kBandWarps x kBandSlots bytes) followed by the
// start of each warp's terms within the segment (kBandWarps uint16).  Structure of group g, warp
// w, slot s: I = g * kBandGroup + s * kBandWarps + w.
struct BandReduceArgs {
    long long n_det;
    int n_str;
    long long e0, width;      // band columns [e0, e0 + width)
    long long ldb;            // band row stride (elements, even)
    const double* Hb;
    const double* Sb;
    int n_groups, n_tiles;
    int seg_max;              // longest segment (terms, a multiple of 16)
    const long long* seg_off;
    const unsigned char* seg_meta;
    const double* term_c;
    const unsigned char* term_d;
    const int* seg_tiles;     // row tiles whose segment has terms, per group ascending
    const int* seg_tile_off;  // group g: seg_tiles[seg_tile_off[g] .. seg_tile_off[g + 1])
    double* Zh;  // n_str x n_det column-major: Z[e * n_str + I]
    double* Zs;
    int* error;  // set to 1 when a tile wait gives up (the results are then incomplete)
    long long spin_limit;
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

// Conditioning certificate of the register-resident spin-pair paths: a block is evaluated there
// only if ||X||_F^2 ||X^-1||_F^2 < kCertificate2, i.e. kappa_F < 1e8.  The last pivot of any LU
// of X is 1 / (an entry of the permuted X^-1) >= 1 / ||X^-1||_F and the first complete-pivoting
// pivot is max|x_ij| <= ||X||_F, so the smallest pivot ratio of the reference's complete-pivoting
// LU stays >= ~1 / (c_k kappa_F) with c_k modest for k <= 16: far above its 1e-12 rank threshold,
// so these blocks are full rank under the reference semantics.  Others take the exact path.
constexpr double kCertificate2 = 1.0e16;

constexpr int kBandWarps = 8;        // warps per band-reduction CTA
constexpr int kBandSlots = 8;        // structures per warp (register accumulators)
constexpr int kBandGroup = kBandWarps * kBandSlots;
constexpr int kBandColumns = 32;     // band columns per CTA (one per lane)
constexpr int kBandTileRows = 64;    // band rows per staged tile
constexpr int kBandMetaBytes = kBandWarps * kBandSlots + 2 * kBandWarps;
constexpr int kSpinBlock = 128;    // right strings per fast-kernel item (threads per CTA)

// Per-thread stack frames of the exact-path kernels instantiated for k <= 8 (reserved when a
// context is created; the k <= 16 instantiations, about four times larger, grow the reservation
// at their first launch).
size_t exact_stack_bytes();
size_t gradient_stack_bytes();

cudaError_t launch_prepare_tables(int n, const double* eri, double* gamma, double* kfull, cudaStream_t stream);
cudaError_t launch_factor_pair_kernel(int np, const double* kfull, double* work, double* cols, int* signs,
                                      double* lf, int ld, int* meta, cudaStream_t stream);
// Spin-pair records of one string table: the per-left-string frame tables first
// (launch_spin_tables, nothing when the register path does not apply), then launch_spin_pairs
// (the frame kernel, listing the blocks it cannot certify) and launch_spin_pairs_exact.
cudaError_t launch_spin_tables(const SpinTableArgs& a, double* tables, cudaStream_t stream, int* launches);
cudaError_t launch_spin_pairs(const SpinTableArgs& a, double* tables, cudaStream_t stream, int* launches);
// The exact path of one string table: the blocks launch_spin_pairs listed, or every block when the
// register path does not apply.
cudaError_t launch_spin_pairs_exact(const SpinTableArgs& a, cudaStream_t stream, int* launches);
// Frame kernels (spin_frame.cu): per-left-string block size, the envelope of the register path,
// the once-per-table bucketing of right strings, and the table and pair launches.
size_t frame_table_doubles(int n, int k, int R);
bool frame_spin_supported(int n, int k, int R);
cudaError_t launch_sort_right_strings(int k, int N, const uint64_t* occ, int* rlist, unsigned* rdesc, int* ebound,
                                      cudaStream_t stream);
cudaError_t launch_frame_tables(const SpinTableArgs& a, double* tables, cudaStream_t stream);
int frame_pair_variants(int n, int k, int R);
cudaError_t launch_frame_pairs(const SpinTableArgs& a, const double* tables, cudaStream_t stream, int variant);
cudaError_t preload_frame_kernels();
// Loads every kernel launch_spin_pairs and its table steps may use (under lazy module loading a
// kernel is otherwise loaded, and its code placed in device memory, at its first launch).
cudaError_t preload_spin_pair_kernels();
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
// FP64 tensor-core contractions over the pair-kernel factor columns (dgemm.cu):
//   launch_factor_project: C[q + c ldC] = sum_m lf[q ld + m] Y[m + c ldY]     (np x cnt)
//   launch_factor_outer:   G[m + q ldG] += sum_c Y[m + c ldY] Z[q + c ldZ]    (R x np); `partial`
//   holds kOuterMaxParts R np doubles of split-K partials, summed in a fixed order.
bool factor_contractions_supported(int np, int R);
cudaError_t launch_factor_project(int np, int R, const double* lf, int ld, const double* Y, long long ldY,
                                  long long cnt, double* C, long long ldC, cudaStream_t stream);
constexpr int kOuterMaxParts = 4 * 148;
cudaError_t launch_factor_outer(int np, int R, const double* Y, long long ldY, const double* Z, long long ldZ,
                                long long cnt, double* G, long long ldG, double* partial, cudaStream_t stream);
// Dynamic shared memory of the band reduction for segments of at most seg_max terms.
size_t band_reduce_smem_bytes(int seg_max);

}  // namespace vbcore
