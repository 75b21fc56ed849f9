/*
 * vbcore: B200-native (sm_100a) VBSCF evaluation core behind a C ABI.
 *
 * Drop-in boundary for the determinant-pair / structure-matrix hot path of
 * Tao-Xia/xmvb-cpp (paths below are relative to that project).  Every entry
 * point names the reference interface it replaces.  Conventions:
 *
 *   - all matrices are column-major (m[col * rows + row]), as the reference's
 *     src/vbscf/determinants/contracts/types.hpp:13-15;
 *   - determinant overlap blocks have rows = right determinant, columns = left
 *     determinant (types.hpp:62-66); cofactor matrices use the same orientation;
 *   - packed pair index pair(a,b) = hi(hi+1)/2 + lo and packed two-electron
 *     storage (pq|rs) at pair(pair(p,q), pair(r,s)) (src/core/pair_index.cpp:10-44);
 *   - status codes instead of exceptions; vb_last_error() gives the message;
 *   - caller-owned buffers; VB_MEM_HOST pointers are copied through the
 *     context's stream, VB_MEM_DEVICE pointers are used in place.
 *
 * There is no CPU fallback: every numerical entry point runs CUDA kernels and
 * fails with VB_ERR_CUDA when no usable sm_100 device is present.
 */
#ifndef VBCORE_H
#define VBCORE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int vb_status;
enum {
    VB_OK = 0,
    VB_ERR_INVALID = 1,     /* bad argument or shape (reference: std::invalid_argument) */
    VB_ERR_CUDA = 2,        /* CUDA runtime failure (reference: check_cuda, context.hpp:20-37) */
    VB_ERR_BUDGET = 3,      /* HBM budget exceeded (reference: context.hpp:213-218) */
    VB_ERR_NUMERIC = 4,     /* non-SPD metric, failed eigensolve (reference: cholesky check_info) */
    VB_ERR_UNSUPPORTED = 5, /* size outside what the kernels implement */
    VB_ERR_TIMEOUT = 6      /* a bounded device wait gave up */
};

enum { VB_MEM_HOST = 0, VB_MEM_DEVICE = 1 };

typedef struct vb_context vb_context;
typedef struct vb_hs_plan vb_hs_plan;

/* ---- context (replaces xmvb::cuda::Context, src/cuda/memory/context.hpp:66-405) ---------- */

/* Create a context on `device` with an HBM byte budget (0 = 90 % of free memory, as
 * context.hpp:68-104).  The context owns one non-blocking stream unless one is attached. */
vb_status vb_context_create(int device, size_t hbm_budget_bytes, vb_context** out);
vb_status vb_context_destroy(vb_context* ctx);
/* Use the caller's cudaStream_t for all work of this context (NULL restores its own).  Waits
 * for the work already queued on the previous stream (the context's scratch memory is reused in
 * stream order). */
vb_status vb_context_set_stream(vb_context* ctx, void* cuda_stream);
vb_status vb_context_synchronize(vb_context* ctx);
/* Polls a grid-barrier wait of the cooperative eigensolver kernels (vb_generalized_eigh, and
 * vb_metric_cholesky up to n = 96; the blocked Cholesky used above that size and for the Davidson
 * shift-invert factor has no grid barrier) makes before it gives up: the kernel
 * then ends and the call returns VB_ERR_TIMEOUT, with the context still usable.  0 restores the
 * built-in default (2^26 polls, seconds).  No reference counterpart: the reference's solvers are
 * library calls (dsygvd) without a device-side wait. */
vb_status vb_context_set_barrier_spin_limit(vb_context* ctx, long long polls);
/* Last error message of this context (or of the last failed create when ctx is NULL). */
const char* vb_last_error(const vb_context* ctx);
/* Bytes currently allocated by the context and the peak (reference: gpu_peak_device_bytes,
 * src/cli/cuvbscf.cpp:121-190). */
vb_status vb_context_memory(const vb_context* ctx, size_t* current_bytes, size_t* peak_bytes);

/* ---- structure generation and expansion (host) ------------------------------------------- */

/* Structure-class generation: keyword as the deck's STR= value ("COV", "ION(1)", "COV ION(1)",
 * "FULL").  Replaces build_generated_raw_structures_from_structure_class
 * (src/input/loading/generated_structures.cpp:674-716).  rows_out (nullable) receives
 * n_structures x (n_active_electrons + 2 n_inactive) 1-based orbital labels, row-major. */
vb_status vb_generate_structures(const char* keyword, int n_active_orbitals, int n_active_electrons,
                                 int spin_multiplicity, int n_inactive, int64_t* n_structures_out,
                                 int32_t* rows_out, int64_t rows_capacity);

/* Determinant expansion of raw structures (StructureExpander::expand,
 * src/vbscf/structures/expansion/expander.cpp:287-557).  Two-call protocol: call with NULL
 * outputs to get the sizes, then with buffers.  Strings are occupation bit masks sorted
 * ascending; determinants are ordered by (alpha rank, beta rank); terms are CSR by determinant
 * with +-1 coefficients. */
typedef struct {
    int32_t n_structures;
    int32_t n_alpha_electrons;
    int32_t n_beta_electrons;
    int32_t n_alpha_strings;
    int32_t n_beta_strings;
    int64_t n_determinants;
    int64_t n_terms;
} vb_expansion_sizes;

vb_status vb_expand_structures(const int32_t* rows, int64_t n_structures, int n_active_electrons,
                               int spin_multiplicity, int n_inactive, vb_expansion_sizes* sizes,
                               uint64_t* alpha_strings, uint64_t* beta_strings, int32_t* det_alpha,
                               int32_t* det_beta, int64_t* term_offsets, int32_t* term_structure,
                               double* term_coefficient);

/* ---- structure Hamiltonian / overlap (the determinant-pair hot path) --------------------- */

/* A plan holds the orbital-independent topology on the device (string tables, determinant
 * list, incidence) and the scratch for the spin-pair records, so repeated evaluations at new
 * orbitals (every optimizer trial) re-upload nothing but S, h and (ij|kl).  It replaces
 * FullDeterminantStructureHamiltonianOverlapBuilder::build
 * (src/vbscf/structures/assembly/hamiltonian_overlap.hpp:70-107) with
 * DeterminantPairEvaluator::{evaluate_same_spin_pair, combine_spin_pair_evaluations}
 * (src/vbscf/determinants/pairs/evaluator.hpp:81-154) as its inner kernels. */
typedef struct {
    int32_t n_orbitals;
    int32_t n_alpha_electrons;
    int32_t n_beta_electrons;
    int32_t n_alpha_strings;
    int32_t n_beta_strings;
    const uint64_t* alpha_strings; /* host, sorted ascending occupation masks */
    const uint64_t* beta_strings;
    int64_t n_determinants;
    const int32_t* det_alpha; /* host, string index per determinant */
    const int32_t* det_beta;
    int32_t n_structures;
    const int64_t* term_offsets; /* host CSR by determinant, n_determinants + 1 */
    const int32_t* term_structure;
    const double* term_coefficient;
} vb_expansion;

vb_status vb_hs_plan_create(vb_context* ctx, const vb_expansion* expansion, vb_hs_plan** out);
vb_status vb_hs_plan_destroy(vb_hs_plan* plan);

/* Evaluate H and S (n_structures^2 each, column-major, symmetric).  Inputs: active overlap
 * S_act (n x n), one-electron h (n x n), packed (ij|kl) of length P(P+1)/2 with
 * P = n(n+1)/2.  mem_space says where all five pointers live.  Stream-ordered; with
 * VB_MEM_HOST the call returns after the results are on the host. */
vb_status vb_hs_plan_execute(vb_hs_plan* plan, const double* ovlp_act, const double* h1e_act,
                             const double* eri_packed, int mem_space, double* hamiltonian_out,
                             double* overlap_out);

/* Diagnostics of the last execute: spin pairs evaluated, pairs routed to the exact
 * full-pivot/SVD path, unordered determinant pairs evaluated (with alpha/beta-exchange
 * symmetry one pair per orbit {(d, e), (flip d, flip e)}), kernel launches, and the number of
 * columns of the pivoted LDL^T factorization of the pair kernel (ij|kl) (its numerical rank). */
typedef struct {
    int64_t spin_pairs;
    int64_t careful_spin_pairs;
    int64_t determinant_pairs;
    int64_t kernel_launches;
    int64_t factor_columns;
} vb_hs_stats;
vb_status vb_hs_plan_stats(const vb_hs_plan* plan, vb_hs_stats* stats);

/* Phase timing with CUDA events on the context stream (the device counterpart of the
 * reference's XMVB_PHASE_TIMING scoped phases, src/core/timing.hpp:411).  When enabled, every
 * execute records events around its phases; vb_hs_plan_phase_times synchronizes and returns
 * the milliseconds of the last execute per phase: [0] integral tables (pair-kernel factorization
 * and the per-left-string frame tables), [1] spin-pair records of the register path (frame
 * kernel), [2] determinant pairs (all bands), [3] band reduction, [4] structure reduction +
 * symmetrization, [5] spin-pair records of the exact path (listed blocks).  Phases [2] and [3] sum over bands. */
enum { VB_PHASE_TABLES = 0, VB_PHASE_SPIN_PAIRS = 1, VB_PHASE_DETERMINANT_PAIRS = 2, VB_PHASE_BAND_REDUCE = 3,
       VB_PHASE_STRUCTURE_REDUCE = 4, VB_PHASE_EXACT_PAIRS = 5, VB_PHASE_COUNT = 6 };
vb_status vb_hs_plan_enable_phase_timing(vb_hs_plan* plan, int enable);
vb_status vb_hs_plan_phase_times(vb_hs_plan* plan, double* milliseconds, int count);

/* ---- determinant-pair level entry points ---------------------------------------------------- */

/* Batched overlap resolution (DeterminantOverlapResolver::resolve_matrix,
 * src/vbscf/determinants/algebra/overlap.hpp:53, overlap.cpp:50-109) plus the first-order
 * cofactor matrix (build_first_order_cofactor_matrix, contractions.cpp:172-237).
 * blocks: batch x k x k column-major; out det[batch], nullity[batch], cofactor (batch x k x k,
 * zero for nullity >= 2).  mem_space applies to all pointers. */
vb_status vb_resolve_overlaps(vb_context* ctx, int k, int64_t batch, const double* blocks, int mem_space,
                              double* det_out, int32_t* nullity_out, double* cofactor_out);

/* Same-spin pair evaluation for explicit (left, right) occupied lists
 * (DeterminantPairEvaluator::evaluate_same_spin_pair, evaluator.cpp:297-352).
 * occ_left/occ_right: batch x k int32 orbital indices (ascending).  out_scalars: batch x 4
 * {det, one-electron H, total same-spin H, nullity}; cofactor_out (nullable): batch x k x k. */
vb_status vb_same_spin_pairs(vb_context* ctx, int n_orbitals, int k, int64_t batch, const int32_t* occ_left,
                             const int32_t* occ_right, const double* ovlp_act, const double* h1e_act,
                             const double* eri_packed, int mem_space, double* out_scalars,
                             double* cofactor_out);

/* Full determinant pairs <left|H|right>, <left|right> for a plan's determinant list
 * (DeterminantPairEvaluator::evaluate, evaluator.cpp:421-466): pairs[2*i] = left index,
 * pairs[2*i+1] = right index.  Outputs H and S per pair. */
vb_status vb_hs_plan_determinant_pairs(vb_hs_plan* plan, const double* ovlp_act, const double* h1e_act,
                                       const double* eri_packed, int64_t n_pairs, const int64_t* pairs,
                                       int mem_space, double* h_out, double* s_out);

/* Analytic gradient of a structure root (accumulate_active_space_gradient and its same-spin /
 * opposite-spin backward parts, src/vbscf/derivatives/gradient/active_space/
 * evaluator.cpp:1046-1133).  With c = structure_coefficients (the S-normalized eigenvector of
 * `eigenvalue`), the gradient of E = c^T (H - eigenvalue S) c, which equals the root's
 * derivative, with respect to the plan inputs at (S, h, eri):
 *   dS_out, dh_out (n x n, symmetric: dE = sum_ij G_ij dS_ij for symmetric perturbations),
 *   deri_out (packed, derivative per stored element; NULL to skip; needs a full-rank pair
 *     kernel, else VB_ERR_UNSUPPORTED),
 *   dri_out (np x n_aux, column-major, np = n(n+1)/2) = dE/dF when the integrals are
 *     (ij|kl) = sum_c F[pair(i,j)][c] F[pair(k,l)][c] with ri_factors = F (NULL to skip).
 * Re-evaluates the spin-pair records of (S, h, eri); synchronizes the context stream. */
vb_status vb_hs_plan_gradient(vb_hs_plan* plan, const double* ovlp_act, const double* h1e_act,
                              const double* eri_packed, int mem_space, const double* structure_coefficients,
                              double eigenvalue, double* dS_out, double* dh_out, double* deri_out,
                              const double* ri_factors, int n_aux, double* dri_out);

/* One structure-space evaluation with H and S kept on the device: the plan at host inputs
 * (S, h, eri as for vb_hs_plan_execute), its lowest root (dense solver up to 200 structures,
 * else the Davidson iteration of vb_lowest_root with `tolerance`) and, when dS_out and dh_out
 * are given, the root's gradient as vb_hs_plan_gradient (reusing the spin-pair records).
 * energy: the root (no nuclear term); coefficients (n_str, may be NULL): its S-normalized
 * eigenvector.  The selected-root solve and gradient accumulation of one trial point
 * (solve_structure_problem, src/vbscf/derivatives/gradient/active_space/evaluator.cpp:466-560,
 * and accumulate_active_space_gradient, :1046-1133).  Host buffers; synchronizes. */
vb_status vb_hs_plan_root_gradient(vb_hs_plan* plan, const double* ovlp_act, const double* h1e_act,
                                   const double* eri_packed, double tolerance, double* energy,
                                   double* coefficients, double* dS_out, double* dh_out, const double* ri_factors,
                                   int n_aux, double* dri_out);

/* ---- metric Cholesky and the structure eigenproblem ------------------------------------------- */

/* Upper Cholesky factor S = U^T U of a symmetric positive-definite metric
 * (overlap_upper, src/vbscf/orbitals/preparation/cholesky.hpp:10-15, Eigen::LLT; also the
 * first stage of dsygvd).  Only the upper triangle of S is read; upper_out (n x n,
 * column-major) receives U with zeros below the diagonal and may alias S.  A non-positive (or
 * non-finite) pivot returns VB_ERR_NUMERIC with *info = order of that leading minor. */
vb_status vb_metric_cholesky(vb_context* ctx, const double* S, int n, int mem_space, double* upper_out, int* info);

/* H C = S C E, LAPACK dsygvd(itype 1, 'V', 'U') semantics as called by
 * GeneralizedEigensolver::solve_dense (src/linalg/eigensolver.cpp:365-388): upper triangles of
 * H and S read, eigenvalues ascending, eigenvectors column-major with C^T S C = I.  S not
 * positive definite: VB_ERR_NUMERIC with *info = n + i (i = order of the failing leading
 * minor), the reference's "overlap_matrix is not positive definite" (eigensolver.cpp:39-49).
 * Synchronizes the context stream. */
vb_status vb_generalized_eigh(vb_context* ctx, const double* H, const double* S, int n, int mem_space,
                              double* eigenvalues, double* eigenvectors, int* info);

/* Lowest root only, by a generalized Davidson iteration on the device (the selected-root
 * structure solve of solve_structure_problem, src/vbscf/derivatives/gradient/active_space/
 * evaluator.cpp:466-560; GeneralizedEigensolver::solve_davidson, src/linalg/eigensolver.hpp:
 * 194-198) for structure spaces too large for the dense solver.  Converged when
 * ||H c - E S c||_2 <= tolerance (||H c|| + |E| ||S c||); eigenvector S-normalized (sign
 * arbitrary).
 * VB_ERR_NUMERIC when max_iterations pass without convergence. */
vb_status vb_lowest_root(vb_context* ctx, const double* H, const double* S, int n, int mem_space, double tolerance,
                         int max_iterations, double* eigenvalue, double* eigenvector, int* iterations);

/* `count` independent problems in device memory (one CTA each): problem b has dimension
 * dims[b], H, S and eigenvectors at element offset offsets[b], eigenvalues at
 * value_offsets[b]; info[b] (host) = 0, n + i (S not positive definite) or -1 (no
 * convergence).  Returns the first failure as VB_ERR_NUMERIC. */
vb_status vb_generalized_eigh_batched(vb_context* ctx, int count, const int* dims, const int64_t* offsets,
                                      const double* H, const double* S, int mem_space, double* eigenvalues,
                                      const int64_t* value_offsets, double* eigenvectors, int* info);

/* ---- VBSCF energy, gradient and orbital optimization ------------------------------------------ */

/* A molecule with s-type contracted Gaussian shells (hydrogen 6-31G and the like), active
 * orbitals restricted to listed basis functions (the deck's fragment/HAO pattern), and a
 * structure class.  Replaces the host side of run_cuvbscf -> xmvb::cuda::solve_scf
 * (src/cli/cuvbscf.cpp:31, src/cuda/vb/scf.hpp:41-46) for this basis family. */
typedef struct vb_scf_problem vb_scf_problem;
typedef struct {
    int32_t n_atoms;
    const double* charges;            /* n_atoms */
    const double* coords;             /* n_atoms x 3, bohr */
    int32_t n_shells;                 /* one basis function per s shell */
    const int32_t* shell_atom;
    const int32_t* shell_nprim;
    const double* shell_exponents;    /* concatenated primitives */
    const double* shell_coefficients; /* for normalized primitives (basis-file convention) */
    int32_t n_active;
    const int32_t* orbital_offsets;   /* CSR: basis functions orbital a may use */
    const int32_t* orbital_functions;
    int32_t n_electrons;
    int32_t multiplicity;
    const char* structures;           /* STR= keyword, e.g. "COV" */
} vb_scf_input;

typedef struct {
    int32_t max_iterations;
    double gradient_tolerance;  /* on the infinity norm of the coefficient gradient */
    int32_t history_size;       /* secant pairs kept */
    double armijo;              /* sufficient-decrease constant */
} vb_scf_options;

typedef struct {
    double energy;
    double gradient_inf;
    int32_t iterations;
    int32_t evaluations;
    int32_t converged;
} vb_scf_result;

/* Host only (no device needed): the AO integrals of the input's shells and the nuclear
 * repulsion; S_ao, h_ao n_bf x n_bf, eri_ao n_bf^4 (any may be NULL). */
vb_status vb_ao_integrals_s(const vb_scf_input* input, double* S_ao, double* h_ao, double* eri_ao,
                            double* nuclear_repulsion);
vb_status vb_scf_problem_create(vb_context* ctx, const vb_scf_input* input, vb_scf_problem** problem);
/* The same problem from AO integrals the caller already has (the reference computes them with
 * libcint and hands them to xmvb::cuda::solve_scf(Context&, const VbScfInput&, AoPairGraph&&,
 * double nuclear_repulsion, const VbScfOptimizerOptions&, observe), src/cuda/vb/scf.hpp:41-46):
 * any basis (s, p, d ...), the AO overlap and core Hamiltonian, and the two-electron integrals as
 * the AoPairGraph's unique-integral stream (src/integrals/ao/input.hpp:36-60): AO pairs
 * (pair_first[p], pair_second[p]) and entries (integral_rows[t], integral_columns[t],
 * integral_values[t]) = (pair row | pair column), each unordered pair of pairs once; absent
 * entries are zero.  The pair matrix is factored once by pivoted Cholesky (to 1e-15 of its
 * largest diagonal), so every evaluation runs the device RI path.  Host buffers, copied. */
typedef struct {
    int32_t n_basis;
    const double* S_ao;  /* n_bf x n_bf, column-major */
    const double* h_ao;  /* core Hamiltonian, n_bf x n_bf */
    int64_t n_pairs;
    const int32_t* pair_first;
    const int32_t* pair_second;
    int64_t n_integrals;
    const int64_t* integral_rows;
    const int64_t* integral_columns;
    const double* integral_values;
    double nuclear_repulsion;
    int32_t n_active;
    const int32_t* orbital_offsets; /* CSR: basis functions orbital a may use */
    const int32_t* orbital_functions;
    int32_t n_electrons;
    int32_t multiplicity;
    const char* structures;         /* STR= keyword, e.g. "COV" */
} vb_scf_integral_input;
vb_status vb_scf_problem_create_from_integrals(vb_context* ctx, const vb_scf_integral_input* input,
                                               vb_scf_problem** problem);
vb_status vb_scf_problem_destroy(vb_scf_problem* problem);
vb_status vb_scf_problem_sizes(const vb_scf_problem* problem, int* n_basis, int* n_active, int* n_structures,
                               double* nuclear_repulsion);
/* AO overlap, core Hamiltonian (n_bf x n_bf) and full (mu nu|la si) (n_bf^4), host buffers
 * (for a problem built from AO integrals, the two-electron integrals of its pair factors). */
vb_status vb_scf_ao_integrals(const vb_scf_problem* problem, double* S_ao, double* h_ao, double* eri_ao);
/* Total energy at coefficients C (n_bf x n_act, column-major, entries outside each orbital's
 * basis functions ignored), and optionally dE/dC (same shape, zero outside the pattern) and
 * the structure H/S (n_str^2 each). */
vb_status vb_scf_energy_gradient(vb_scf_problem* problem, const double* coefficients, double* energy,
                                 double* gradient, double* hamiltonian_out, double* overlap_out);
/* Limited-memory quasi-Newton (two-loop recursion, scaled identity initial inverse, Armijo
 * backtracking) over the allowed coefficients, the P-LBFGS backend's scheme
 * (run_plbfgs_backend, src/vbscf/optimization/backends/plbfgs.cpp:19-228). */
vb_status vb_solve_scf(vb_scf_problem* problem, const double* initial_coefficients, const vb_scf_options* options,
                       vb_scf_result* result, double* coefficients_out);
/* Precision of the per-evaluation RI transform in vb_solve_scf (no counterpart in the reference,
 * which is FP64 only).  VB_PRECISION_BF16X3: the solve evaluates with the split-precision
 * transform (vb_active_transform_ri_precision) while the gradient's infinity norm is above
 * switch_gradient, then re-evaluates the current point in FP64, drops its secant history and
 * finishes in FP64, so the converged point and energy are those of an FP64 solve to the
 * gradient tolerance.  VB_PRECISION_FP64 (default) uses FP64 throughout.  *split_evaluations
 * (vb_scf_problem_split_evaluations) counts the split-precision evaluations of the last solve. */
vb_status vb_scf_problem_set_precision(vb_scf_problem* problem, int precision, double switch_gradient);
vb_status vb_scf_problem_split_evaluations(const vb_scf_problem* problem, int32_t* split_evaluations);

/* ---- batched and served work ------------------------------------------------------------------ */

/* An engine: n_workers host workers, each with its own context (stream, memory pool), sharing
 * one GPU.  No counterpart in the reference (one instance per process); requests mirror its
 * solve entry point (xmvb::cuda::solve_scf, src/cuda/vb/scf.hpp:41-46). */
typedef struct vb_engine vb_engine;
vb_status vb_engine_create(int device, size_t hbm_budget_bytes, int n_workers, vb_engine** engine);
vb_status vb_engine_destroy(vb_engine* engine);
const char* vb_engine_last_error(const vb_engine* engine);

/* Batched form: register an active-space instance (its plan stays on the device, assigned to
 * the least-loaded worker); not concurrent with evaluate. */
vb_status vb_engine_add_instance(vb_engine* engine, const vb_expansion* expansion, int64_t* instance_id);
/* Energy (lowest structure root, no nuclear term) and, when dS/dh are given, its gradient with
 * respect to S, h and the RI factors (ri_factors[i]: n(n+1)/2 x n_aux[i], column-major; NULL
 * entries skip) for every listed instance; host buffers; returns when all are done. */
vb_status vb_engine_evaluate_instances(vb_engine* engine, int count, const int64_t* ids, const double* const* S,
                                       const double* const* h, const double* const* eri,
                                       const double* const* ri_factors, const int* n_aux, double* energies,
                                       double* const* dS, double* const* dh, double* const* dri);

/* Serving: queue a VBSCF solve (copied); admitted first-in first-out when the HBM budget holds
 * its estimated footprint (or when nothing else runs). */
vb_status vb_engine_submit_scf(vb_engine* engine, const vb_scf_input* input, const double* initial_coefficients,
                               const vb_scf_options* options, int64_t tag);
/* Up to `capacity` completed solves (wait != 0: block until one completes or all are done):
 * tag, total energy, gradient infinity norm, iterations, converged, status, seconds queued and
 * seconds from submission to completion. */
vb_status vb_engine_poll(vb_engine* engine, int capacity, int wait, int64_t* tags, double* energies,
                         double* gradient_inf, int32_t* iterations, int32_t* converged, int32_t* status,
                         double* wait_s, double* latency_s, int* n_out);
vb_status vb_engine_pending(vb_engine* engine, int* queued, int* running, size_t* bytes_in_use);

/* ---- RI AO -> active-space transform ----------------------------------------------------------- */

/* transform_ri_active_integrals (src/integrals/active/ri.cpp:33-96) in FP64.  B_packed:
 * metric-whitened AO-pair factors [n_aux x n_bf(n_bf+1)/2], column-major (row = auxiliary
 * function, column = AO pair hi(hi+1)/2+lo; RiAoFactorization::metric_whitened_ao_pair_factors);
 * C: active coefficients [n_bf x n_act], column-major, n_act <= 16.  Outputs:
 *   one_index [(n_act n_aux) x n_bf], row a*n_aux + P (ri_one_index_factors; may be NULL),
 *   L [n_aux x n_act(n_act+1)/2] (ri_active_pair_factors),
 *   K_packed [P(P+1)/2] (pack_ri_active_integrals, ri.cpp:13-31; may be NULL).
 * VB_MEM_HOST: synchronous.  VB_MEM_DEVICE: stream-ordered on the context stream. */
vb_status vb_active_transform_ri(vb_context* ctx, const double* B_packed, int n_aux, int n_bf, const double* C,
                                 int n_act, int mem_space, double* one_index, double* L, double* K_packed);

/* Precision of the one-index step (the flop-carrying GEMM) of the RI transform. */
enum { VB_PRECISION_FP64 = 0, VB_PRECISION_BF16X3 = 1 };

/* vb_active_transform_ri with a selectable precision for the one-index step (same arguments and
 * outputs).  VB_PRECISION_BF16X3: each FP64 operand is rounded to FP32 and split into three BF16
 * parts, the products of order <= 2 run on the tensor cores with FP32 accumulation and an FP64
 * recombination (relative error of order 1e-7 against FP64; n_bf <= 1536); the second index and
 * the packing stay FP64.  The reference computes this step in FP64 only
 * (transform_ri_one_index, src/integrals/ao/ri_transform.cpp:10-37). */
vb_status vb_active_transform_ri_precision(vb_context* ctx, const double* B_packed, int n_aux, int n_bf,
                                           const double* C, int n_act, int precision, int mem_space,
                                           double* one_index, double* L, double* K_packed);

/* Adjoint of the transform: given dE/dL [n_aux x n_act(n_act+1)/2] and the one-index factors
 * of the forward call, dE/dC [n_bf x n_act] (column-major), the orbital pull-back of RI pair
 * factors that the reference's gradients take from ri_one_index_factors
 * (src/integrals/response/ri.cpp:370). */
vb_status vb_active_transform_ri_adjoint(vb_context* ctx, const double* one_index, const double* dL, int n_aux,
                                         int n_bf, int n_act, int mem_space, double* dC);

/* RI pair factors in a new orbital frame, replacing transform_ri_pair_factors (mode 0),
 * transform_ri_pair_factor_direction (mode 1) and transform_ri_pair_factor_direction_from_orthogonal
 * (mode 2) of src/integrals/active/ri_transform.cpp:178-211 (declared in ri_transform.hpp:24-60).
 * factors / factor_direction: [n_aux x n(n+1)/2] column-major, row P packing the symmetric n x n
 * factor B_P at (i, j), i >= j, i (i+1)/2 + j; frame Q and frame_direction: n x n column-major.
 *   mode 0: out = Q^T B Q                                  (factor_direction, frame_direction unused)
 *   mode 1: out = Q^T dB Q + dQ^T B Q + Q^T B dQ           (factors = B, factor_direction = dB,
 *                                                           frame_direction = dQ)
 *   mode 2: out = Q^T dB Q - K^T Bbar - Bbar K             (factors = Bbar = Q^T B Q,
 *                                                           factor_direction = dB, frame_direction = K)
 * Same packed layout out.  n <= 64. */
vb_status vb_ri_pair_factors_frame(vb_context* ctx, int mode, const double* factors, const double* factor_direction,
                                   int n_aux, int n, const double* frame, const double* frame_direction,
                                   int mem_space, double* out);

/* ---- launch-schedule autotuner ---------------------------------------------------------------- */

/* No counterpart in the reference.  The first evaluation of a shape (electrons per string, active
 * orbitals, factor rank) on a device times the launch variants of the spin-pair kernel (warps per
 * CTA x CTAs per SM) and of the determinant-pair kernel (block size x blocks per SM) with CUDA
 * events and keeps the fastest for the process; the environment variable VBCORE_AUTOTUNE=0 keeps
 * the default schedules.  The report lists one line per tuned key ("key -> variant (ms: ...)");
 * `needed` receives its length + 1. */
vb_status vb_autotune_report(char* buffer, size_t capacity, size_t* needed);
vb_status vb_autotune_clear(void);

/* ---- allocation-free spin-pair evaluation ------------------------------------------------- */

/* No counterpart in the reference.  For callers that cannot allocate device memory where
 * they need the numbers (a serving loop that reserves all HBM up front and forbids allocation
 * on the request path, or an application whose own allocator owns the device budget): every
 * unordered pair (u <= v) of one spin-string table is evaluated with the structure plan's
 * kernels, but all scratch comes from a file-scope 32 MiB device array instead of cudaMalloc
 * (each GPU that loads the library holds that array until exit).  Tables needing more scratch
 * than that are rejected with VB_ERR_BUDGET (about 250 strings of 5 electrons in 10 orbitals
 * fit; use the plan API above for larger ones).
 *
 * At most 8 electrons per string (k > 8 returns VB_ERR_UNSUPPORTED: the stack reserved by the
 * set-up call covers the exact-path kernels for k <= 8 only).
 *
 * All pointers are device pointers: strings = n_strings occupation masks (k bits set, orbitals
 * < n_orbitals), S_act and h (n x n), packed (ij|kl); out_scalars receives, for pair index
 * t = u N - u (u - 1) / 2 + (v - u), {det, one-electron H, total same-spin H, nullity} at
 * out_scalars[4 t .. 4 t + 3].  The work is enqueued on `cuda_stream` (the output is complete
 * when the stream reaches it); every call synchronizes the stream once, midway, to read back
 * the pair-kernel rank.  The first call made with a device current is that device's set-up
 * call: it raises the device's stack limit to what the exact-path kernels need (later calls
 * then never make the runtime grow the local-memory reservation), loads every kernel a call may
 * launch (lazy module loading then places no code in device memory during a later call) and
 * looks up the scratch array's address (cudaGetSymbolAddress).  No call can be recorded into
 * a CUDA graph: each one synchronizes its stream.  Calls share the array and keep its last
 * contents; calls that overlap on the GPU race on it. */
vb_status vb_spin_pairs_noalloc(void* cuda_stream, int n_orbitals, int k, int n_strings, const uint64_t* strings,
                                const double* ovlp_act, const double* h1e_act, const double* eri_packed,
                                double* out_scalars);

#ifdef __cplusplus
}
#endif

#endif /* VBCORE_H */
