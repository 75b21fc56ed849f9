// The structure H/S plan object shared by the plan, gradient and solver translation units.
#pragma once

#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "internal.h"
#include "kernels.h"

using namespace vbcore;

// Term segments of the band reduction per (structure group, row tile) (see BandReduceArgs).
struct BandSegments {
    int n_groups = 0, n_tiles = 0, seg_max = 0;
    DeviceBuffer off, meta, coef, row;
    // row tiles with terms, per group ascending (CSR: tile_off[g] .. tile_off[g + 1] index tiles)
    DeviceBuffer tiles, tile_off;
};

struct vb_hs_plan {
    vb_context* ctx = nullptr;
    int n = 0, ka = 0, kb = 0, np = 0, gd = 0;
    int n_str = 0;
    long long n_det = 0;
    int Na = 0, Nb = 0;
    bool shared_tables = false;
    DeviceBuffer occ_a, occ_b, det_alpha, det_beta;
    DeviceBuffer rec_a, rec_b, tables_a, tables_b;
    int stride_a = 0, stride_b = 0;
    long long npairs_a = 0, npairs_b = 0;
    // counters: [0, 1] listed (exact-path) spin pairs alpha/beta, [2, 3] the gradient's listed
    // pairs, [4, 5] the frame kernel's task counters alpha/beta, [7] the band reduction's
    // timeout flag
    DeviceBuffer counters, list_a, list_b;
    // right strings of each left string bucketed by hole set (see SpinTableArgs::rlist)
    DeviceBuffer rlist_a, rlist_b, rdesc_a, rdesc_b, ebound_a, ebound_b;
    int rec_stride_alloc = 0;  // record stride the spin-pair records are allocated for
    DeviceBuffer S_in, h_in, eri_in, gamma, kfull;
    // pair-kernel factorization: lf[q * np + m], scratch, signs, meta = {r_pos, r_neg} (+ host copy)
    DeviceBuffer lf, fwork, fcols, fsigns, fmeta;
    int* meta_host = nullptr;
    int R = 0, r_pos = 0;
    long long band_width = 0;  // determinant columns per band (bands live in the context scratch)
    long long band_ld = 0;     // band row stride (band_width rounded up to 32 elements)
    DeviceBuffer Hout, Sout;
    DeviceBuffer str_off, str_det, str_coef;
    // structure incidence by determinant (CSR) and the gradient's adjoint scratch
    DeviceBuffer det_off, det_str, det_coef;
    DeviceBuffer adj_a, adj_b, grad_acc;
    // host inputs of the last host-pointer evaluation whose records are still resident
    std::vector<double> last_inputs;
    bool records_current = false;
    BandSegments segments;
    // spin-flip map of the determinant list (folds the determinant-pair work in half)
    DeviceBuffer flip;
    // determinants by alpha string (CSR: alpha_off[i] .. alpha_off[i + 1] index alpha_dets)
    DeviceBuffer alpha_off, alpha_dets;
    bool has_flip = false;
    // internal position of each determinant of the caller's list when the plan reorders them
    // (empty: the caller's order), host copy and device copy
    std::vector<long long> det_position;
    DeviceBuffer det_position_dev;
    long long det_pair_evaluations = 0;  // unordered determinant pairs evaluated (orbit representatives)
    vb_hs_stats stats{};
    bool evaluated = false;
    // phase timing: per phase a pool of (start, stop) event pairs, `used` pairs this execute
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events[VB_PHASE_COUNT];
    int used[VB_PHASE_COUNT] = {};
    ~vb_hs_plan() {
        if (meta_host) cudaFreeHost(meta_host);
        for (auto& v : events)
            for (auto& e : v) {
                cudaEventDestroy(e.first);
                cudaEventDestroy(e.second);
            }
    }
};


namespace vbcore {

vb_status upload(vb_context* ctx, DeviceBuffer& buf, const void* src, size_t bytes);
int record_stride(int R);
SpinTableArgs table_args(vb_hs_plan* p, bool beta, const double* S, const double* h, const double* eri);
FullPairArgs full_args(vb_hs_plan* p);
// Uploads host inputs (mem == VB_MEM_HOST), builds the integral tables and the pair-kernel
// factorization, and evaluates every spin-pair record; *dS, *dh, *deri receive the device
// copies of the inputs.
// True when the resident spin-pair records were evaluated from exactly these host inputs.
bool records_match(const vb_hs_plan* p, const double* S, const double* h, const double* eri, int mem);
vb_status prepare_spin_records(vb_hs_plan* p, const double* S, const double* h, const double* eri, int mem,
                               const double** dS, const double** dh, const double** deri, int* launches);

}  // namespace vbcore
