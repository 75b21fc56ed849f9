// Structure H/S plans and the determinant-pair level entry points of the C ABI.
//
// A plan uploads the orbital-independent topology once (string tables, determinant list,
// structure incidence) and owns the spin-pair record scratch; execute() then runs, all
// stream-ordered on the context's stream:
//   prepare_tables -> spin_pairs (fast + exact, per distinct spin table)
//   -> per band of determinant columns: full_pairs -> band_reduce (per structure chunk)
//   -> structure_reduce + symmetrize.
// This is the B200 counterpart of FullDeterminantStructureHamiltonianOverlapBuilder::build
// (src/vbscf/structures/assembly/hamiltonian_overlap.hpp:70-107 in the reference).
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "device_algebra.cuh"
#include "internal.h"
#include "kernels.h"
#include "plan.h"

using namespace vbcore;

namespace vbcore {

vb_status upload(vb_context* ctx, DeviceBuffer& buf, const void* src, size_t bytes) {
    vb_status st = buf.allocate(ctx, bytes);
    if (st != VB_OK) return st;
    if (bytes == 0) return VB_OK;
    cudaError_t err = cudaMemcpyAsync(buf.ptr, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (err != cudaSuccess) return cuda_error(ctx, err, "cudaMemcpyAsync (plan upload)");
    return VB_OK;
}

}  // namespace vbcore

namespace {

// Determinant indices of the caller's list -> the plan's order (indices outside the list pass
// through unchanged, as they would without a reorder).
__global__ void translate_pairs_kernel(long long count, const long long* __restrict__ in,
                                       const long long* __restrict__ position, long long n_det,
                                       long long* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const long long d = in[i];
        out[i] = (d >= 0 && d < n_det) ? position[d] : d;
    }
}

std::vector<uint64_t> occupation_rows(const uint64_t* masks, int count, int k, int n, std::string* error) {
    std::vector<uint64_t> rows(2 * (size_t)count, ~uint64_t{0});
    for (int s = 0; s < count; ++s) {
        uint8_t bytes[16];
        std::memset(bytes, 0xFF, sizeof(bytes));
        int m = 0;
        for (int o = 0; o < 64; ++o)
            if ((masks[s] >> o) & 1) {
                if (m >= 16 || o >= n) {
                    *error = "string occupation outside the active space or above 16 electrons";
                    return {};
                }
                bytes[m++] = (uint8_t)o;
            }
        if (m != k) {
            *error = "string electron count does not match the spin's electron count";
            return {};
        }
        std::memcpy(&rows[2 * (size_t)s], bytes, 16);
    }
    return rows;
}

// Phase bracket: records a start event on construction and a stop event on close().
struct PhaseMark {
    vb_hs_plan* p;
    int phase;
    cudaEvent_t stop = nullptr;
    PhaseMark(vb_hs_plan* plan, int ph) : p(plan), phase(ph) {
        if (!p->timing) return;
        auto& pool = p->events[phase];
        if (p->used[phase] == (int)pool.size()) {
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            pool.push_back({a, b});
        }
        auto& pr = pool[p->used[phase]++];
        cudaEventRecord(pr.first, p->ctx->stream);
        stop = pr.second;
    }
    void close() {
        if (stop) cudaEventRecord(stop, p->ctx->stream);
        stop = nullptr;
    }
    ~PhaseMark() { close(); }
};

}  // namespace

namespace vbcore {

int record_stride(int R) {
    const int s = R + 4;
    return (s + 1) / 2 * 2;
}

}  // namespace vbcore

extern "C" {

vb_status vb_hs_plan_create(vb_context* ctx, const vb_expansion* ex, vb_hs_plan** out) {
    if (!ctx || !ex || !out) return set_error(ctx, VB_ERR_INVALID, "vb_hs_plan_create: null argument");
    *out = nullptr;
    const int n = ex->n_orbitals;
    if (n <= 0 || n > kMaxOrbitals) return set_error(ctx, VB_ERR_UNSUPPORTED, "n_orbitals must be in 1..64");
    if (ex->n_alpha_electrons < 0 || ex->n_alpha_electrons > kMaxElectrons || ex->n_beta_electrons < 0 ||
        ex->n_beta_electrons > kMaxElectrons)
        return set_error(ctx, VB_ERR_UNSUPPORTED, "electrons per spin must be in 0..16");
    if (ex->n_determinants <= 0 || ex->n_structures <= 0)
        return set_error(ctx, VB_ERR_INVALID, "at least one determinant and one structure are required");
    if (ex->n_alpha_electrons > 0 && (ex->n_alpha_strings <= 0 || !ex->alpha_strings))
        return set_error(ctx, VB_ERR_INVALID, "alpha string table missing");
    if (ex->n_beta_electrons > 0 && (ex->n_beta_strings <= 0 || !ex->beta_strings))
        return set_error(ctx, VB_ERR_INVALID, "beta string table missing");
    if (!ex->det_alpha || !ex->det_beta || !ex->term_offsets || !ex->term_structure || !ex->term_coefficient)
        return set_error(ctx, VB_ERR_INVALID, "expansion arrays missing");
    cudaSetDevice(ctx->device);
    vb_hs_plan* p = new (std::nothrow) vb_hs_plan();
    if (!p) return set_error(ctx, VB_ERR_INVALID, "out of host memory");
    p->ctx = ctx;
    p->n = n;
    p->ka = ex->n_alpha_electrons;
    p->kb = ex->n_beta_electrons;
    p->np = n * (n + 1) / 2;
    p->gd = n * (n - 1) / 2;
    p->n_str = ex->n_structures;
    p->n_det = ex->n_determinants;
    p->Na = p->ka > 0 ? ex->n_alpha_strings : 0;
    p->Nb = p->kb > 0 ? ex->n_beta_strings : 0;
    auto fail = [&](vb_status st) {
        delete p;
        return st;
    };
    // validate the determinant list and incidence
    for (long long d = 0; d < p->n_det; ++d) {
        if ((p->ka > 0 && (ex->det_alpha[d] < 0 || ex->det_alpha[d] >= p->Na)) ||
            (p->kb > 0 && (ex->det_beta[d] < 0 || ex->det_beta[d] >= p->Nb)))
            return fail(set_error(ctx, VB_ERR_INVALID, "determinant string index out of range"));
    }
    if (ex->term_offsets[0] != 0) return fail(set_error(ctx, VB_ERR_INVALID, "term offsets must start at 0"));
    for (long long d = 0; d < p->n_det; ++d)
        if (ex->term_offsets[d + 1] < ex->term_offsets[d])
            return fail(set_error(ctx, VB_ERR_INVALID, "term offsets must be non-decreasing"));
    const long long n_terms = ex->term_offsets[p->n_det];
    for (long long t = 0; t < n_terms; ++t)
        if (ex->term_structure[t] < 0 || ex->term_structure[t] >= p->n_str)
            return fail(set_error(ctx, VB_ERR_INVALID, "term structure index out of range"));

    // Determinant order.  Structures that share few determinants (ionic structures: determinants
    // cluster by occupation pattern) leave each band-reduction structure group reading a row tile
    // for a handful of its rows.  Placing every determinant at the first structure that uses it
    // makes the determinants of consecutive structures contiguous; the reorder is taken when it at
    // least halves the (structure group, row tile) segments.  Everything the plan computes is per
    // structure or per spin string, so only vb_hs_plan_determinant_pairs translates indices.
    std::vector<int32_t> r_alpha, r_beta, r_str;
    std::vector<int64_t> r_off;
    std::vector<double> r_coef;
    vb_expansion reordered;
    {
        const long long nd = p->n_det;
        std::vector<long long> first(nd, (long long)p->n_str);
        for (long long d = 0; d < nd; ++d)
            for (long long t = ex->term_offsets[d]; t < ex->term_offsets[d + 1]; ++t)
                first[d] = std::min<long long>(first[d], ex->term_structure[t]);
        std::vector<long long> order(nd);
        for (long long d = 0; d < nd; ++d) order[d] = d;
        // within a structure group's range, determinants stay in alpha-major order (the spin-pair
        // records of neighbouring determinant pairs stay neighbours)
        std::stable_sort(order.begin(), order.end(), [&](long long x, long long y) {
            const long long gx = first[x] / kBandGroup, gy = first[y] / kBandGroup;
            if (gx != gy) return gx < gy;
            if (ex->det_alpha[x] != ex->det_alpha[y]) return ex->det_alpha[x] < ex->det_alpha[y];
            return ex->det_beta[x] < ex->det_beta[y];
        });
        std::vector<long long> pos(nd);
        for (long long i = 0; i < nd; ++i) pos[order[i]] = i;
        const long long tiles = (nd + kBandTileRows - 1) / kBandTileRows;
        auto segments = [&](bool moved) {
            std::vector<long long> keys;
            keys.reserve((size_t)n_terms);
            for (long long d = 0; d < nd; ++d)
                for (long long t = ex->term_offsets[d]; t < ex->term_offsets[d + 1]; ++t)
                    keys.push_back((long long)(ex->term_structure[t] / kBandGroup) * tiles +
                                   (moved ? pos[d] : d) / kBandTileRows);
            std::sort(keys.begin(), keys.end());
            return (long long)(std::unique(keys.begin(), keys.end()) - keys.begin());
        };
        if (2 * segments(true) <= segments(false)) {
            r_alpha.resize(nd);
            r_beta.resize(nd);
            r_off.assign(nd + 1, 0);
            r_str.resize(n_terms);
            r_coef.resize(n_terms);
            for (long long i = 0; i < nd; ++i) {
                const long long d = order[i];
                r_alpha[i] = ex->det_alpha[d];
                r_beta[i] = ex->det_beta[d];
                const long long t0 = ex->term_offsets[d], cnt = ex->term_offsets[d + 1] - t0;
                std::copy(ex->term_structure + t0, ex->term_structure + t0 + cnt, r_str.begin() + r_off[i]);
                std::copy(ex->term_coefficient + t0, ex->term_coefficient + t0 + cnt, r_coef.begin() + r_off[i]);
                r_off[i + 1] = r_off[i] + cnt;
            }
            reordered = *ex;
            reordered.det_alpha = r_alpha.data();
            reordered.det_beta = r_beta.data();
            reordered.term_offsets = r_off.data();
            reordered.term_structure = r_str.data();
            reordered.term_coefficient = r_coef.data();
            ex = &reordered;
            p->det_position = std::move(pos);
        }
    }

    std::string err;
    std::vector<uint64_t> occa, occb;
    if (p->ka > 0) {
        occa = occupation_rows(ex->alpha_strings, p->Na, p->ka, n, &err);
        if (occa.empty()) return fail(set_error(ctx, VB_ERR_INVALID, err));
    }
    if (p->kb > 0) {
        occb = occupation_rows(ex->beta_strings, p->Nb, p->kb, n, &err);
        if (occb.empty()) return fail(set_error(ctx, VB_ERR_INVALID, err));
    }
    p->shared_tables = p->ka > 0 && p->ka == p->kb && p->Na == p->Nb &&
                       std::equal(ex->alpha_strings, ex->alpha_strings + p->Na, ex->beta_strings);
    vb_status st;
    if ((st = upload(ctx, p->occ_a, occa.data(), occa.size() * 8)) != VB_OK) return fail(st);
    if ((st = upload(ctx, p->occ_b, occb.data(), occb.size() * 8)) != VB_OK) return fail(st);
    if ((st = upload(ctx, p->det_alpha, ex->det_alpha, sizeof(int32_t) * p->n_det)) != VB_OK) return fail(st);
    {
        const long long n_terms = ex->term_offsets[p->n_det];
        if ((st = upload(ctx, p->det_off, ex->term_offsets, sizeof(int64_t) * (p->n_det + 1))) != VB_OK) return fail(st);
        if ((st = upload(ctx, p->det_str, ex->term_structure, sizeof(int32_t) * n_terms)) != VB_OK) return fail(st);
        if ((st = upload(ctx, p->det_coef, ex->term_coefficient, sizeof(double) * n_terms)) != VB_OK) return fail(st);
    }
    if ((st = upload(ctx, p->det_beta, ex->det_beta, sizeof(int32_t) * p->n_det)) != VB_OK) return fail(st);

    // spin-pair records are allocated by the first execute, once the factor rank is known
    p->npairs_a = (long long)p->Na * (p->Na + 1) / 2;
    p->npairs_b = p->shared_tables ? 0 : (long long)p->Nb * (p->Nb + 1) / 2;
    if ((st = p->list_a.allocate(ctx, sizeof(unsigned long long) * std::max(1LL, p->npairs_a))) != VB_OK) return fail(st);
    if (!p->shared_tables &&
        (st = p->list_b.allocate(ctx, sizeof(unsigned long long) * std::max(1LL, p->npairs_b))) != VB_OK)
        return fail(st);
    if ((st = p->counters.allocate(ctx, 8 * sizeof(unsigned long long))) != VB_OK) return fail(st);
    // right strings of every left string bucketed by hole set (depends on the strings only), and
    // the per-left-string frame tables, sized for the largest factor rank
    for (int beta = 0; beta < 2; ++beta) {
        const int k = beta ? p->kb : p->ka;
        if (k <= 0 || (beta && p->shared_tables) || !frame_spin_supported(n, k, 0)) continue;
        const long long N = beta ? p->Nb : p->Na;
        DeviceBuffer& rl = beta ? p->rlist_b : p->rlist_a;
        DeviceBuffer& rd = beta ? p->rdesc_b : p->rdesc_a;
        DeviceBuffer& eb = beta ? p->ebound_b : p->ebound_a;
        DeviceBuffer& tb = beta ? p->tables_b : p->tables_a;
        if ((st = rl.allocate(ctx, sizeof(int) * (size_t)std::max(1LL, N * (N + 1) / 2))) != VB_OK) return fail(st);
        if ((st = rd.allocate(ctx, sizeof(unsigned) * (size_t)std::max(1LL, N * (N + 1) / 2))) != VB_OK) return fail(st);
        if ((st = eb.allocate(ctx, sizeof(int) * (size_t)N * (k + 2))) != VB_OK) return fail(st);
        if ((st = tb.allocate(ctx, sizeof(double) * frame_table_doubles(n, k, p->np) * N)) != VB_OK) return fail(st);
        const cudaError_t err = launch_sort_right_strings(k, (int)N, (beta ? p->occ_b : p->occ_a).as<uint64_t>(),
                                                         rl.as<int>(), rd.as<unsigned>(), eb.as<int>(), ctx->stream);
        if (err != cudaSuccess) return fail(cuda_error(ctx, err, "sort_right_strings"));
    }

    // inputs and derived integral tables
    if ((st = p->S_in.allocate(ctx, sizeof(double) * n * n)) != VB_OK) return fail(st);
    if ((st = p->h_in.allocate(ctx, sizeof(double) * n * n)) != VB_OK) return fail(st);
    if ((st = p->eri_in.allocate(ctx, sizeof(double) * (size_t)p->np * (p->np + 1) / 2)) != VB_OK) return fail(st);
    if ((st = p->gamma.allocate(ctx, sizeof(double) * std::max(1, p->gd * p->gd))) != VB_OK) return fail(st);
    if ((st = p->kfull.allocate(ctx, sizeof(double) * p->np * p->np)) != VB_OK) return fail(st);
    for (DeviceBuffer* b : {&p->lf, &p->fwork, &p->fcols})
        if ((st = b->allocate(ctx, sizeof(double) * p->np * p->np)) != VB_OK) return fail(st);
    if ((st = p->fsigns.allocate(ctx, sizeof(int) * p->np)) != VB_OK) return fail(st);
    if ((st = p->fmeta.allocate(ctx, sizeof(int) * 2)) != VB_OK) return fail(st);
    if (cudaMallocHost(&p->meta_host, sizeof(int) * 4) != cudaSuccess) return fail(set_error(ctx, VB_ERR_CUDA, "cudaMallocHost"));

    // spin-flip map: determinant with the alpha and beta strings exchanged; usable when every
    // determinant's image exists and carries the same structure coefficients
    std::vector<int> flipmap;
    if (p->shared_tables) {
        std::vector<long long> key(p->n_det);
        for (long long d = 0; d < p->n_det; ++d) key[d] = (long long)ex->det_alpha[d] * p->Na + ex->det_beta[d];
        std::vector<long long> order(p->n_det);
        for (long long d = 0; d < p->n_det; ++d) order[d] = d;
        std::sort(order.begin(), order.end(), [&](long long x, long long y) { return key[x] < key[y]; });
        flipmap.assign(p->n_det, -1);
        bool ok = true;
        for (long long d = 0; d < p->n_det && ok; ++d) {
            const long long want = (long long)ex->det_beta[d] * p->Na + ex->det_alpha[d];
            auto it = std::lower_bound(order.begin(), order.end(), want,
                                       [&](long long idx, long long v) { return key[idx] < v; });
            if (it == order.end() || key[*it] != want) {
                ok = false;
                break;
            }
            const long long f = *it;
            flipmap[d] = (int)f;
            const long long n1 = ex->term_offsets[d + 1] - ex->term_offsets[d];
            const long long n2 = ex->term_offsets[f + 1] - ex->term_offsets[f];
            if (n1 != n2) {
                ok = false;
                break;
            }
            for (long long q = 0; q < n1; ++q)
                if (ex->term_structure[ex->term_offsets[d] + q] != ex->term_structure[ex->term_offsets[f] + q] ||
                    ex->term_coefficient[ex->term_offsets[d] + q] != ex->term_coefficient[ex->term_offsets[f] + q]) {
                    ok = false;
                    break;
                }
        }
        if (ok) {
            p->has_flip = true;
            // determinants grouped by alpha string, for the gradient's per-record adjoint sums
            std::vector<int> aoff(p->Na + 1, 0), adets(p->n_det);
            for (long long d = 0; d < p->n_det; ++d) ++aoff[ex->det_alpha[d] + 1];
            for (int i = 0; i < p->Na; ++i) aoff[i + 1] += aoff[i];
            std::vector<int> next(aoff.begin(), aoff.end() - 1);
            for (long long d = 0; d < p->n_det; ++d) adets[next[ex->det_alpha[d]]++] = (int)d;
            if ((st = upload(ctx, p->alpha_off, aoff.data(), sizeof(int) * aoff.size())) != VB_OK) return fail(st);
            if ((st = upload(ctx, p->alpha_dets, adets.data(), sizeof(int) * std::max<size_t>(1, adets.size()))) != VB_OK)
                return fail(st);
            // orbits of unordered pairs {d, e} under the flip (Burnside): (P + fixed pairs) / 2
            long long fixed_dets = 0;
            for (long long d = 0; d < p->n_det; ++d) fixed_dets += flipmap[d] == d;
            const long long P = p->n_det * (p->n_det + 1) / 2;
            p->det_pair_evaluations = (P + fixed_dets * (fixed_dets + 1) / 2 + (p->n_det - fixed_dets) / 2) / 2;
            if ((st = upload(ctx, p->flip, flipmap.data(), sizeof(int) * p->n_det)) != VB_OK) return fail(st);
        }
    }

    if (!p->has_flip) p->det_pair_evaluations = p->n_det * (p->n_det + 1) / 2;

    // band of determinant columns: keep the two band buffers within ~1 GB and 1/8 of the budget
    const size_t band_cap = std::min<size_t>((size_t)1 << 30, ctx->budget / 8);
    long long width = (long long)(band_cap / (16 * (size_t)p->n_det));
    width = std::max(32LL, std::min(width, p->n_det));
    p->band_width = width;
    p->band_ld = (width + 31) / 32 * 32;
    // the bands and the structure-reduce buffers (Z, W) are the context's execute scratch
    const size_t wbytes = sizeof(double) * (size_t)p->n_str * p->n_str;
    for (DeviceBuffer* b : {&p->Hout, &p->Sout})
        if ((st = b->allocate(ctx, wbytes)) != VB_OK) return fail(st);

    // structure-major incidence (CSC of T)
    std::vector<long long> soff(p->n_str + 1, 0);
    for (long long t = 0; t < n_terms; ++t) ++soff[ex->term_structure[t] + 1];
    for (int I = 0; I < p->n_str; ++I) soff[I + 1] += soff[I];
    std::vector<long long> sdet(n_terms), next(soff.begin(), soff.end() - 1);
    std::vector<double> scoef(n_terms);
    for (long long d = 0; d < p->n_det; ++d)
        for (long long t = ex->term_offsets[d]; t < ex->term_offsets[d + 1]; ++t) {
            const long long pos = next[ex->term_structure[t]]++;
            sdet[pos] = d;
            scoef[pos] = ex->term_coefficient[t];
        }
    if ((st = upload(ctx, p->str_off, soff.data(), sizeof(long long) * soff.size())) != VB_OK) return fail(st);
    if ((st = upload(ctx, p->str_det, sdet.data(), sizeof(long long) * std::max<size_t>(1, sdet.size()))) != VB_OK)
        return fail(st);
    if ((st = upload(ctx, p->str_coef, scoef.data(), sizeof(double) * std::max<size_t>(1, scoef.size()))) != VB_OK)
        return fail(st);

    // band-reduction term segments: for every (structure group, row tile) the terms (row in the
    // tile, coefficient) of the group's structures ordered by (warp, slot, determinant)
    {
        BandSegments& b = p->segments;
        b.n_groups = (p->n_str + kBandGroup - 1) / kBandGroup;
        b.n_tiles = (int)((p->n_det + kBandTileRows - 1) / kBandTileRows);
        const size_t nseg = (size_t)b.n_groups * b.n_tiles;
        std::vector<long long> off(nseg + 1, 0);
        std::vector<unsigned char> meta(nseg * kBandMetaBytes, 0);
        std::vector<double> coef;
        std::vector<unsigned char> row;
        std::vector<long long> cur(soff.begin(), soff.end() - 1);  // next term of each structure
        std::vector<int> tiles, tile_off(b.n_groups + 1, 0);
        for (int g = 0; g < b.n_groups; ++g)
            for (int t = 0; t < b.n_tiles; ++t) {
                const size_t seg = (size_t)g * b.n_tiles + t;
                off[seg] = (long long)coef.size();
                unsigned char* m = meta.data() + seg * kBandMetaBytes;
                const long long r0 = (long long)t * kBandTileRows, r1 = r0 + kBandTileRows;
                int within = 0;
                for (int w = 0; w < kBandWarps; ++w) {
                    const unsigned short start = (unsigned short)within;
                    std::memcpy(m + kBandWarps * kBandSlots + 2 * w, &start, 2);
                    for (int sl = 0; sl < kBandSlots; ++sl) {
                        const int I = g * kBandGroup + sl * kBandWarps + w;
                        int cnt = 0;
                        if (I < p->n_str)
                            for (; cur[I] < soff[I + 1] && sdet[cur[I]] < r1; ++cur[I], ++cnt) {
                                row.push_back((unsigned char)(sdet[cur[I]] - r0));
                                coef.push_back(scoef[cur[I]]);
                            }
                        m[w * kBandSlots + sl] = (unsigned char)cnt;
                        within += cnt;
                    }
                }
                if (within > 0) tiles.push_back(t);
                tile_off[g + 1] = (int)tiles.size();
                while (coef.size() % 16) {
                    coef.push_back(0.0);
                    row.push_back(0);
                }
                b.seg_max = std::max(b.seg_max, (int)((long long)coef.size() - off[seg]));
            }
        off[nseg] = (long long)coef.size();
        if ((st = upload(ctx, b.tiles, tiles.data(), sizeof(int) * std::max<size_t>(1, tiles.size()))) != VB_OK)
            return fail(st);
        if ((st = upload(ctx, b.tile_off, tile_off.data(), sizeof(int) * tile_off.size())) != VB_OK) return fail(st);
        if ((st = upload(ctx, b.off, off.data(), sizeof(long long) * off.size())) != VB_OK) return fail(st);
        if ((st = upload(ctx, b.meta, meta.data(), std::max<size_t>(16, meta.size()))) != VB_OK) return fail(st);
        if ((st = upload(ctx, b.coef, coef.data(), sizeof(double) * std::max<size_t>(1, coef.size()))) != VB_OK)
            return fail(st);
        if ((st = upload(ctx, b.row, row.data(), std::max<size_t>(16, row.size()))) != VB_OK) return fail(st);
    }
    cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    if (e2 != cudaSuccess) return fail(cuda_error(ctx, e2, "plan upload"));
    *out = p;
    return VB_OK;
}

vb_status vb_hs_plan_destroy(vb_hs_plan* plan) {
    if (!plan) return VB_OK;
    cudaStreamSynchronize(plan->ctx->stream);
    delete plan;
    return VB_OK;
}

}  // extern "C"

namespace vbcore {

SpinTableArgs table_args(vb_hs_plan* p, bool beta, const double* S, const double* h, const double* eri) {
    SpinTableArgs a{};
    a.n = p->n;
    a.k = beta ? p->kb : p->ka;
    a.n_strings = beta ? p->Nb : p->Na;
    a.occ = beta ? p->occ_b.as<uint64_t>() : p->occ_a.as<uint64_t>();
    a.n_pairs = beta ? p->npairs_b : p->npairs_a;
    a.S = S;
    a.h = h;
    a.gamma = p->gamma.as<double>();
    a.eri = eri;
    a.gamma_dim = p->gd;
    a.lf = p->lf.as<double>();
    a.ld = p->np;
    a.R = p->R;
    a.records = beta ? p->rec_b.as<double>() : p->rec_a.as<double>();
    a.rec_stride = record_stride(p->R);
    a.careful_count = p->counters.as<unsigned long long>() + (beta ? 1 : 0);
    a.careful_list = beta ? p->list_b.as<unsigned long long>() : p->list_a.as<unsigned long long>();
    a.items = nullptr;
    a.n_items = 0;
    a.all_careful = 0;
    a.r_pos = p->r_pos;
    a.rlist = beta ? p->rlist_b.as<int>() : p->rlist_a.as<int>();
    a.rdesc = beta ? p->rdesc_b.as<unsigned>() : p->rdesc_a.as<unsigned>();
    a.ebound = beta ? p->ebound_b.as<int>() : p->ebound_a.as<int>();
    a.task_counter = p->counters.as<unsigned long long>() + 4 + (beta ? 1 : 0);
    return a;
}

FullPairArgs full_args(vb_hs_plan* p) {
    FullPairArgs a{};
    a.ka = p->ka;
    a.kb = p->kb;
    a.n_det = p->n_det;
    a.det_alpha = p->det_alpha.as<int>();
    a.det_beta = p->det_beta.as<int>();
    a.Na = p->Na;
    a.Nb = p->shared_tables ? p->Na : p->Nb;
    a.rec_a = p->rec_a.as<double>();
    a.rec_b = p->shared_tables ? p->rec_a.as<double>() : p->rec_b.as<double>();
    a.stride_a = record_stride(p->R);
    a.stride_b = record_stride(p->R);
    a.R = p->R;
    a.r_pos = p->r_pos;
    return a;
}

// Stage inputs and evaluate the spin-pair records of every distinct table.
bool records_match(const vb_hs_plan* p, const double* S, const double* h, const double* eri, int mem) {
    if (mem != VB_MEM_HOST || !p->records_current) return false;
    const size_t n2 = (size_t)p->n * p->n, ne = (size_t)p->np * (p->np + 1) / 2;
    if (p->last_inputs.size() != 2 * n2 + ne) return false;
    return std::memcmp(p->last_inputs.data(), S, sizeof(double) * n2) == 0 &&
           std::memcmp(p->last_inputs.data() + n2, h, sizeof(double) * n2) == 0 &&
           std::memcmp(p->last_inputs.data() + 2 * n2, eri, sizeof(double) * ne) == 0;
}

vb_status prepare_spin_records(vb_hs_plan* p, const double* S, const double* h, const double* eri, int mem,
                               const double** dS, const double** dh, const double** deri, int* launches) {
    vb_context* ctx = p->ctx;
    cudaStream_t s = ctx->stream;
    const size_t n2 = sizeof(double) * p->n * p->n;
    const size_t ne = sizeof(double) * (size_t)p->np * (p->np + 1) / 2;
    p->records_current = false;
    if (mem == VB_MEM_HOST) {
        const size_t a = (size_t)p->n * p->n, b = (size_t)p->np * (p->np + 1) / 2;
        p->last_inputs.resize(2 * a + b);
        std::memcpy(p->last_inputs.data(), S, n2);
        std::memcpy(p->last_inputs.data() + a, h, n2);
        std::memcpy(p->last_inputs.data() + 2 * a, eri, ne);
    }
    if (mem == VB_MEM_HOST) {
        cudaError_t err = cudaMemcpyAsync(p->S_in.ptr, S, n2, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(p->h_in.ptr, h, n2, cudaMemcpyHostToDevice, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(p->eri_in.ptr, eri, ne, cudaMemcpyHostToDevice, s);
        if (err != cudaSuccess) return cuda_error(ctx, err, "input upload");
        *dS = p->S_in.as<double>();
        *dh = p->h_in.as<double>();
        *deri = p->eri_in.as<double>();
    } else {
        *dS = S;
        *dh = h;
        *deri = eri;
    }
    for (int& u : p->used) u = 0;
    PhaseMark tables(p, VB_PHASE_TABLES);
    cudaError_t err = launch_prepare_tables(p->n, *deri, p->gamma.as<double>(), p->kfull.as<double>(), s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "prepare_tables");
    ++*launches;
    err = launch_factor_pair_kernel(p->np, p->kfull.as<double>(), p->fwork.as<double>(), p->fcols.as<double>(),
                                    p->fsigns.as<int>(), p->lf.as<double>(), p->np, p->fmeta.as<int>(), s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "factor_pair_kernel");
    ++*launches;
    // the factor rank sizes the spin-pair launch: one 8-byte read-back per evaluation
    err = cudaMemcpyAsync(p->meta_host, p->fmeta.ptr, sizeof(int) * 2, cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "factor rank read-back");
    p->r_pos = p->meta_host[0];
    p->R = p->meta_host[0] + p->meta_host[1];
    tables.close();
    if (record_stride(p->R) > p->rec_stride_alloc) {
        // (re)size the records for this rank; a later execute with a lower rank reuses them
        const int stride = record_stride(p->R);
        vb_status st = p->rec_a.allocate(ctx, sizeof(double) * stride * std::max(1LL, p->npairs_a));
        if (st == VB_OK && !p->shared_tables && p->kb > 0)
            st = p->rec_b.allocate(ctx, sizeof(double) * stride * std::max(1LL, p->npairs_b));
        if (st != VB_OK) {
            p->rec_a.release();
            p->rec_b.release();
            p->rec_stride_alloc = 0;
            return st;
        }
        p->rec_stride_alloc = stride;
    }
    {
        // per-left-string frame tables (they depend on S, h and the factor columns)
        PhaseMark frame(p, VB_PHASE_TABLES);
        if (p->ka > 0) {
            err = launch_spin_tables(table_args(p, false, *dS, *dh, *deri), p->tables_a.as<double>(), s, launches);
            if (err != cudaSuccess) return cuda_error(ctx, err, "frame tables (alpha)");
        }
        if (p->kb > 0 && !p->shared_tables) {
            err = launch_spin_tables(table_args(p, true, *dS, *dh, *deri), p->tables_b.as<double>(), s, launches);
            if (err != cudaSuccess) return cuda_error(ctx, err, "frame tables (beta)");
        }
    }
    PhaseMark spin(p, VB_PHASE_SPIN_PAIRS);
    err = cudaMemsetAsync(p->counters.ptr, 0, 8 * sizeof(unsigned long long), s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "cudaMemsetAsync");
    if (p->ka > 0) {
        err = launch_spin_pairs(table_args(p, false, *dS, *dh, *deri), p->tables_a.as<double>(), s, launches);
        if (err != cudaSuccess) return cuda_error(ctx, err, "spin_pairs (alpha)");
    }
    if (p->kb > 0 && !p->shared_tables) {
        err = launch_spin_pairs(table_args(p, true, *dS, *dh, *deri), p->tables_b.as<double>(), s, launches);
        if (err != cudaSuccess) return cuda_error(ctx, err, "spin_pairs (beta)");
    }
    spin.close();
    PhaseMark exact(p, VB_PHASE_EXACT_PAIRS);
    if (p->ka > 0) {
        err = launch_spin_pairs_exact(table_args(p, false, *dS, *dh, *deri), s, launches);
        if (err != cudaSuccess) return cuda_error(ctx, err, "spin_pairs exact (alpha)");
    }
    if (p->kb > 0 && !p->shared_tables) {
        err = launch_spin_pairs_exact(table_args(p, true, *dS, *dh, *deri), s, launches);
        if (err != cudaSuccess) return cuda_error(ctx, err, "spin_pairs exact (beta)");
    }
    p->records_current = mem == VB_MEM_HOST;
    return VB_OK;
}

}  // namespace vbcore

extern "C" {

namespace {

// Inputs in `mem`; outputs: H_out/S_out in `mem`, or (H_out == nullptr) left in the plan's
// device buffers Hout/Sout.
vb_status execute_impl(vb_hs_plan* p, const double* S, const double* h, const double* eri, int mem, double* H_out,
                       double* S_out) {
    vb_context* ctx = p->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int launches = 0;
    const double *dS, *dh, *deri;
    vb_status st = prepare_spin_records(p, S, h, eri, mem, &dS, &dh, &deri, &launches);
    if (st != VB_OK) return st;
    // execute scratch of the context: bands [n_det x width] and Z [n_det x n_str] (H, S), W [n_str^2] (H, S)
    double* scr[6];
    {
        const size_t band = sizeof(double) * (size_t)p->n_det * p->band_ld;
        const size_t zb = sizeof(double) * (size_t)p->n_str * p->n_det;
        const size_t wb = sizeof(double) * (size_t)p->n_str * p->n_str;
        const size_t sizes[6] = {band, band, zb, zb, wb, wb};
        for (int i = 0; i < 6; ++i) {
            scr[i] = static_cast<double*>(context_scratch(ctx, i, sizes[i], &st));
            if (!scr[i]) return st;
        }
    }
    FullPairArgs fa = full_args(p);
    fa.flip = p->has_flip ? p->flip.as<int>() : nullptr;
    for (long long e0 = 0; e0 < p->n_det; e0 += p->band_width) {
        const long long e1 = std::min(p->n_det, e0 + p->band_width);
        const long long B = e1 - e0;
        fa.e0 = e0;
        fa.e1 = e1;
        fa.n_items = e0 * B + B * (B + 1) / 2;
        fa.ldb = p->band_ld;
        fa.Hb = scr[0];
        fa.Sb = scr[1];
        PhaseMark pairs(p, VB_PHASE_DETERMINANT_PAIRS);
        cudaError_t err = launch_full_pairs(fa, s, &launches);
        if (err != cudaSuccess) return cuda_error(ctx, err, "full_pairs");
        pairs.close();
        PhaseMark reduce(p, VB_PHASE_BAND_REDUCE);
        {
            BandReduceArgs ba{};
            ba.n_det = p->n_det;
            ba.n_str = p->n_str;
            ba.e0 = e0;
            ba.width = B;
            ba.Hb = fa.Hb;
            ba.Sb = fa.Sb;
            ba.ldb = p->band_ld;
            ba.n_groups = p->segments.n_groups;
            ba.n_tiles = p->segments.n_tiles;
            ba.seg_max = p->segments.seg_max;
            ba.seg_off = p->segments.off.as<long long>();
            ba.seg_meta = p->segments.meta.as<unsigned char>();
            ba.term_c = p->segments.coef.as<double>();
            ba.term_d = p->segments.row.as<unsigned char>();
            ba.seg_tiles = p->segments.tiles.as<int>();
            ba.seg_tile_off = p->segments.tile_off.as<int>();
            ba.error = reinterpret_cast<int*>(p->counters.as<unsigned long long>() + 7);
            ba.spin_limit = ctx->barrier_spin_limit > 0 ? ctx->barrier_spin_limit : (1ll << 26);
            ba.Zh = scr[2];
            ba.Zs = scr[3];
            err = launch_band_reduce(ba, s, &launches);
            if (err != cudaSuccess) return cuda_error(ctx, err, "band_reduce");
        }
    }
    StructureReduceArgs ra{};
    ra.n_str = p->n_str;
    ra.n_det = p->n_det;
    ra.str_off = p->str_off.as<long long>();
    ra.str_det = p->str_det.as<long long>();
    ra.str_coef = p->str_coef.as<double>();
    ra.Zh = scr[2];
    ra.Zs = scr[3];
    ra.Wh = scr[4];
    ra.Ws = scr[5];
    const bool to_plan = H_out == nullptr;
    double* Hdst = (mem == VB_MEM_DEVICE && !to_plan) ? H_out : p->Hout.as<double>();
    double* Sdst = (mem == VB_MEM_DEVICE && !to_plan) ? S_out : p->Sout.as<double>();
    PhaseMark sreduce(p, VB_PHASE_STRUCTURE_REDUCE);
    cudaError_t err = launch_structure_reduce(ra, Hdst, Sdst, s, &launches);
    if (err != cudaSuccess) return cuda_error(ctx, err, "structure_reduce");
    sreduce.close();
    if (mem == VB_MEM_HOST && !to_plan) {
        const size_t wbytes = sizeof(double) * (size_t)p->n_str * p->n_str;
        err = cudaMemcpyAsync(H_out, Hdst, wbytes, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(S_out, Sdst, wbytes, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(p->meta_host + 2, p->counters.as<unsigned long long>() + 7, sizeof(int),
                                  cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) return cuda_error(ctx, err, "result download");
        if (p->meta_host[2]) return set_error(ctx, VB_ERR_TIMEOUT, "band_reduce: a tile wait timed out");
    }
    p->stats.spin_pairs = p->npairs_a + p->npairs_b;
    p->stats.determinant_pairs = p->det_pair_evaluations;
    p->stats.kernel_launches = launches;
    p->stats.factor_columns = p->R;
    p->evaluated = true;
    return VB_OK;
}

// Reads the band reduction's timeout flag of the last execute (synchronizes the stream).
vb_status band_status(vb_hs_plan* p) {
    cudaStream_t s = p->ctx->stream;
    cudaError_t err = cudaMemcpyAsync(p->meta_host + 2, p->counters.as<unsigned long long>() + 7, sizeof(int),
                                      cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(p->ctx, err, "band status");
    if (p->meta_host[2]) return set_error(p->ctx, VB_ERR_TIMEOUT, "band_reduce: a tile wait timed out");
    return VB_OK;
}

}  // namespace

vb_status vb_hs_plan_execute(vb_hs_plan* p, const double* S, const double* h, const double* eri, int mem,
                             double* H_out, double* S_out) {
    if (!p) return VB_ERR_INVALID;
    vb_context* ctx = p->ctx;
    if (!S || !h || !eri || !H_out || !S_out) return set_error(ctx, VB_ERR_INVALID, "vb_hs_plan_execute: null pointer");
    if (mem != VB_MEM_HOST && mem != VB_MEM_DEVICE) return set_error(ctx, VB_ERR_INVALID, "bad memory space");
    return execute_impl(p, S, h, eri, mem, H_out, S_out);
}

vb_status vb_hs_plan_root_gradient(vb_hs_plan* p, const double* S, const double* h, const double* eri,
                                   double tolerance, double* energy, double* coefficients, double* dS_out,
                                   double* dh_out, const double* ri_factors, int n_aux, double* dri_out) {
    if (!p) return VB_ERR_INVALID;
    vb_context* ctx = p->ctx;
    if (!S || !h || !eri || !energy)
        return set_error(ctx, VB_ERR_INVALID, "vb_hs_plan_root_gradient: null pointer");
    vb_status st = execute_impl(p, S, h, eri, VB_MEM_HOST, nullptr, nullptr);
    if (st == VB_OK) st = band_status(p);
    if (st != VB_OK) return st;
    const int ns = p->n_str;
    std::vector<double> c(ns);
    double E = 0.0;
    if (ns <= 200) {
        DeviceBuffer w, V;
        if ((st = w.allocate(ctx, sizeof(double) * ns)) != VB_OK) return st;
        if ((st = V.allocate(ctx, sizeof(double) * (size_t)ns * ns)) != VB_OK) return st;
        int info = 0;
        st = vb_generalized_eigh(ctx, p->Hout.as<double>(), p->Sout.as<double>(), ns, VB_MEM_DEVICE, w.as<double>(),
                                 V.as<double>(), &info);
        if (st != VB_OK) return st;
        cudaError_t err = cudaMemcpyAsync(&E, w.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(c.data(), V.ptr, sizeof(double) * ns, cudaMemcpyDeviceToHost, ctx->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
        if (err != cudaSuccess) return cuda_error(ctx, err, "vb_hs_plan_root_gradient");
    } else {
        DeviceBuffer x;
        if ((st = x.allocate(ctx, sizeof(double) * ns)) != VB_OK) return st;
        int its = 0;
        st = vb_lowest_root(ctx, p->Hout.as<double>(), p->Sout.as<double>(), ns, VB_MEM_DEVICE, tolerance, 2000, &E,
                            x.as<double>(), &its);
        if (st != VB_OK) return st;
        cudaError_t err = cudaMemcpyAsync(c.data(), x.ptr, sizeof(double) * ns, cudaMemcpyDeviceToHost, ctx->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
        if (err != cudaSuccess) return cuda_error(ctx, err, "vb_hs_plan_root_gradient");
    }
    *energy = E;
    if (coefficients) std::copy(c.begin(), c.end(), coefficients);
    if (!dS_out || !dh_out) return VB_OK;
    return vb_hs_plan_gradient(p, S, h, eri, VB_MEM_HOST, c.data(), E, dS_out, dh_out, nullptr, ri_factors, n_aux,
                               dri_out);
}

vb_status vb_hs_plan_enable_phase_timing(vb_hs_plan* p, int enable) {
    if (!p) return VB_ERR_INVALID;
    p->timing = enable != 0;
    return VB_OK;
}

vb_status vb_hs_plan_phase_times(vb_hs_plan* p, double* ms, int count) {
    if (!p || !ms || count < 0) return VB_ERR_INVALID;
    for (int ph = 0; ph < count && ph < VB_PHASE_COUNT; ++ph) {
        double total = 0.0;
        for (int i = 0; i < p->used[ph]; ++i) {
            auto& pr = p->events[ph][i];
            cudaError_t err = cudaEventSynchronize(pr.second);
            if (err != cudaSuccess) return cuda_error(p->ctx, err, "phase timing");
            float t = 0.f;
            err = cudaEventElapsedTime(&t, pr.first, pr.second);
            if (err != cudaSuccess) return cuda_error(p->ctx, err, "phase timing");
            total += t;
        }
        ms[ph] = p->timing ? total : 0.0;
    }
    for (int ph = VB_PHASE_COUNT; ph < count; ++ph) ms[ph] = 0.0;
    return VB_OK;
}

vb_status vb_hs_plan_stats(const vb_hs_plan* p, vb_hs_stats* stats) {
    if (!p || !stats) return VB_ERR_INVALID;
    vb_hs_stats s = p->stats;
    if (p->evaluated) {
        unsigned long long c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        cudaError_t err = cudaMemcpyAsync(c, p->counters.ptr, sizeof(c), cudaMemcpyDeviceToHost, p->ctx->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(p->ctx->stream);
        if (err != cudaSuccess) return cuda_error(p->ctx, err, "stats download");
        if ((int)c[7]) return set_error(p->ctx, VB_ERR_TIMEOUT, "band_reduce: a tile wait timed out");
        auto all_exact = [&](int k) { return !frame_spin_supported(p->n, k, p->R); };
        const bool all_a = p->ka > 0 && all_exact(p->ka);
        const bool all_b = p->kb > 0 && !p->shared_tables && all_exact(p->kb);
        s.careful_spin_pairs = (long long)(all_a ? p->npairs_a : c[0]) + (long long)(all_b ? p->npairs_b : c[1]);
    }
    *stats = s;
    return VB_OK;
}

vb_status vb_hs_plan_determinant_pairs(vb_hs_plan* p, const double* S, const double* h, const double* eri,
                                       int64_t n_pairs, const int64_t* pairs, int mem, double* h_out, double* s_out) {
    if (!p) return VB_ERR_INVALID;
    vb_context* ctx = p->ctx;
    if (n_pairs < 0 || (n_pairs > 0 && (!pairs || !h_out || !s_out)))
        return set_error(ctx, VB_ERR_INVALID, "vb_hs_plan_determinant_pairs: bad arguments");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int launches = 0;
    const double *dS, *dh, *deri;
    vb_status st = prepare_spin_records(p, S, h, eri, mem, &dS, &dh, &deri, &launches);
    if (st != VB_OK) return st;
    if (mem == VB_MEM_HOST)
        for (int64_t i = 0; i < 2 * n_pairs; ++i)
            if (pairs[i] < 0 || pairs[i] >= p->n_det)
                return set_error(ctx, VB_ERR_INVALID, "determinant index out of range");
    DeviceBuffer dp, dh_o, ds_o;
    const long long* pp = reinterpret_cast<const long long*>(pairs);
    double *ho = h_out, *so = s_out;
    std::vector<int64_t> moved;
    if (mem == VB_MEM_HOST && !p->det_position.empty()) {
        // the caller's determinant indices -> the plan's order
        moved.resize((size_t)(2 * n_pairs));
        for (int64_t i = 0; i < 2 * n_pairs; ++i) moved[i] = p->det_position[pairs[i]];
        pairs = moved.data();
    }
    if (mem == VB_MEM_DEVICE && !p->det_position.empty() && n_pairs > 0) {
        if (!p->det_position_dev.ptr &&
            (st = upload(ctx, p->det_position_dev, p->det_position.data(), sizeof(long long) * p->n_det)) != VB_OK)
            return st;
        if ((st = dp.allocate(ctx, sizeof(int64_t) * 2 * n_pairs)) != VB_OK) return st;
        translate_pairs_kernel<<<(unsigned)std::min<long long>(4096, (2 * n_pairs + 255) / 256), 256, 0, s>>>(
            2 * n_pairs, reinterpret_cast<const long long*>(pairs), p->det_position_dev.as<long long>(), p->n_det,
            dp.as<long long>());
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return cuda_error(ctx, err, "vb_hs_plan_determinant_pairs");
        pp = dp.as<long long>();
    }
    if (mem == VB_MEM_HOST) {
        if ((st = upload(ctx, dp, pairs, sizeof(int64_t) * 2 * std::max<int64_t>(1, n_pairs))) != VB_OK) return st;
        if ((st = dh_o.allocate(ctx, sizeof(double) * std::max<int64_t>(1, n_pairs))) != VB_OK) return st;
        if ((st = ds_o.allocate(ctx, sizeof(double) * std::max<int64_t>(1, n_pairs))) != VB_OK) return st;
        pp = dp.as<long long>();
        ho = dh_o.as<double>();
        so = ds_o.as<double>();
    }
    cudaError_t err = launch_listed_pairs(full_args(p), n_pairs, pp, ho, so, s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "listed_pairs");
    if (mem == VB_MEM_HOST && n_pairs > 0) {
        err = cudaMemcpyAsync(h_out, ho, sizeof(double) * n_pairs, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(s_out, so, sizeof(double) * n_pairs, cudaMemcpyDeviceToHost, s);
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "listed pairs download");
    return VB_OK;
}

vb_status vb_resolve_overlaps(vb_context* ctx, int k, int64_t batch, const double* blocks, int mem, double* det_out,
                              int32_t* nullity_out, double* cofactor_out) {
    if (!ctx) return VB_ERR_INVALID;
    if (k < 1 || k > dev::KMAX || batch < 0 || !blocks || !det_out || !nullity_out)
        return set_error(ctx, VB_ERR_INVALID, "vb_resolve_overlaps: bad arguments");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    DeviceBuffer db, dd, dn, dc;
    const double* b = blocks;
    double* det = det_out;
    int* nul = nullity_out;
    double* cof = cofactor_out;
    vb_status st;
    const size_t kk = (size_t)k * k;
    if (mem == VB_MEM_HOST) {
        if ((st = upload(ctx, db, blocks, sizeof(double) * kk * std::max<int64_t>(1, batch))) != VB_OK) return st;
        if ((st = dd.allocate(ctx, sizeof(double) * std::max<int64_t>(1, batch))) != VB_OK) return st;
        if ((st = dn.allocate(ctx, sizeof(int) * std::max<int64_t>(1, batch))) != VB_OK) return st;
        if (cofactor_out && (st = dc.allocate(ctx, sizeof(double) * kk * std::max<int64_t>(1, batch))) != VB_OK)
            return st;
        b = db.as<double>();
        det = dd.as<double>();
        nul = dn.as<int>();
        cof = cofactor_out ? dc.as<double>() : nullptr;
    }
    cudaError_t err = launch_resolve_blocks(k, batch, b, det, nul, cof, s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "resolve_blocks");
    if (mem == VB_MEM_HOST && batch > 0) {
        err = cudaMemcpyAsync(det_out, det, sizeof(double) * batch, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(nullity_out, nul, sizeof(int) * batch, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess && cofactor_out)
            err = cudaMemcpyAsync(cofactor_out, cof, sizeof(double) * kk * batch, cudaMemcpyDeviceToHost, s);
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "resolve download");
    return VB_OK;
}

vb_status vb_same_spin_pairs(vb_context* ctx, int n, int k, int64_t batch, const int32_t* occ_left,
                             const int32_t* occ_right, const double* S, const double* h, const double* eri, int mem,
                             double* out_scalars, double* cofactor_out) {
    if (!ctx) return VB_ERR_INVALID;
    if (n < 1 || n > kMaxOrbitals || k < 1 || k > dev::KMAX || k > n || batch < 0 || !occ_left || !occ_right || !S ||
        !h || !eri || !out_scalars)
        return set_error(ctx, VB_ERR_INVALID, "vb_same_spin_pairs: bad arguments");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t np = (size_t)n * (n + 1) / 2;
    const size_t kk = (size_t)k * k;
    const int64_t nb = std::max<int64_t>(1, batch);
    DeviceBuffer dl, dr, dS, dh, de, dsc, dc;
    const int* l = occ_left;
    const int* r = occ_right;
    const double *pS = S, *ph = h, *pe = eri;
    double* sc = out_scalars;
    double* cof = cofactor_out;
    vb_status st;
    if (mem == VB_MEM_HOST) {
        for (int64_t i = 0; i < batch * k; ++i)
            if (occ_left[i] < 0 || occ_left[i] >= n || occ_right[i] < 0 || occ_right[i] >= n)
                return set_error(ctx, VB_ERR_INVALID, "orbital index out of range");
        if ((st = upload(ctx, dl, occ_left, sizeof(int) * k * nb)) != VB_OK) return st;
        if ((st = upload(ctx, dr, occ_right, sizeof(int) * k * nb)) != VB_OK) return st;
        if ((st = upload(ctx, dS, S, sizeof(double) * n * n)) != VB_OK) return st;
        if ((st = upload(ctx, dh, h, sizeof(double) * n * n)) != VB_OK) return st;
        if ((st = upload(ctx, de, eri, sizeof(double) * np * (np + 1) / 2)) != VB_OK) return st;
        if ((st = dsc.allocate(ctx, sizeof(double) * 4 * nb)) != VB_OK) return st;
        if (cofactor_out && (st = dc.allocate(ctx, sizeof(double) * kk * nb)) != VB_OK) return st;
        l = dl.as<int>();
        r = dr.as<int>();
        pS = dS.as<double>();
        ph = dh.as<double>();
        pe = de.as<double>();
        sc = dsc.as<double>();
        cof = cofactor_out ? dc.as<double>() : nullptr;
    }
    cudaError_t err = launch_same_spin_list(n, k, batch, l, r, pS, ph, pe, sc, cof, s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "same_spin_list");
    if (mem == VB_MEM_HOST && batch > 0) {
        err = cudaMemcpyAsync(out_scalars, sc, sizeof(double) * 4 * batch, cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess && cofactor_out)
            err = cudaMemcpyAsync(cofactor_out, cof, sizeof(double) * kk * batch, cudaMemcpyDeviceToHost, s);
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_error(ctx, err, "same-spin download");
    return VB_OK;
}

}  // extern "C"
