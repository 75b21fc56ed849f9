// Host-side structure-class generation and structure -> determinant expansion.
//
// Generation follows src/input/loading/generated_structures.cpp of the reference:
// Young-pattern rows (:249-297), covalent alpha/beta pattern pairs (:299-391), bond
// reordering (:393-433), class parsing and counting (:131-245), and the flat row layout
// (:475-603).  Expansion follows src/vbscf/structures/expansion/expander.cpp: every bond with
// distinct ends is swapped independently, the +-1 coefficient is the product of the
// alpha and beta sort parities (:34-70, 130-192), strings are ordered by occupation mask and
// determinants by (alpha rank, beta rank), with CSR terms per determinant in structure
// order and coalesced duplicates (:287-557, types.hpp:46-99).
#include <algorithm>
#include <cctype>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>

#include "internal.h"

namespace vbcore {
namespace {

uint64_t binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    uint64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
    return r;
}

template <typename Visit>
void young_patterns(int n_alpha, int n_beta, int n_orbitals, int row_stride, Visit&& visit) {
    if (n_alpha <= 0) return;
    if (n_orbitals <= 0 || n_orbitals < n_alpha) throw std::invalid_argument("invalid orbital count in structure generator");
    std::vector<int> row(row_stride, 0);
    for (int i = 0; i < n_alpha; ++i) row[i] = i + 1;
    const int mult = n_alpha - n_beta + 1;
    std::vector<int> maxv(n_alpha, 0);
    if (mult == 1) {
        maxv[n_beta - 1] = n_orbitals - 1;
    } else {
        maxv[n_alpha - 1] = n_orbitals;
        for (int idx = n_alpha - 1; idx >= n_beta + 1; --idx) maxv[idx - 1] = maxv[idx] - 1;
        if (n_beta > 0) maxv[n_beta - 1] = maxv[n_beta] - 2;
    }
    for (int idx = n_beta - 1; idx >= 1; --idx) maxv[idx - 1] = maxv[idx] - 2;
    while (true) {
        visit(row);
        int pivot = n_alpha - 1;
        while (pivot >= 0 && row[pivot] == maxv[pivot]) --pivot;
        if (pivot < 0) break;
        ++row[pivot];
        for (int s = pivot + 1; s < n_alpha; ++s) row[s] = row[s - 1] + 1;
    }
}

bool compatible(const std::vector<int>& alpha, const std::vector<int>& cand, int n_alpha, int n_beta) {
    for (int bi = 0; bi < n_beta; ++bi) {
        if (cand[bi] < alpha[bi]) return false;
        for (int ai = bi; ai < n_alpha; ++ai)
            if (cand[bi] == alpha[ai]) return false;
    }
    return true;
}

void pad_open_shell(std::vector<int>& beta, int n_alpha, int n_beta, int n_orbitals) {
    for (int idx = n_beta; idx < n_alpha; ++idx) beta[idx] = n_orbitals + n_alpha - idx;
}

template <typename Visit>
void covalent_pattern_pairs(int n_alpha, int n_beta, int n_orbitals, int row_stride, Visit&& visit) {
    if (n_alpha <= 0) return;
    if (n_beta <= 0) {
        young_patterns(n_alpha, 0, n_orbitals, row_stride,
                       [&](const std::vector<int>& a) { visit(a, std::vector<int>(row_stride, 0)); });
        return;
    }
    if (n_alpha + n_beta == n_orbitals) {
        young_patterns(n_alpha, n_beta, n_orbitals, row_stride, [&](const std::vector<int>& a) {
            std::vector<int> b(row_stride, 0);
            int nb = 0;
            for (int lab = 1; lab <= n_orbitals; ++lab)
                if (std::find(a.begin(), a.begin() + n_alpha, lab) == a.begin() + n_alpha) b[nb++] = lab;
            pad_open_shell(b, n_alpha, n_beta, n_orbitals);
            visit(a, b);
        });
        return;
    }
    young_patterns(n_alpha, n_beta, n_orbitals, row_stride, [&](const std::vector<int>& a) {
        young_patterns(n_beta, 0, n_orbitals, n_beta, [&](const std::vector<int>& cand) {
            if (!compatible(a, cand, n_alpha, n_beta)) return;
            std::vector<int> b(row_stride, 0);
            std::copy(cand.begin(), cand.begin() + n_beta, b.begin());
            pad_open_shell(b, n_alpha, n_beta, n_orbitals);
            visit(a, b);
        });
    });
}

// Pair each alpha label, largest first, with the smallest remaining beta label above it; the
// returned alpha row lists the partner of beta_row[b] at position b.
std::vector<int> reorder_bonds(const std::vector<int>& alpha, const std::vector<int>& beta, int n_vector,
                               int n_row, int n_orbitals) {
    std::vector<int> left(3 * n_orbitals + 2, 0), right(3 * n_orbitals + 2, 0);
    std::vector<int> rb(beta.begin(), beta.begin() + n_row);
    int remaining = n_vector;
    for (int v = 0; v < n_vector; ++v) right[rb[v] - 1] = v + 1;
    for (int v = n_vector; v >= 1; --v) {
        const int left_max = alpha[remaining - 1];
        int m = 0;
        for (; m < remaining; ++m)
            if (left_max <= rb[m]) {
                left[left_max - 1] = right[rb[m] - 1];
                break;
            }
        if (m >= remaining) throw std::runtime_error("structure generator: unmatched bond label");
        for (int s = m; s < remaining - 1; ++s) rb[s] = rb[s + 1];
        --remaining;
    }
    for (int v = 0; v < n_vector; ++v) rb[left[alpha[v] - 1] - 1] = alpha[v];
    std::vector<int> out = alpha;
    for (int v = 0; v < n_vector; ++v) out[v] = rb[v];
    return out;
}

uint64_t spin_tableau_count(int n, int spin) {
    if (n < 0 || spin <= 0 || spin > n + 1) return 0;
    if (n == 0) return 1;
    if ((n - spin + 1) % 2) return 0;
    const int beta = (n - spin + 1) / 2;
    return binom(n, beta) - (beta ? binom(n, beta - 1) : 0);
}

uint64_t count_for_class(int ic, int ndb, int n_skipped, int n_orb, int n_el, int mult) {
    const int tab = n_orb - 2 * ic - n_skipped + ndb;
    if (tab < 0) return 0;
    return binom(n_orb, ic) * binom(n_orb - ic, n_skipped + ic - ndb) * spin_tableau_count(tab, mult);
}

std::vector<int> parse_classes(const std::string& keyword_in, int n_orb, int n_el, int mult) {
    std::string kw = keyword_in;
    for (char& ch : kw) ch = (char)std::toupper((unsigned char)ch);
    const int ndb = std::max(0, n_el - n_orb);
    const int reduced_beta = (n_el - 2 * ndb - mult + 1) / 2;
    if (reduced_beta < 0) throw std::invalid_argument("structure class generation requires a non-negative beta count");
    std::vector<int> classes;
    if (kw.find("FULL") != std::string::npos) {
        for (int i = 0; i <= reduced_beta; ++i) classes.push_back(i);
    } else {
        if (kw.find("COV") != std::string::npos) classes.push_back(0);
        const size_t pos = kw.find("ION(");
        if (pos != std::string::npos) {
            const size_t end = kw.find(')', pos + 4);
            if (end == std::string::npos) throw std::invalid_argument("structure class contains ION( without ')'");
            std::string body = kw.substr(pos + 4, end - pos - 4);
            for (char& ch : body)
                if (ch == ',') ch = ' ';
            size_t i = 0;
            while (i < body.size()) {
                while (i < body.size() && body[i] == ' ') ++i;
                size_t j = i;
                while (j < body.size() && body[j] != ' ') ++j;
                if (j > i) {
                    const std::string tok = body.substr(i, j - i);
                    const size_t dash = tok.find('-');
                    if (dash != std::string::npos) {
                        const int a = std::stoi(tok.substr(0, dash)), b = std::stoi(tok.substr(dash + 1));
                        for (int c = a; c <= b; ++c) classes.push_back(c);
                    } else {
                        classes.push_back(std::stoi(tok));
                    }
                }
                i = j;
            }
        } else if (kw.find("ION") != std::string::npos) {
            for (int i = 1; i <= reduced_beta; ++i) classes.push_back(i);
        }
    }
    if (classes.empty()) throw std::invalid_argument("unsupported or empty structure class specification: " + keyword_in);
    std::sort(classes.begin(), classes.end());
    classes.erase(std::unique(classes.begin(), classes.end()), classes.end());
    if (classes.front() < 0) throw std::invalid_argument("structure class cannot be smaller than 0");
    if (classes.back() > reduced_beta) throw std::invalid_argument("structure class exceeds the maximum ionic order");
    for (int& c : classes) c += ndb;
    return classes;
}

int sort_sign(const std::vector<int>& orbs, uint64_t* mask) {
    uint64_t m = 0;
    int sign = 1;
    for (int o : orbs) {
        if (o < 0 || o >= 64) throw std::invalid_argument("active orbital index out of range (0..63)");
        const uint64_t flag = uint64_t{1} << o;
        if (m & flag) throw std::invalid_argument("duplicate orbital in an occupied spin string");
        const uint64_t higher = o == 63 ? 0 : (m >> (o + 1));
        if (__builtin_popcountll(higher) & 1) sign = -sign;
        m |= flag;
    }
    *mask = m;
    return sign;
}

}  // namespace

std::vector<std::vector<int>> generate_structures(const std::string& keyword, int n_orb, int n_el, int mult,
                                                  int n_inactive) {
    if (n_orb <= 0 || n_el <= 0 || mult <= 0) throw std::invalid_argument("counts must be positive");
    const int nb = (n_el - mult + 1) / 2;
    const int na = n_el - nb;
    if (nb < 0) throw std::invalid_argument("active beta electron count is negative in structure generator");
    if (nb > n_orb) throw std::invalid_argument("active beta electron count exceeds the active orbital count");
    const int n_total = n_el + 2 * n_inactive;
    std::vector<std::vector<int>> out;
    if ((nb == 0 && n_el == mult - 1 && n_el == n_orb) || (nb == n_orb && mult == 1)) {
        std::vector<int> row(n_total, 0);
        const int tp = n_inactive + nb;
        for (int i = 0; i < tp; ++i) row[2 * i] = row[2 * i + 1] = i + 1;
        for (int o = 0; o < mult - 1; ++o) row[2 * tp + o] = tp + o + 1;
        out.push_back(row);
        return out;
    }
    const int shift = n_inactive;
    auto emit = [&](int ic, const std::vector<int>& ion, const std::vector<int>& remaining, const std::vector<int>& a,
                    const std::vector<int>& b, int n_cov_a, int n_cov_b) {
        std::vector<int> row(n_total, 0);
        for (int i = 0; i < n_inactive; ++i) row[2 * i] = row[2 * i + 1] = i + 1;
        const int off = 2 * n_inactive;
        if (ic > 0) {
            for (int ii = 0; ii < ic; ++ii) row[off + 2 * ii] = row[off + 2 * ii + 1] = ion[ii] + shift;
            for (int bi = 0; bi < n_cov_b; ++bi) {
                row[off + 2 * ic + 2 * bi] = remaining[a[bi] - 1] + shift;
                row[off + 2 * ic + 2 * bi + 1] = remaining[b[bi] - 1] + shift;
            }
            for (int ai = n_cov_b; ai < n_cov_a; ++ai) row[off + 2 * ic + n_cov_b + ai] = remaining[a[ai] - 1] + shift;
        } else {
            for (int bi = 0; bi < n_cov_b; ++bi) {
                row[off + 2 * bi] = a[bi] + shift;
                row[off + 2 * bi + 1] = b[bi] + shift;
            }
            for (int ai = n_cov_b; ai < n_cov_a; ++ai) row[off + n_cov_b + ai] = a[ai] + shift;
        }
        out.push_back(std::move(row));
    };
    const std::vector<int> classes = parse_classes(keyword, n_orb, n_el, mult);
    for (int ic : classes) {
        if (ic < 0 || ic > nb) throw std::invalid_argument("structure class exceeds the active beta electron count");
        const int n_cov_a = na - ic, n_cov_b = nb - ic;
        if (ic > 0) {
            young_patterns(ic, 0, n_orb, ic, [&](const std::vector<int>& ion) {
                std::vector<int> remaining;
                for (int lab = 1; lab <= n_orb; ++lab)
                    if (std::find(ion.begin(), ion.begin() + ic, lab) == ion.begin() + ic) remaining.push_back(lab);
                if (n_cov_a <= 0) {
                    emit(ic, ion, remaining, {}, {}, n_cov_a, n_cov_b);
                    return;
                }
                covalent_pattern_pairs(n_cov_a, n_cov_b, n_orb - ic, na,
                                       [&](const std::vector<int>& a, const std::vector<int>& b) {
                                           std::vector<int> ra = n_cov_b > 0 ? reorder_bonds(a, b, n_cov_a, na, n_orb) : a;
                                           emit(ic, ion, remaining, ra, b, n_cov_a, n_cov_b);
                                       });
            });
        } else {
            covalent_pattern_pairs(na, nb, n_orb, na, [&](const std::vector<int>& a, const std::vector<int>& b) {
                std::vector<int> ra = nb > 0 ? reorder_bonds(a, b, na, na, n_orb) : a;
                emit(0, {}, {}, ra, b, n_cov_a, n_cov_b);
            });
        }
    }
    const int n_skipped = std::max(0, n_orb - n_el);
    const int ndb = std::max(0, n_el - n_orb);
    uint64_t expected = 0;
    for (int ic : classes) expected += count_for_class(ic, ndb, n_skipped, n_orb, n_el, mult);
    if (out.size() != expected) throw std::runtime_error("raw structure generation count mismatch");
    return out;
}

Expansion expand_structures(const std::vector<std::vector<int>>& rows, int n_el_active, int mult, int n_inactive) {
    const int n_open = mult - 1;
    const int n_paired = n_el_active - n_open;
    if (n_open < 0 || n_paired < 0 || n_paired % 2) throw std::invalid_argument("raw structure electron and spin counts are inconsistent");
    const int nb = n_paired / 2;
    Expansion ex;
    ex.n_structures = (int)rows.size();
    ex.n_alpha = nb + n_open;
    ex.n_beta = nb;
    std::map<std::pair<uint64_t, uint64_t>, std::vector<std::pair<int, double>>> per_det;
    std::vector<int> active(n_el_active), alpha, beta, variable;
    for (int s = 0; s < (int)rows.size(); ++s) {
        const auto& row = rows[s];
        if ((int)row.size() < n_el_active + 2 * n_inactive) throw std::invalid_argument("structure row too short");
        for (int i = 0; i < n_el_active; ++i) active[i] = row[i + 2 * n_inactive] - n_inactive - 1;
        variable.clear();
        for (int p = 0; p < nb; ++p)
            if (active[2 * p] != active[2 * p + 1]) variable.push_back(p);
        const uint64_t n_choice = uint64_t{1} << variable.size();
        for (uint64_t choice = 0; choice < n_choice; ++choice) {
            alpha.clear();
            beta.clear();
            size_t vi = 0;
            for (int p = 0; p < nb; ++p) {
                int sw = 0;
                if (vi < variable.size() && variable[vi] == p) {
                    sw = (int)((choice >> vi) & 1);
                    ++vi;
                }
                alpha.push_back(active[2 * p + sw]);
                beta.push_back(active[2 * p + 1 - sw]);
            }
            for (int i = 2 * nb; i < n_el_active; ++i) alpha.push_back(active[i]);
            uint64_t am = 0, bm = 0;
            const int sign = sort_sign(alpha, &am) * sort_sign(beta, &bm);
            per_det[{am, bm}].push_back({s, (double)sign});
        }
    }
    std::vector<uint64_t> am, bm;
    for (const auto& kv : per_det) {
        am.push_back(kv.first.first);
        bm.push_back(kv.first.second);
    }
    std::sort(am.begin(), am.end());
    am.erase(std::unique(am.begin(), am.end()), am.end());
    std::sort(bm.begin(), bm.end());
    bm.erase(std::unique(bm.begin(), bm.end()), bm.end());
    auto rank = [](const std::vector<uint64_t>& v, uint64_t m) {
        return (int32_t)(std::lower_bound(v.begin(), v.end(), m) - v.begin());
    };
    struct Key {
        int32_t a, b;
        const std::vector<std::pair<int, double>>* terms;
    };
    std::vector<Key> keys;
    keys.reserve(per_det.size());
    for (const auto& kv : per_det) keys.push_back({rank(am, kv.first.first), rank(bm, kv.first.second), &kv.second});
    std::sort(keys.begin(), keys.end(), [](const Key& x, const Key& y) { return x.a != y.a ? x.a < y.a : x.b < y.b; });
    ex.alpha_strings = am;
    ex.beta_strings = bm;
    ex.offsets.push_back(0);
    for (const Key& k : keys) {
        ex.det_alpha.push_back(k.a);
        ex.det_beta.push_back(k.b);
        std::map<int, double> merged;
        for (const auto& t : *k.terms) merged[t.first] += t.second;
        for (const auto& m : merged)
            if (m.second != 0.0) {
                ex.term_structure.push_back(m.first);
                ex.term_coefficient.push_back(m.second);
            }
        ex.offsets.push_back((int64_t)ex.term_structure.size());
    }
    return ex;
}

}  // namespace vbcore

using namespace vbcore;

extern "C" {

vb_status vb_generate_structures(const char* keyword, int n_active_orbitals, int n_active_electrons,
                                 int spin_multiplicity, int n_inactive, int64_t* n_structures_out, int32_t* rows_out,
                                 int64_t rows_capacity) {
    if (!keyword || !n_structures_out) return set_error(nullptr, VB_ERR_INVALID, "vb_generate_structures: null argument");
    try {
        auto rows = generate_structures(keyword, n_active_orbitals, n_active_electrons, spin_multiplicity, n_inactive);
        *n_structures_out = (int64_t)rows.size();
        if (rows_out) {
            const int64_t width = n_active_electrons + 2 * n_inactive;
            if (rows_capacity < (int64_t)rows.size() * width)
                return set_error(nullptr, VB_ERR_INVALID, "vb_generate_structures: rows_out too small");
            for (size_t s = 0; s < rows.size(); ++s)
                for (int64_t i = 0; i < width; ++i) rows_out[s * width + i] = rows[s][i];
        }
        return VB_OK;
    } catch (const std::exception& e) {
        return set_error(nullptr, VB_ERR_INVALID, e.what());
    }
}

vb_status vb_expand_structures(const int32_t* rows, int64_t n_structures, int n_active_electrons,
                               int spin_multiplicity, int n_inactive, vb_expansion_sizes* sizes,
                               uint64_t* alpha_strings, uint64_t* beta_strings, int32_t* det_alpha, int32_t* det_beta,
                               int64_t* term_offsets, int32_t* term_structure, double* term_coefficient) {
    if (!rows || !sizes || n_structures <= 0) return set_error(nullptr, VB_ERR_INVALID, "vb_expand_structures: bad arguments");
    try {
        const int width = n_active_electrons + 2 * n_inactive;
        std::vector<std::vector<int>> r(n_structures, std::vector<int>(width));
        for (int64_t s = 0; s < n_structures; ++s)
            for (int i = 0; i < width; ++i) r[s][i] = rows[s * width + i];
        Expansion ex = expand_structures(r, n_active_electrons, spin_multiplicity, n_inactive);
        sizes->n_structures = ex.n_structures;
        sizes->n_alpha_electrons = ex.n_alpha;
        sizes->n_beta_electrons = ex.n_beta;
        sizes->n_alpha_strings = (int32_t)ex.alpha_strings.size();
        sizes->n_beta_strings = (int32_t)ex.beta_strings.size();
        sizes->n_determinants = (int64_t)ex.det_alpha.size();
        sizes->n_terms = (int64_t)ex.term_structure.size();
        if (alpha_strings) std::copy(ex.alpha_strings.begin(), ex.alpha_strings.end(), alpha_strings);
        if (beta_strings) std::copy(ex.beta_strings.begin(), ex.beta_strings.end(), beta_strings);
        if (det_alpha) std::copy(ex.det_alpha.begin(), ex.det_alpha.end(), det_alpha);
        if (det_beta) std::copy(ex.det_beta.begin(), ex.det_beta.end(), det_beta);
        if (term_offsets) std::copy(ex.offsets.begin(), ex.offsets.end(), term_offsets);
        if (term_structure) std::copy(ex.term_structure.begin(), ex.term_structure.end(), term_structure);
        if (term_coefficient) std::copy(ex.term_coefficient.begin(), ex.term_coefficient.end(), term_coefficient);
        return VB_OK;
    } catch (const std::exception& e) {
        return set_error(nullptr, VB_ERR_INVALID, e.what());
    }
}

}  // extern "C"
