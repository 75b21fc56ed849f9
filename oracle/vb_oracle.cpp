// CPU oracle for the VBSCF determinant-pair hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity checker and the timed CPU
// baseline; no product code links or calls it. It restates, in plain C++ with
// no Eigen/LAPACK, the reference algorithm of Tao-Xia/xmvb-cpp (paths relative
// to that project):
//
//   * overlap resolution: src/vbscf/determinants/algebra/overlap.cpp:50-109
//     (Eigen FullPivLU with a relative rank threshold, BDCSVD fallback).
//     Eigen is a third-party dependency that is absent here (unpinned,
//     not vendored). Its published FullPivLU semantics are restated below:
//     complete pivoting, first strict maximum in column-major order,
//     rank = #{i : |u_ii| > threshold * max_i |u_ii|}. BDCSVD falls back to a
//     two-sided Jacobi SVD for matrices smaller than 16; a two-sided Jacobi SVD
//     is used here, with singular values sorted in decreasing order.
//   * first cofactors: src/vbscf/determinants/pairs/contractions.cpp:172-237
//   * second cofactors: src/vbscf/determinants/pairs/contractions.cpp:901-983
//   * same-spin H: src/vbscf/determinants/algebra/hamiltonian.cpp:35-163
//   * opposite-spin coupling: src/vbscf/determinants/pairs/evaluator.cpp:95-148
//   * full pair: src/vbscf/determinants/pairs/evaluator.cpp:354-384, 421-466
//   * structure H/S: src/vbscf/structures/assembly/hamiltonian_overlap.cpp:890-1022
//     (H_IJ = sum_{d in I, e in J} c_d c_e H_de; any deterministic FP64 order)
//   * cached evaluation (the reference's CPU hot-loop shape, the timed CPU baseline):
//     build_same_spin_pair_cache, src/vbscf/determinants/pairs/same_spin_cache.cpp:430-477
//     (every ordered spin pair of a string table, OpenMP dynamic,1 over left strings), with the
//     sparse packed-pair projection and its dense image over the pair kernel
//     (same_spin_cache.cpp:166-182, 186-284), and per determinant pair the sparse dot
//     contract_sparse_projection_with_dense_image, contractions.cpp:136-147
//   * packed indices: src/core/pair_index.cpp:10-44
//   * RI transform: src/integrals/ao/ri_transform.cpp:10-37,
//     src/integrals/active/ri.cpp:13-96
//
// Matrices are column-major (m[col * rows + row]); overlap blocks have rows =
// right determinant, columns = left determinant
// (src/vbscf/determinants/contracts/types.hpp:13-15, 62-66).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline long long pair_index(long long a, long long b) {
    const long long hi = a > b ? a : b;
    const long long lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

inline double eri_lookup(const double* packed, int p, int q, int r, int s) {
    return packed[pair_index(pair_index(p, q), pair_index(r, s))];
}

struct Resolved {
    int k = 0;
    std::vector<double> x;  // k*k overlap block
    double det = 0.0;
    int nullity = 0;
    bool have_inverse = false;
    std::vector<double> inv;  // k*k
    bool have_svd = false;
    std::vector<double> sv, u, v;  // sv descending; u, v column-major
    double parity = 1.0;
};

// Eigen FullPivLU restated: returns rank; fills det and (when rank == k) inverse.
int full_pivot_lu(int k, const double* x, double threshold, double* det, std::vector<double>* inv) {
    std::vector<double> lu(x, x + k * k);
    auto at = [&](int i, int j) -> double& { return lu[j * k + i]; };
    std::vector<int> rowt(k), colt(k);
    int ntrans = 0;
    int nonzero = k;
    double maxpivot = 0.0;
    for (int s = 0; s < k; ++s) {
        double best = -1.0;
        int br = s, bc = s;
        for (int j = s; j < k; ++j)
            for (int i = s; i < k; ++i) {
                const double v = std::fabs(at(i, j));
                if (v > best) {
                    best = v;
                    br = i;
                    bc = j;
                }
            }
        if (best == 0.0) {
            nonzero = s;
            for (int t = s; t < k; ++t) {
                rowt[t] = t;
                colt[t] = t;
            }
            break;
        }
        if (best > maxpivot) maxpivot = best;
        rowt[s] = br;
        colt[s] = bc;
        if (br != s) {
            for (int j = 0; j < k; ++j) std::swap(at(s, j), at(br, j));
            ++ntrans;
        }
        if (bc != s) {
            for (int i = 0; i < k; ++i) std::swap(at(i, s), at(i, bc));
            ++ntrans;
        }
        const double piv = at(s, s);
        for (int i = s + 1; i < k; ++i) at(i, s) /= piv;
        for (int j = s + 1; j < k; ++j)
            for (int i = s + 1; i < k; ++i) at(i, j) -= at(i, s) * at(s, j);
    }
    int rank = 0;
    const double cut = maxpivot * threshold;
    for (int i = 0; i < nonzero; ++i)
        if (std::fabs(at(i, i)) > cut) ++rank;
    double d = (ntrans % 2) ? -1.0 : 1.0;
    for (int i = 0; i < k; ++i) d *= at(i, i);
    *det = d;
    if (inv != nullptr && rank == k) {
        inv->assign(k * k, 0.0);
        std::vector<double> c(k);
        for (int col = 0; col < k; ++col) {
            std::fill(c.begin(), c.end(), 0.0);
            c[col] = 1.0;
            for (int s = 0; s < k; ++s) std::swap(c[s], c[rowt[s]]);
            for (int i = 0; i < k; ++i)
                for (int j = 0; j < i; ++j) c[i] -= at(i, j) * c[j];
            for (int i = k - 1; i >= 0; --i) {
                for (int j = i + 1; j < k; ++j) c[i] -= at(i, j) * c[j];
                c[i] /= at(i, i);
            }
            for (int s = k - 1; s >= 0; --s) std::swap(c[s], c[colt[s]]);
            for (int i = 0; i < k; ++i) (*inv)[col * k + i] = c[i];
        }
    }
    return rank;
}

// Two-sided cyclic Jacobi SVD of a square matrix: x = u diag(sv) v^T.
void jacobi_svd(int k, const double* x, std::vector<double>* sv, std::vector<double>* u,
                std::vector<double>* v) {
    std::vector<double> a(x, x + k * k);
    auto A = [&](int i, int j) -> double& { return a[j * k + i]; };
    u->assign(k * k, 0.0);
    v->assign(k * k, 0.0);
    for (int i = 0; i < k; ++i) (*u)[i * k + i] = (*v)[i * k + i] = 1.0;
    double scale = 0.0;
    for (double e : a) scale = std::max(scale, std::fabs(e));
    if (scale == 0.0) scale = 1.0;
    for (double& e : a) e /= scale;
    const double eps2 = 2.0 * std::numeric_limits<double>::epsilon();
    const double tiny = std::numeric_limits<double>::min();
    double maxdiag = 0.0;
    for (int i = 0; i < k; ++i) maxdiag = std::max(maxdiag, std::fabs(A(i, i)));
    for (int sweep = 0; sweep < 100; ++sweep) {
        bool done = true;
        for (int p = 1; p < k; ++p)
            for (int q = 0; q < p; ++q) {
                const double thr = std::max(tiny, eps2 * maxdiag);
                if (!(std::fabs(A(p, q)) > thr || std::fabs(A(q, p)) > thr)) continue;
                done = false;
                // 2x2 block M over (q, p). G1 = [[c1, s1], [-s1, c1]] makes G1 M symmetric
                // (s1/c1 = (m10 - m01)/(m00 + m11)); J = [[c2, s2], [-s2, c2]] then
                // diagonalizes it: J^T G1 M J = diag. Rows take L = J^T G1, columns take J.
                const double m00 = A(q, q), m01 = A(q, p), m10 = A(p, q), m11 = A(p, p);
                const double t = m00 + m11, d = m10 - m01;
                double c1 = 1.0, s1 = 0.0;
                if (std::fabs(d) >= tiny) {
                    const double uu = t / d;
                    const double tmp = std::sqrt(1.0 + uu * uu);
                    s1 = (uu >= 0 ? 1.0 : -1.0) / tmp;
                    c1 = std::fabs(uu) / tmp;
                }
                const double b00 = c1 * m00 + s1 * m10;
                const double b01 = c1 * m01 + s1 * m11;
                const double b11 = -s1 * m01 + c1 * m11;
                double c2 = 1.0, s2 = 0.0;
                if (b01 != 0.0) {
                    const double tau = (b11 - b00) / (2.0 * b01);
                    const double tt = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
                    c2 = 1.0 / std::sqrt(1.0 + tt * tt);
                    s2 = tt * c2;
                }
                const double l00 = c2 * c1 + s2 * s1, l01 = c2 * s1 - s2 * c1;
                const double l10 = s2 * c1 - c2 * s1, l11 = s2 * s1 + c2 * c1;
                for (int j = 0; j < k; ++j) {
                    const double aq = A(q, j), ap = A(p, j);
                    A(q, j) = l00 * aq + l01 * ap;
                    A(p, j) = l10 * aq + l11 * ap;
                }
                for (int i = 0; i < k; ++i) {
                    const double aq = A(i, q), ap = A(i, p);
                    A(i, q) = c2 * aq - s2 * ap;
                    A(i, p) = s2 * aq + c2 * ap;
                }
                // u <- u L^T (columns q,p); v <- v J
                for (int i = 0; i < k; ++i) {
                    double& uq = (*u)[q * k + i];
                    double& up = (*u)[p * k + i];
                    const double a0 = uq, a1 = up;
                    uq = l00 * a0 + l01 * a1;
                    up = l10 * a0 + l11 * a1;
                    double& vq = (*v)[q * k + i];
                    double& vp = (*v)[p * k + i];
                    const double b0 = vq, b1 = vp;
                    vq = c2 * b0 - s2 * b1;
                    vp = s2 * b0 + c2 * b1;
                }
                maxdiag = std::max(maxdiag, std::max(std::fabs(A(p, p)), std::fabs(A(q, q))));
            }
        if (done) break;
    }
    sv->assign(k, 0.0);
    for (int i = 0; i < k; ++i) {
        const double di = A(i, i);
        (*sv)[i] = std::fabs(di) * scale;
        if (di < 0)
            for (int r = 0; r < k; ++r) (*u)[i * k + r] = -(*u)[i * k + r];
    }
    std::vector<int> order(k);
    for (int i = 0; i < k; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a0, int b0) { return (*sv)[a0] > (*sv)[b0]; });
    std::vector<double> s2v(k), u2(k * k), v2(k * k);
    for (int i = 0; i < k; ++i) {
        s2v[i] = (*sv)[order[i]];
        for (int r = 0; r < k; ++r) {
            u2[i * k + r] = (*u)[order[i] * k + r];
            v2[i * k + r] = (*v)[order[i] * k + r];
        }
    }
    *sv = s2v;
    *u = u2;
    *v = v2;
}

double orth_det_sign(int k, const std::vector<double>& q) {
    double det = 0.0;
    full_pivot_lu(k, q.data(), 1e-300, &det, nullptr);
    return det >= 0.0 ? 1.0 : -1.0;
}

Resolved resolve(int k, const double* x, double threshold) {
    Resolved r;
    r.k = k;
    r.x.assign(x, x + k * k);
    if (k == 0) {
        r.det = 1.0;
        return r;
    }
    double det = 0.0;
    std::vector<double> inv;
    const int rank = full_pivot_lu(k, x, threshold, &det, &inv);
    if (rank == k) {
        r.nullity = 0;
        r.det = det;
        r.have_inverse = true;
        r.inv = inv;
        return r;
    }
    jacobi_svd(k, x, &r.sv, &r.u, &r.v);
    r.have_svd = true;
    r.nullity = 0;
    for (double s : r.sv)
        if (s < threshold) ++r.nullity;
    r.parity = orth_det_sign(k, r.u) * orth_det_sign(k, r.v);
    if (r.nullity == 0) {
        double prod = 1.0;
        for (double s : r.sv) prod *= s;
        r.det = r.parity * prod;
        r.inv.assign(k * k, 0.0);
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) {
                double acc = 0.0;
                for (int t = 0; t < k; ++t) acc += r.v[t * k + rr] * (1.0 / r.sv[t]) * r.u[t * k + c];
                r.inv[c * k + rr] = acc;
            }
        r.have_inverse = true;
    } else {
        r.det = 0.0;
    }
    return r;
}

double leading_product(const Resolved& r, int count) {
    double p = 1.0;
    for (int i = 0; i < count; ++i) p *= r.sv[i];
    return p;
}

// contractions.cpp:172-237
std::vector<double> first_cofactor(const Resolved& r) {
    const int k = r.k;
    std::vector<double> cof(k * k, 0.0);
    if (k == 0) return cof;
    if (k <= 3) {
        auto X = [&](int i, int j) { return r.x[j * k + i]; };
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) {
                double value = 1.0;
                if (k == 2) {
                    value = X(1 - i, 1 - j);
                } else if (k == 3) {
                    const int rr = i == 0 ? 1 : 0, s = i == 2 ? 1 : 2;
                    const int c = j == 0 ? 1 : 0, d = j == 2 ? 1 : 2;
                    const double product = X(rr, d) * X(s, c);
                    value = std::fma(X(rr, c), X(s, d), -product) - std::fma(X(rr, d), X(s, c), -product);
                }
                cof[j * k + i] = (i + j) % 2 ? -value : value;
            }
        return cof;
    }
    if (r.nullity == 0) {
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) cof[c * k + rr] = r.det * r.inv[rr * k + c];
        return cof;
    }
    if (r.nullity == 1) {
        const int ni = k - 1;
        const double pre = r.parity * leading_product(r, k - 1);
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) cof[c * k + rr] = pre * (r.u[ni * k + rr] * r.v[ni * k + c]);
    }
    return cof;
}

double partial_pivot_det(int n, std::vector<double> m) {
    double det = 1.0;
    for (int s = 0; s < n; ++s) {
        int p = s;
        for (int i = s + 1; i < n; ++i)
            if (std::fabs(m[s * n + i]) > std::fabs(m[s * n + p])) p = i;
        if (m[s * n + p] == 0.0) return 0.0;
        if (p != s) {
            for (int j = 0; j < n; ++j) std::swap(m[j * n + s], m[j * n + p]);
            det = -det;
        }
        det *= m[s * n + s];
        for (int i = s + 1; i < n; ++i) {
            const double l = m[s * n + i] / m[s * n + s];
            for (int j = s + 1; j < n; ++j) m[j * n + i] -= l * m[j * n + s];
        }
    }
    return det;
}

// contractions.cpp:901-983
double second_cofactor(const Resolved& r, int r1, int r2, int c1, int c2) {
    const int k = r.k;
    if (r1 == r2 || c1 == c2) return 0.0;
    if (k < 2) return 0.0;
    const double sign = (r1 + r2 + c1 + c2) % 2 ? -1.0 : 1.0;
    if (k == 2) return sign;
    if (k == 3) return sign * r.x[(3 - c1 - c2) * k + (3 - r1 - r2)];
    if (r.nullity == 0 && r.det != 0.0) {
        const int m = k - 2;
        std::vector<double> minor(m * m);
        int mc = 0;
        for (int c = 0; c < k; ++c) {
            if (c == c1 || c == c2) continue;
            int mr = 0;
            for (int rr = 0; rr < k; ++rr) {
                if (rr == r1 || rr == r2) continue;
                minor[mc * m + mr] = r.x[c * k + rr];
                ++mr;
            }
            ++mc;
        }
        return sign * (m == 0 ? 1.0 : partial_pivot_det(m, minor));
    }
    auto U = [&](int row, int col) { return r.u[col * k + row]; };
    auto V = [&](int row, int col) { return r.v[col * k + row]; };
    if (r.nullity == 1) {
        const int ni = k - 1;
        const double pre = r.parity * leading_product(r, k - 1);
        const double rn1 = U(r1, ni), rn2 = U(r2, ni), ln1 = V(c1, ni), ln2 = V(c2, ni);
        double acc = 0.0;
        for (int s = 0; s < k - 1; ++s) {
            const double rw = U(r1, s) * rn2 - U(r2, s) * rn1;
            const double lw = V(c1, s) * ln2 - V(c2, s) * ln1;
            acc += (rw * lw) / r.sv[s];
        }
        return pre * acc;
    }
    if (r.nullity == 2) {
        const int a = k - 2, b = k - 1;
        const double pre = r.parity * leading_product(r, k - 2);
        const double rw = U(r1, a) * U(r2, b) - U(r2, a) * U(r1, b);
        const double lw = V(c1, a) * V(c2, b) - V(c2, a) * V(c1, b);
        return pre * rw * lw;
    }
    return 0.0;
}

struct SpinPair {
    Resolved res;
    std::vector<double> cof;  // valid when nullity <= 1
    double h1 = 0.0, htot = 0.0;
};

std::vector<double> overlap_block(int n, const int* occL, const int* occR, int k, const double* S) {
    std::vector<double> x(k * k);
    for (int c = 0; c < k; ++c)
        for (int r = 0; r < k; ++r) x[c * k + r] = S[occL[c] * n + occR[r]];
    return x;
}

// hamiltonian.cpp:35-163 (packed-kernel branch)
void same_spin_h(int n, int k, const int* occL, const int* occR, const double* h, const double* eri,
                 SpinPair* sp) {
    const Resolved& r = sp->res;
    sp->h1 = sp->htot = 0.0;
    if (r.nullity >= 3) return;
    double total = 0.0;
    if (r.nullity <= 1) {
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) total += h[occL[c] * n + occR[rr]] * sp->cof[c * k + rr];
    }
    sp->h1 = total;
    if (k < 2) {
        sp->htot = total;
        return;
    }
    auto cof = [&](int rr, int c) { return sp->cof[c * k + rr]; };
    if (r.nullity == 0 && k > 3) {
        const double inv_det = 1.0 / r.det;
        double two = 0.0;
        for (int c1 = 0; c1 < k - 1; ++c1)
            for (int r1 = 0; r1 < k - 1; ++r1) {
                const double c11 = cof(r1, c1);
                for (int c2 = c1 + 1; c2 < k; ++c2) {
                    const double c12 = cof(r1, c2);
                    double ps = 0.0;
                    for (int r2 = r1 + 1; r2 < k; ++r2) {
                        const double minor2 = c11 * cof(r2, c2) - c12 * cof(r2, c1);
                        ps += (eri_lookup(eri, occR[r1], occL[c1], occR[r2], occL[c2]) -
                               eri_lookup(eri, occR[r1], occL[c2], occR[r2], occL[c1])) *
                              minor2;
                    }
                    two += ps;
                }
            }
        total += two * inv_det;
    } else {
        for (int c1 = 0; c1 < k - 1; ++c1)
            for (int r1 = 0; r1 < k - 1; ++r1)
                for (int c2 = c1 + 1; c2 < k; ++c2)
                    for (int r2 = r1 + 1; r2 < k; ++r2) {
                        const double c2nd = second_cofactor(r, r1, r2, c1, c2);
                        total += (eri_lookup(eri, occR[r1], occL[c1], occR[r2], occL[c2]) -
                                  eri_lookup(eri, occR[r1], occL[c2], occR[r2], occL[c1])) *
                                 c2nd;
                    }
    }
    sp->htot = total;
}

SpinPair prepare_spin_pair(int n, int k, const int* occL, const int* occR, const double* S, double thr) {
    SpinPair sp;
    const std::vector<double> x = overlap_block(n, occL, occR, k, S);
    sp.res = resolve(k, x.data(), thr);
    if (sp.res.nullity <= 1) sp.cof = first_cofactor(sp.res);
    return sp;
}

// evaluator.cpp:95-148
double opposite_spin(int n, int ka, const int* aL, const int* aR, const SpinPair& a, int kb, const int* bL,
                     const int* bR, const SpinPair& b, const double* eri) {
    if (ka == 0 || kb == 0) return 0.0;
    if (a.res.nullity >= 2 || b.res.nullity >= 2) return 0.0;
    double acc = 0.0;
    for (int ac = 0; ac < ka; ++ac)
        for (int ar = 0; ar < ka; ++ar) {
            const double ca = a.cof[ac * ka + ar];
            for (int bc = 0; bc < kb; ++bc)
                for (int br = 0; br < kb; ++br)
                    acc += ca * b.cof[bc * kb + br] * eri_lookup(eri, bR[br], bL[bc], aR[ar], aL[ac]);
        }
    (void)n;
    return acc;
}

struct PairResult {
    double s, h;
};

// evaluator.cpp:421-466 + 354-384
PairResult full_pair(int n, int ka, const int* aL, const int* aR, int kb, const int* bL, const int* bR,
                     const double* S, const double* h, const double* eri, double thr) {
    SpinPair a = prepare_spin_pair(n, ka, aL, aR, S, thr);
    SpinPair b = prepare_spin_pair(n, kb, bL, bR, S, thr);
    if (ka > 0 && a.res.nullity < 3 && b.res.nullity == 0) same_spin_h(n, ka, aL, aR, h, eri, &a);
    if (kb > 0 && b.res.nullity < 3 && a.res.nullity == 0) same_spin_h(n, kb, bL, bR, h, eri, &b);
    PairResult out;
    out.s = a.res.det * b.res.det;
    out.h = a.htot * b.res.det + b.htot * a.res.det + opposite_spin(n, ka, aL, aR, a, kb, bL, bR, b, eri);
    return out;
}

// The ordered spin-pair cache (same_spin_cache.cpp:430-477) in flat arrays: per entry the
// resolved overlap's determinant, the same-spin energy, and the opposite-spin payload: the sparse
// projection p_q = sum_{pair(R_r, L_c) = q} A(r, c) of the first cofactors onto packed pairs, in
// first-touch order (left column outer, right row inner) without exact zeros, and its dense image
// K p over the packed pair kernel (same_spin_cache.cpp:186-284).
struct SpinCache {
    int kk = 0, np = 0;
    std::vector<double> det, htot, val, image;
    std::vector<int> nnz, idx;
    void resize(size_t entries, int k, int n_pairs) {
        kk = std::max(1, k * k);
        np = n_pairs;
        det.assign(entries, 0.0);
        htot.assign(entries, 0.0);
        nnz.assign(entries, 0);
        idx.assign(entries * kk, 0);
        val.assign(entries * kk, 0.0);
        image.assign(entries * (size_t)np, 0.0);
    }
};

void build_cache_entry(int n, int k, const int* occL, const int* occR, const double* S, const double* h,
                       const double* eri, const double* kdense, double thr, SpinCache* cache, size_t e,
                       std::vector<double>& dense, std::vector<char>& touched, std::vector<int>& order) {
    const int np = cache->np;
    SpinPair sp = prepare_spin_pair(n, k, occL, occR, S, thr);
    if (k > 0 && sp.res.nullity < 3) same_spin_h(n, k, occL, occR, h, eri, &sp);
    cache->det[e] = k > 0 ? sp.res.det : 1.0;
    cache->htot[e] = sp.htot;
    cache->nnz[e] = 0;
    if (k == 0 || sp.res.nullity >= 2) return;
    order.clear();
    for (int c = 0; c < k; ++c)
        for (int r = 0; r < k; ++r) {
            const int q = (int)pair_index(occR[r], occL[c]);
            if (!touched[q]) {
                touched[q] = 1;
                dense[q] = 0.0;
                order.push_back(q);
            }
            dense[q] += sp.cof[c * k + r];
        }
    int* ix = &cache->idx[e * cache->kk];
    double* vx = &cache->val[e * cache->kk];
    int m = 0;
    for (int q : order) {
        touched[q] = 0;
        if (dense[q] != 0.0) {
            ix[m] = q;
            vx[m++] = dense[q];
        }
    }
    cache->nnz[e] = m;
    double* img = &cache->image[e * (size_t)np];
    for (int t = 0; t < m; ++t) {
        const double* col = kdense + (size_t)ix[t] * np;
        const double v = vx[t];
        for (int row = 0; row < np; ++row) img[row] += col[row] * v;
    }
}

}  // namespace

extern "C" {

int oracle_version() { return 1; }

// Full-pivot LU restatement (Eigen semantics). inv may be null.
int oracle_full_pivot_lu(int k, const double* x, double threshold, double* det, double* inv) {
    std::vector<double> iv;
    const int rank = full_pivot_lu(k, x, threshold, det, inv ? &iv : nullptr);
    if (inv && rank == k) std::memcpy(inv, iv.data(), sizeof(double) * k * k);
    return rank;
}

void oracle_jacobi_svd(int k, const double* x, double* sv, double* u, double* v) {
    std::vector<double> s, uu, vv;
    jacobi_svd(k, x, &s, &uu, &vv);
    std::memcpy(sv, s.data(), sizeof(double) * k);
    std::memcpy(u, uu.data(), sizeof(double) * k * k);
    std::memcpy(v, vv.data(), sizeof(double) * k * k);
}

// Resolve one overlap block: out = {det, nullity, parity}; cof (k*k) = first cofactor matrix
// (zero for nullity >= 2, closed forms for k <= 3).
void oracle_resolve(int k, const double* x, double threshold, double* out, double* cof) {
    Resolved r = resolve(k, x, threshold);
    out[0] = r.det;
    out[1] = r.nullity;
    out[2] = r.parity;
    std::vector<double> c = r.nullity <= 1 ? first_cofactor(r) : std::vector<double>(k * k, 0.0);
    std::memcpy(cof, c.data(), sizeof(double) * k * k);
}

double oracle_second_cofactor(int k, const double* x, double threshold, int r1, int r2, int c1, int c2) {
    Resolved r = resolve(k, x, threshold);
    return second_cofactor(r, r1, r2, c1, c2);
}

// One same-spin determinant pair: out = {det, h1, htot, nullity}; cof = first cofactor (k*k).
void oracle_spin_pair(int n, int k, const int* occL, const int* occR, const double* S, const double* h,
                      const double* eri, double threshold, double* out, double* cof) {
    SpinPair sp = prepare_spin_pair(n, k, occL, occR, S, threshold);
    if (k > 0 && sp.res.nullity < 3) same_spin_h(n, k, occL, occR, h, eri, &sp);
    out[0] = sp.res.det;
    out[1] = sp.h1;
    out[2] = sp.htot;
    out[3] = sp.res.nullity;
    if (cof) {
        for (int i = 0; i < k * k; ++i) cof[i] = sp.res.nullity <= 1 ? sp.cof[i] : 0.0;
    }
}

// One full determinant pair: out = {S_de, H_de}.
void oracle_full_pair(int n, int ka, const int* aL, const int* aR, int kb, const int* bL, const int* bR,
                      const double* S, const double* h, const double* eri, double threshold, double* out) {
    PairResult p = full_pair(n, ka, aL, aR, kb, bL, bR, S, h, eri, threshold);
    out[0] = p.s;
    out[1] = p.h;
}

// Determinant-pair matrices for a list of determinants: Hd/Sd are n_det x n_det column-major
// (Hd[e*n_det + d] = <d|H|e>). Rows of alpha_occ/beta_occ are the determinants' occupied lists.
void oracle_determinant_matrices(int n, int n_det, int ka, const int* alpha_occ, int kb, const int* beta_occ,
                                 const double* S, const double* h, const double* eri, double threshold,
                                 int n_threads, double* Hd, double* Sd) {
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int e = 0; e < n_det; ++e)
        for (int d = 0; d <= e; ++d) {
            PairResult p = full_pair(n, ka, alpha_occ + d * ka, alpha_occ + e * ka, kb, beta_occ + d * kb,
                                     beta_occ + e * kb, S, h, eri, threshold);
            Hd[(size_t)e * n_det + d] = Hd[(size_t)d * n_det + e] = p.h;
            Sd[(size_t)e * n_det + d] = Sd[(size_t)d * n_det + e] = p.s;
        }
}

// Structure H/S: H_IJ = sum_{d,e} c_dI c_eJ H_de over all ordered determinant pairs, computed from
// unordered pairs (d <= e) and H_de = H_ed. Incidence is CSR by determinant: terms
// [off[d], off[d+1]) hold (structure, coefficient). pair_limit > 0 evaluates only the first
// pair_limit unordered pairs in column order (a bounded sample for timing); the output is then
// partial. Returns the number of unordered pairs evaluated.
long long oracle_structure_matrices(int n, int n_det, int ka, const int* alpha_occ, int kb, const int* beta_occ,
                                    const long long* off, const int* term_struct, const double* term_coef,
                                    int n_str, const double* S, const double* h, const double* eri,
                                    double threshold, int n_threads, long long pair_limit, double* Hs,
                                    double* Ss) {
    const size_t ns2 = (size_t)n_str * n_str;
    std::fill(Hs, Hs + ns2, 0.0);
    std::fill(Ss, Ss + ns2, 0.0);
    long long total = (long long)n_det * (n_det + 1) / 2;
    if (pair_limit > 0 && pair_limit < total) total = pair_limit;
    int nt = 1;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
    nt = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> accH(nt, std::vector<double>(ns2, 0.0)), accS(nt, std::vector<double>(ns2, 0.0));
    // column e holds unordered pairs (d <= e): linear index e(e+1)/2 + d
    const int chunk = 64;
    const long long n_chunks = (total + chunk - 1) / chunk;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (long long ch = 0; ch < n_chunks; ++ch) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* aH = accH[tid].data();
        double* aS = accS[tid].data();
        const long long lo = ch * chunk, hi = std::min(total, lo + chunk);
        long long e = (long long)((std::sqrt(8.0 * (double)lo + 1.0) - 1.0) / 2.0);
        while (e * (e + 1) / 2 > lo) --e;
        while ((e + 1) * (e + 2) / 2 <= lo) ++e;
        long long d = lo - e * (e + 1) / 2;
        for (long long li = lo; li < hi; ++li) {
            PairResult p = full_pair(n, ka, alpha_occ + d * ka, alpha_occ + e * ka, kb, beta_occ + d * kb,
                                     beta_occ + e * kb, S, h, eri, threshold);
            for (long long td = off[d]; td < off[d + 1]; ++td)
                for (long long te = off[e]; te < off[e + 1]; ++te) {
                    const size_t I = term_struct[td], J = term_struct[te];
                    const double w = term_coef[td] * term_coef[te];
                    aH[J * n_str + I] += w * p.h;
                    aS[J * n_str + I] += w * p.s;
                    if (d != e) {
                        aH[I * n_str + J] += w * p.h;
                        aS[I * n_str + J] += w * p.s;
                    }
                }
            if (++d > e) {
                ++e;
                d = 0;
            }
        }
    }
    for (int t = 0; t < nt; ++t)
        for (size_t i = 0; i < ns2; ++i) {
            Hs[i] += accH[t][i];
            Ss[i] += accS[t][i];
        }
    return total;
}

// Cached structure H/S in the shape of the reference's CPU hot loop: first the ordered spin-pair
// cache (one entry per (left, right) string pair, OpenMP dynamic,1 over left strings), then every
// ordered determinant pair (d, e) as S = S_a S_b, H = H_a S_b + H_b S_a + p_a . (K p_b) over the
// cached entries, accumulated into the structure matrices.  String tables: a_occ (Na x ka),
// b_occ (Nb x kb); shared != 0 when both spins use the same table (one cache serves both).
// Determinants: det_a/det_b string ids.  n_det_rows > 0 restricts the work to the determinant rows
// d < n_det_rows (and the cache to the left strings those rows use): a bounded sample for timing,
// with a partial result.  timings[0..3] = {cache seconds, cache entries, pair seconds, ordered
// determinant pairs}.
void oracle_cached_structure_matrices(int n, int ka, int Na, const int* a_occ, int kb, int Nb, const int* b_occ,
                                      int shared, int n_det, const int* det_a, const int* det_b,
                                      const long long* off, const int* term_struct, const double* term_coef,
                                      int n_str, const double* S, const double* h, const double* eri,
                                      double threshold, int n_threads, int n_det_rows, double* Hs, double* Ss,
                                      double* timings) {
    const int np = n * (n + 1) / 2;
    std::vector<double> kdense((size_t)np * np);
    for (int col = 0; col < np; ++col)
        for (int row = 0; row < np; ++row) kdense[(size_t)col * np + row] = eri[pair_index(row, col)];
    const int rows = (n_det_rows > 0 && n_det_rows < n_det) ? n_det_rows : n_det;
    // left strings whose cache rows the sampled determinant rows need
    std::vector<int> slot_a(Na, -1), slot_b(Nb, -1), left_a, left_b;
    for (int d = 0; d < rows; ++d) {
        if (slot_a[det_a[d]] < 0) {
            slot_a[det_a[d]] = (int)left_a.size();
            left_a.push_back(det_a[d]);
        }
        if (shared) {
            if (slot_a[det_b[d]] < 0) {
                slot_a[det_b[d]] = (int)left_a.size();
                left_a.push_back(det_b[d]);
            }
        } else if (slot_b[det_b[d]] < 0) {
            slot_b[det_b[d]] = (int)left_b.size();
            left_b.push_back(det_b[d]);
        }
    }
    if (n_threads > 0) {
#ifdef _OPENMP
        omp_set_num_threads(n_threads);
#endif
    }
    SpinCache cache_a, cache_b;
    cache_a.resize(left_a.size() * (size_t)Na, ka, np);
    cache_b.resize(left_b.size() * (size_t)Nb, kb, np);
    const auto t0 = std::chrono::steady_clock::now();
    auto fill = [&](const std::vector<int>& left, int N, int k, const int* occ, SpinCache& cache) {
#ifdef _OPENMP
#pragma omp parallel
#endif
        {
            std::vector<double> dense(np, 0.0);
            std::vector<char> touched(np, 0);
            std::vector<int> order;
            order.reserve(std::max(1, k * k));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (long long li = 0; li < (long long)left.size(); ++li)
                for (int v = 0; v < N; ++v)
                    build_cache_entry(n, k, occ + (size_t)left[li] * k, occ + (size_t)v * k, S, h, eri, kdense.data(),
                                      threshold, &cache, (size_t)li * N + v, dense, touched, order);
        }
    };
    fill(left_a, Na, ka, a_occ, cache_a);
    if (!shared) fill(left_b, Nb, kb, b_occ, cache_b);
    const auto t1 = std::chrono::steady_clock::now();
    const size_t ns2 = (size_t)n_str * n_str;
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> accH(nt, std::vector<double>(ns2, 0.0)), accS(nt, std::vector<double>(ns2, 0.0));
    const std::vector<int>& sb = shared ? slot_a : slot_b;
    const SpinCache& cb = shared ? cache_a : cache_b;
    const int Nbb = shared ? Na : Nb;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int d = 0; d < rows; ++d) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* aH = accH[tid].data();
        double* aS = accS[tid].data();
        const size_t rowa = (size_t)slot_a[det_a[d]] * Na;
        const size_t rowb = (size_t)sb[det_b[d]] * Nbb;
        for (int e = 0; e < n_det; ++e) {
            const size_t ea = rowa + det_a[e], eb = rowb + det_b[e];
            const double s_de = cache_a.det[ea] * cb.det[eb];
            double h_de = cache_a.htot[ea] * cb.det[eb] + cb.htot[eb] * cache_a.det[ea];
            const int m = cache_a.nnz[ea];
            if (m > 0 && cb.nnz[eb] > 0) {
                const int* ix = &cache_a.idx[ea * cache_a.kk];
                const double* vx = &cache_a.val[ea * cache_a.kk];
                const double* img = &cb.image[eb * (size_t)cb.np];
                double opp = 0.0;
                for (int t = 0; t < m; ++t) opp += vx[t] * img[ix[t]];
                h_de += opp;
            }
            for (long long td = off[d]; td < off[d + 1]; ++td)
                for (long long te = off[e]; te < off[e + 1]; ++te) {
                    const size_t I = term_struct[td], J = term_struct[te];
                    const double w = term_coef[td] * term_coef[te];
                    aH[J * n_str + I] += w * h_de;
                    aS[J * n_str + I] += w * s_de;
                }
        }
    }
    const auto t2 = std::chrono::steady_clock::now();
    std::fill(Hs, Hs + ns2, 0.0);
    std::fill(Ss, Ss + ns2, 0.0);
    for (int t = 0; t < nt; ++t)
        for (size_t i = 0; i < ns2; ++i) {
            Hs[i] += accH[t][i];
            Ss[i] += accS[t][i];
        }
    timings[0] = std::chrono::duration<double>(t1 - t0).count();
    timings[1] = (double)(cache_a.det.size() + cache_b.det.size());
    timings[2] = std::chrono::duration<double>(t2 - t1).count();
    timings[3] = (double)rows * n_det;
}

// RI transform: B packed [n_aux x n_bf(n_bf+1)/2] column-major (row = aux function, column = AO
// pair hi(hi+1)/2+lo), C [n_bf x n_act] column-major. L [n_aux x P] with P = n_act(n_act+1)/2,
// L[Q, pair(a,b)] = sum_{mu,nu} C(mu,a) B_Q(mu,nu) C(nu,b) (ri_transform.cpp:10-37, ri.cpp:33-96);
// K packed P(P+1)/2 with K[pair(p,q)] = sum_Q L[Q,p] L[Q,q] (ri.cpp:13-31).
void oracle_ri_transform(int n_aux, int n_bf, int n_act, const double* B, const double* C, int n_threads,
                         double* L, double* K) {
    const long long npair_ao = (long long)n_bf * (n_bf + 1) / 2;
    const int P = n_act * (n_act + 1) / 2;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (int q = 0; q < n_aux; ++q) {
        std::vector<double> T((size_t)n_bf * n_act, 0.0);  // T[mu, a] = sum_nu B_q(mu,nu) C(nu,a)
        for (int mu = 0; mu < n_bf; ++mu)
            for (int nu = 0; nu < n_bf; ++nu) {
                const double b = B[(size_t)pair_index(mu, nu) * n_aux + q];
                for (int a = 0; a < n_act; ++a) T[(size_t)a * n_bf + mu] += b * C[(size_t)a * n_bf + nu];
            }
        for (int a = 0; a < n_act; ++a)
            for (int b = 0; b <= a; ++b) {
                double acc = 0.0;
                for (int mu = 0; mu < n_bf; ++mu) acc += C[(size_t)a * n_bf + mu] * T[(size_t)b * n_bf + mu];
                L[(size_t)pair_index(a, b) * n_aux + q] = acc;
            }
    }
    (void)npair_ao;
    for (int p = 0; p < P; ++p)
        for (int q = 0; q <= p; ++q) {
            double acc = 0.0;
            for (int a = 0; a < n_aux; ++a) acc += L[(size_t)p * n_aux + a] * L[(size_t)q * n_aux + a];
            K[pair_index(p, q)] = acc;
        }
}

}  // extern "C"
