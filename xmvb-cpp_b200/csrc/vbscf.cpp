// VBSCF energy, orbital gradient and the quasi-Newton orbital optimization (host driver).
//
// The counterpart of xmvb::cuda::solve_scf (src/cuda/vb/scf.hpp:41-46) with the P-LBFGS
// backend (run_plbfgs_backend, src/vbscf/optimization/backends/plbfgs.cpp:19-228) instead of
// CIAH.  Per energy+gradient evaluation (every optimizer trial point):
//   host:   S_act = C^T S_ao C, h_act = C^T h_ao C
//   device: (pq|rs) through the RI transform of the AO pair Cholesky vectors (an exact
//           factorization of (mu nu|la si) to 1e-15 of its largest diagonal, computed once per
//           problem), structure H/S (vb_hs_plan_execute), lowest root (dense solver or Davidson),
//           gradient with respect to S_act, h_act and the pair factors (vb_hs_plan_gradient),
//           and the transform adjoint to the coefficients (vb_active_transform_ri_adjoint)
//   host:   the one-electron chain rule, restricted to each orbital's allowed basis functions
//           (the HAO fragment pattern of the deck).
// Energy = lowest root + nuclear repulsion (src/vbscf/workflow/evaluator.cpp:103-108; no
// inactive orbitals, so the one-electron reference energy is zero).
//
// AO integrals are closed-form s-type contracted Gaussians (overlap, kinetic, nuclear
// attraction and repulsion through the Boys function F0), which covers hydrogen 6-31G; the
// reference takes them from libcint.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace vbcore {
namespace {

constexpr double kPi = 3.14159265358979323846;

double boys0(double t) {
    if (t < 1.0e-8) return 1.0 - t / 3.0 + t * t / 10.0;
    const double s = std::sqrt(t);
    return 0.5 * std::sqrt(kPi / t) * std::erf(s);
}

struct Basis {
    int n_bf = 0;
    std::vector<int> atom;                      // per basis function
    std::vector<std::vector<double>> exps, cs;  // normalized contraction coefficients
};

double dist2(const double* a, const double* b) {
    const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return dx * dx + dy * dy + dz * dz;
}

Basis make_basis(int n_shells, const int32_t* shell_atom, const int32_t* shell_nprim, const double* exps, const double* coefs) {
    Basis b;
    b.n_bf = n_shells;
    int off = 0;
    for (int s = 0; s < n_shells; ++s) {
        std::vector<double> e(exps + off, exps + off + shell_nprim[s]);
        std::vector<double> c(coefs + off, coefs + off + shell_nprim[s]);
        off += shell_nprim[s];
        // primitive normalization (2a/pi)^(3/4), then unit self-overlap of the contraction
        for (size_t i = 0; i < e.size(); ++i) c[i] *= std::pow(2.0 * e[i] / kPi, 0.75);
        double norm = 0.0;
        for (size_t i = 0; i < e.size(); ++i)
            for (size_t j = 0; j < e.size(); ++j) norm += c[i] * c[j] * std::pow(kPi / (e[i] + e[j]), 1.5);
        for (double& v : c) v /= std::sqrt(norm);
        b.atom.push_back(shell_atom[s]);
        b.exps.push_back(e);
        b.cs.push_back(c);
    }
    return b;
}

struct AoIntegrals {
    std::vector<double> S, H;  // n x n column-major
    std::vector<double> eri;   // full n^4, (mu nu|la si) at mu + n (nu + n (la + n si))
    double enuc = 0.0;
};

AoIntegrals ao_integrals(const Basis& b, int n_atoms, const double* Z, const double* xyz) {
    const int n = b.n_bf;
    AoIntegrals ao;
    ao.S.assign((size_t)n * n, 0.0);
    ao.H.assign((size_t)n * n, 0.0);
    ao.eri.assign((size_t)n * n * n * n, 0.0);
    for (int i = 0; i < n_atoms; ++i)
        for (int j = i + 1; j < n_atoms; ++j) ao.enuc += Z[i] * Z[j] / std::sqrt(dist2(xyz + 3 * i, xyz + 3 * j));
    for (int m = 0; m < n; ++m)
        for (int v = 0; v <= m; ++v) {
            const double* A = xyz + 3 * b.atom[m];
            const double* B = xyz + 3 * b.atom[v];
            const double ab2 = dist2(A, B);
            double s = 0.0, t = 0.0, pot = 0.0;
            for (size_t i = 0; i < b.exps[m].size(); ++i)
                for (size_t j = 0; j < b.exps[v].size(); ++j) {
                    const double a = b.exps[m][i], bb = b.exps[v][j], p = a + bb, mu = a * bb / p;
                    const double cc = b.cs[m][i] * b.cs[v][j];
                    const double sij = std::pow(kPi / p, 1.5) * std::exp(-mu * ab2);
                    s += cc * sij;
                    t += cc * mu * (3.0 - 2.0 * mu * ab2) * sij;
                    double P[3];
                    for (int k = 0; k < 3; ++k) P[k] = (a * A[k] + bb * B[k]) / p;
                    for (int c = 0; c < n_atoms; ++c)
                        pot -= cc * Z[c] * 2.0 * kPi / p * std::exp(-mu * ab2) * boys0(p * dist2(P, xyz + 3 * c));
                }
            ao.S[m + (size_t)v * n] = ao.S[v + (size_t)m * n] = s;
            ao.H[m + (size_t)v * n] = ao.H[v + (size_t)m * n] = t + pot;
        }
    auto idx = [n](int a, int bq, int c, int d) { return (size_t)a + (size_t)n * (bq + (size_t)n * (c + (size_t)n * d)); };
    for (int m = 0; m < n; ++m)
        for (int v = 0; v <= m; ++v)
            for (int l = 0; l < n; ++l)
                for (int sg = 0; sg <= l; ++sg) {
                    if (m * (m + 1) / 2 + v < l * (l + 1) / 2 + sg) continue;
                    const double* A = xyz + 3 * b.atom[m];
                    const double* B = xyz + 3 * b.atom[v];
                    const double* C = xyz + 3 * b.atom[l];
                    const double* D = xyz + 3 * b.atom[sg];
                    double val = 0.0;
                    for (size_t i = 0; i < b.exps[m].size(); ++i)
                        for (size_t j = 0; j < b.exps[v].size(); ++j) {
                            const double a = b.exps[m][i], bb = b.exps[v][j], p = a + bb;
                            const double cab = b.cs[m][i] * b.cs[v][j] * std::exp(-a * bb / p * dist2(A, B));
                            double P[3];
                            for (int k = 0; k < 3; ++k) P[k] = (a * A[k] + bb * B[k]) / p;
                            for (size_t k2 = 0; k2 < b.exps[l].size(); ++k2)
                                for (size_t l2 = 0; l2 < b.exps[sg].size(); ++l2) {
                                    const double c = b.exps[l][k2], d = b.exps[sg][l2], q = c + d;
                                    const double ccd = b.cs[l][k2] * b.cs[sg][l2] * std::exp(-c * d / q * dist2(C, D));
                                    double Q[3];
                                    for (int k = 0; k < 3; ++k) Q[k] = (c * C[k] + d * D[k]) / q;
                                    const double pre = 2.0 * std::pow(kPi, 2.5) / (p * q * std::sqrt(p + q));
                                    val += cab * ccd * pre * boys0(p * q / (p + q) * dist2(P, Q));
                                }
                        }
                    const int I[8][4] = {{m, v, l, sg}, {v, m, l, sg}, {m, v, sg, l}, {v, m, sg, l},
                                         {l, sg, m, v}, {sg, l, m, v}, {l, sg, v, m}, {sg, l, v, m}};
                    for (auto& t4 : I) ao.eri[idx(t4[0], t4[1], t4[2], t4[3])] = val;
                }
    return ao;
}

int pidx(int a, int b) { return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; }

// structure spaces up to this size take the dense all-root solver, larger ones the
// lowest-root Davidson iteration
constexpr int kDenseStructureLimit = 200;

struct Active {
    std::vector<double> S, h, eri;  // eri packed
    std::vector<double> T3;         // (kappa x|y z): kappa + nbf (x + na (y + na z))
};

Active transform(const AoIntegrals& ao, int nbf, int na, const std::vector<double>& C) {
    Active r;
    std::vector<double> SC((size_t)nbf * na, 0.0), HC((size_t)nbf * na, 0.0);
    for (int a = 0; a < na; ++a)
        for (int m = 0; m < nbf; ++m) {
            double s = 0.0, hh = 0.0;
            for (int v = 0; v < nbf; ++v) {
                s += ao.S[m + (size_t)v * nbf] * C[v + (size_t)a * nbf];
                hh += ao.H[m + (size_t)v * nbf] * C[v + (size_t)a * nbf];
            }
            SC[m + (size_t)a * nbf] = s;
            HC[m + (size_t)a * nbf] = hh;
        }
    r.S.assign((size_t)na * na, 0.0);
    r.h.assign((size_t)na * na, 0.0);
    for (int a = 0; a < na; ++a)
        for (int b = 0; b < na; ++b) {
            double s = 0.0, hh = 0.0;
            for (int m = 0; m < nbf; ++m) {
                s += C[m + (size_t)a * nbf] * SC[m + (size_t)b * nbf];
                hh += C[m + (size_t)a * nbf] * HC[m + (size_t)b * nbf];
            }
            r.S[a + (size_t)b * na] = s;
            r.h[a + (size_t)b * na] = hh;
        }
    // quarter transforms: (mu nu|la si) -> (mu nu|la d) -> (mu nu|c d) -> (mu b|c d) = T3 -> (a b|c d)
    const size_t n3 = (size_t)nbf * nbf * nbf;
    std::vector<double> t1(n3 * na, 0.0);  // mu + n(nu + n(la + n d))
    for (int d = 0; d < na; ++d)
        for (int s = 0; s < nbf; ++s) {
            const double c = C[s + (size_t)d * nbf];
            if (c == 0.0) continue;
            for (size_t e = 0; e < n3; ++e) t1[e + n3 * d] += c * ao.eri[e + n3 * s];
        }
    const size_t n2 = (size_t)nbf * nbf;
    std::vector<double> t2(n2 * na * na, 0.0);  // mu + n(nu + n(c + na d))
    for (int d = 0; d < na; ++d)
        for (int c = 0; c < na; ++c)
            for (int l = 0; l < nbf; ++l) {
                const double cc = C[l + (size_t)c * nbf];
                if (cc == 0.0) continue;
                for (size_t e = 0; e < n2; ++e) t2[e + n2 * (c + (size_t)na * d)] += cc * t1[e + n2 * (l + (size_t)nbf * d)];
            }
    r.T3.assign((size_t)nbf * na * na * na, 0.0);  // kappa + n(b + na(c + na d))
    for (int cd = 0; cd < na * na; ++cd)
        for (int b = 0; b < na; ++b)
            for (int v = 0; v < nbf; ++v) {
                const double cv = C[v + (size_t)b * nbf];
                if (cv == 0.0) continue;
                for (int m = 0; m < nbf; ++m)
                    r.T3[m + (size_t)nbf * (b + (size_t)na * cd)] += cv * t2[m + (size_t)nbf * (v + (size_t)nbf * cd)];
            }
    const int P = na * (na + 1) / 2;
    r.eri.assign((size_t)P * (P + 1) / 2, 0.0);
    for (int a = 0; a < na; ++a)
        for (int b = 0; b <= a; ++b)
            for (int c = 0; c < na; ++c)
                for (int d = 0; d <= c; ++d) {
                    const int pq = pidx(a, b), rs = pidx(c, d);
                    if (pq < rs) continue;
                    double v = 0.0;
                    for (int m = 0; m < nbf; ++m)
                        v += C[m + (size_t)a * nbf] * r.T3[m + (size_t)nbf * (b + (size_t)na * (c + (size_t)na * d))];
                    r.eri[(size_t)pq * (pq + 1) / 2 + rs] = v;
                }
    return r;
}

// Pivoted Cholesky of the AO pair Coulomb matrix V[(mu nu), (la si)] = (mu nu|la si) over
// packed pairs: V = B^T B with B [rank x n_pairs] (row = Cholesky vector, column = AO pair
// hi(hi+1)/2+lo), stopping when the largest remaining diagonal falls to tol times the largest
// initial one.  The packed factor has the layout of metric-whitened RI factors, so the active
// transform, the pair-kernel factorization and the gradient run through the RI path.
template <class PairMatrix>
std::vector<double> pair_cholesky(int P, const PairMatrix& V, double tol, int* rank) {
    std::vector<double> diag(P);
    double dmax = 0.0;
    for (int p = 0; p < P; ++p) dmax = std::max(dmax, diag[p] = V(p, p));
    std::vector<std::vector<double>> rows;
    std::vector<char> used(P, 0);
    while ((int)rows.size() < P) {
        int piv = -1;
        double best = tol * dmax;
        for (int p = 0; p < P; ++p)
            if (!used[p] && diag[p] > best) {
                best = diag[p];
                piv = p;
            }
        if (piv < 0) break;
        std::vector<double> row(P);
        const double sq = std::sqrt(diag[piv]);
        for (int q = 0; q < P; ++q) {
            double v = V(piv, q);
            for (const auto& r : rows) v -= r[piv] * r[q];
            row[q] = v / sq;
        }
        for (int q = 0; q < P; ++q) diag[q] -= row[q] * row[q];
        used[piv] = 1;
        rows.push_back(std::move(row));
    }
    *rank = (int)rows.size();
    std::vector<double> B((size_t)rows.size() * P);  // column-major [rank x P]
    for (size_t c = 0; c < rows.size(); ++c)
        for (int q = 0; q < P; ++q) B[c + rows.size() * (size_t)q] = rows[c][q];
    return B;
}

std::vector<double> ao_pair_cholesky(const AoIntegrals& ao, int n, double tol, int* rank) {
    const int P = n * (n + 1) / 2;
    std::vector<int> pm(P), pn(P);
    for (int m = 0, t = 0; m < n; ++m)
        for (int v = 0; v <= m; ++v, ++t) {
            pm[t] = m;
            pn[t] = v;
        }
    auto V = [&](int p, int q) {
        return ao.eri[(size_t)pm[p] + (size_t)n * (pn[p] + (size_t)n * (pm[q] + (size_t)n * pn[q]))];
    };
    return pair_cholesky(P, V, tol, rank);
}

}  // namespace
}  // namespace vbcore

using namespace vbcore;

struct vb_scf_problem {
    vb_context* ctx = nullptr;
    Basis basis;
    AoIntegrals ao;
    std::vector<double> chol;  // AO pair Cholesky vectors, [n_chol x n_bf(n_bf+1)/2]
    int n_chol = 0;
    int n_act = 0;
    std::vector<std::vector<int>> pattern;
    std::vector<int32_t> rows;
    std::vector<uint64_t> alpha, beta;
    std::vector<int32_t> det_a, det_b, term_str;
    std::vector<int64_t> term_off;
    std::vector<double> term_coef;
    vb_hs_plan* plan = nullptr;
    int n_str = 0;
    // RI transform precision of vb_solve_scf (split until the gradient falls to precision_switch)
    int precision = VB_PRECISION_FP64;
    double precision_switch = 0.0;
    bool split_now = false;
    int split_evaluations = 0;
    ~vb_scf_problem() {
        if (plan) vb_hs_plan_destroy(plan);
    }
};

namespace {

// One energy + gradient evaluation at coefficients C (n_bf x n_act, column-major).
vb_status evaluate(vb_scf_problem* pr, const std::vector<double>& C, double* energy, std::vector<double>* grad,
                   std::vector<double>* Hs_out, std::vector<double>* Ss_out) {
    const int nbf = pr->basis.n_bf, na = pr->n_act, nc = pr->n_chol;
    const int P = na * (na + 1) / 2;
    // one-electron parts on the host (n_bf x n_act), two-electron parts through the device RI
    // transform of the AO Cholesky vectors: (pq|rs) = sum_c L[c, pq] L[c, rs]
    std::vector<double> SC((size_t)nbf * na, 0.0), HC((size_t)nbf * na, 0.0);
    for (int a = 0; a < na; ++a)
        for (int m = 0; m < nbf; ++m) {
            double sacc = 0.0, hacc = 0.0;
            for (int v = 0; v < nbf; ++v) {
                sacc += pr->ao.S[m + (size_t)v * nbf] * C[v + (size_t)a * nbf];
                hacc += pr->ao.H[m + (size_t)v * nbf] * C[v + (size_t)a * nbf];
            }
            SC[m + (size_t)a * nbf] = sacc;
            HC[m + (size_t)a * nbf] = hacc;
        }
    std::vector<double> Sact((size_t)na * na), hact((size_t)na * na);
    for (int a = 0; a < na; ++a)
        for (int b = 0; b < na; ++b) {
            double sacc = 0.0, hacc = 0.0;
            for (int m = 0; m < nbf; ++m) {
                sacc += C[m + (size_t)a * nbf] * SC[m + (size_t)b * nbf];
                hacc += C[m + (size_t)a * nbf] * HC[m + (size_t)b * nbf];
            }
            Sact[a + (size_t)b * na] = sacc;
            hact[a + (size_t)b * na] = hacc;
        }
    std::vector<double> L((size_t)nc * P), K((size_t)P * (P + 1) / 2), T((size_t)na * nc * nbf);
    vb_status st;
    if (pr->split_now) {
        st = vb_active_transform_ri_precision(pr->ctx, pr->chol.data(), nc, nbf, C.data(), na, VB_PRECISION_BF16X3,
                                              VB_MEM_HOST, grad ? T.data() : nullptr, L.data(), K.data());
        ++pr->split_evaluations;
    } else {
        st = vb_active_transform_ri(pr->ctx, pr->chol.data(), nc, nbf, C.data(), na, VB_MEM_HOST,
                                    grad ? T.data() : nullptr, L.data(), K.data());
    }
    if (st != VB_OK) return st;
    const int ns = pr->n_str;
    std::vector<double> F;  // pair factors F = L^T (P x n_chol), the gradient's RI input
    if (grad) {
        F.resize((size_t)P * nc);
        for (int c = 0; c < nc; ++c)
            for (int q = 0; q < P; ++q) F[q + (size_t)c * P] = L[c + (size_t)nc * q];
    }
    std::vector<double> gS, gh, gF;
    double root = 0.0;
    if (!Hs_out && !Ss_out) {
        // structure H/S stay on the device: root and gradient in one call
        if (grad) {
            gS.resize((size_t)na * na);
            gh.resize((size_t)na * na);
            gF.resize((size_t)P * nc);
        }
        st = vb_hs_plan_root_gradient(pr->plan, Sact.data(), hact.data(), K.data(), 1.0e-11, &root, nullptr,
                                      grad ? gS.data() : nullptr, grad ? gh.data() : nullptr,
                                      grad ? F.data() : nullptr, nc, grad ? gF.data() : nullptr);
        if (st != VB_OK) return st;
        *energy = root + pr->ao.enuc;
        if (!grad) return VB_OK;
    }
    std::vector<double> Hs, Ss;
    if (Hs_out || Ss_out) {
        Hs.resize((size_t)ns * ns);
        Ss.resize((size_t)ns * ns);
        st = vb_hs_plan_execute(pr->plan, Sact.data(), hact.data(), K.data(), VB_MEM_HOST, Hs.data(), Ss.data());
        if (st != VB_OK) return st;
        std::vector<double> w(ns), V((size_t)ns * ns);
        int info = 0;
        if (ns <= kDenseStructureLimit) {
            st = vb_generalized_eigh(pr->ctx, Hs.data(), Ss.data(), ns, VB_MEM_HOST, w.data(), V.data(), &info);
        } else {
            int its = 0;
            st = vb_lowest_root(pr->ctx, Hs.data(), Ss.data(), ns, VB_MEM_HOST, 1.0e-11, 2000, w.data(), V.data(), &its);
        }
        if (st != VB_OK) return st;
        *energy = w[0] + pr->ao.enuc;
        if (Hs_out) *Hs_out = Hs;
        if (Ss_out) *Ss_out = Ss;
        if (!grad) return VB_OK;
        // gradient with respect to S_act, h_act and the pair factors F
        gS.resize((size_t)na * na);
        gh.resize((size_t)na * na);
        gF.resize((size_t)P * nc);
        st = vb_hs_plan_gradient(pr->plan, Sact.data(), hact.data(), K.data(), VB_MEM_HOST, V.data(), w[0], gS.data(),
                                 gh.data(), nullptr, F.data(), nc, gF.data());
        if (st != VB_OK) return st;
    }
    // dE/dC = 2 S_ao C G_S + 2 h_ao C G_h + RI adjoint of dE/dL
    std::vector<double> gL((size_t)nc * P), gC((size_t)nbf * na);
    for (int c = 0; c < nc; ++c)
        for (int q = 0; q < P; ++q) gL[c + (size_t)nc * q] = gF[q + (size_t)c * P];
    st = vb_active_transform_ri_adjoint(pr->ctx, T.data(), gL.data(), nc, nbf, na, VB_MEM_HOST, gC.data());
    if (st != VB_OK) return st;
    std::vector<double>& g = *grad;
    g.assign((size_t)nbf * na, 0.0);
    for (int a = 0; a < na; ++a)
        for (int m = 0; m < nbf; ++m) {
            double acc = gC[m + (size_t)a * nbf];
            for (int b = 0; b < na; ++b)
                acc += 2.0 * (SC[m + (size_t)b * nbf] * gS[b + (size_t)a * na] + HC[m + (size_t)b * nbf] * gh[b + (size_t)a * na]);
            g[m + (size_t)a * nbf] = acc;
        }
    // parameters outside each orbital's allowed basis functions stay fixed
    for (int a = 0; a < na; ++a) {
        std::vector<char> allowed(nbf, 0);
        for (int m : pr->pattern[a]) allowed[m] = 1;
        for (int m = 0; m < nbf; ++m)
            if (!allowed[m]) g[m + (size_t)a * nbf] = 0.0;
    }
    return VB_OK;
}

}  // namespace

namespace {

// Orbital pattern, structures, expansion and the structure H/S plan of a problem (shared by both
// creation paths).  Deletes `pr` and returns the failure on error.
vb_status finish_problem(vb_context* ctx, vb_scf_problem* pr, int n_active, const int32_t* orbital_offsets,
                         const int32_t* orbital_functions, int n_electrons, int multiplicity, const char* structures,
                         const char* who) {
    pr->n_act = n_active;
    for (int a = 0; a < n_active; ++a) {
        std::vector<int> f;
        for (int t = orbital_offsets[a]; t < orbital_offsets[a + 1]; ++t) {
            if (orbital_functions[t] < 0 || orbital_functions[t] >= pr->basis.n_bf) {
                delete pr;
                return set_error(ctx, VB_ERR_INVALID, std::string(who) + ": orbital basis function out of range");
            }
            f.push_back(orbital_functions[t]);
        }
        pr->pattern.push_back(f);
    }
    int64_t ns = 0;
    vb_status st = vb_generate_structures(structures, n_active, n_electrons, multiplicity, 0, &ns, nullptr, 0);
    if (st != VB_OK) {
        delete pr;
        return set_error(ctx, st, std::string(who) + ": " + vb_last_error(nullptr));
    }
    pr->rows.resize((size_t)ns * n_electrons);
    vb_generate_structures(structures, n_active, n_electrons, multiplicity, 0, &ns, pr->rows.data(),
                           (int64_t)pr->rows.size());
    vb_expansion_sizes sz{};
    st = vb_expand_structures(pr->rows.data(), ns, n_electrons, multiplicity, 0, &sz, nullptr, nullptr, nullptr,
                              nullptr, nullptr, nullptr, nullptr);
    if (st != VB_OK) {
        delete pr;
        return set_error(ctx, st, std::string(who) + ": expansion failed");
    }
    pr->alpha.resize(sz.n_alpha_strings);
    pr->beta.resize(sz.n_beta_strings);
    pr->det_a.resize(sz.n_determinants);
    pr->det_b.resize(sz.n_determinants);
    pr->term_off.resize(sz.n_determinants + 1);
    pr->term_str.resize(sz.n_terms);
    pr->term_coef.resize(sz.n_terms);
    vb_expand_structures(pr->rows.data(), ns, n_electrons, multiplicity, 0, &sz, pr->alpha.data(), pr->beta.data(),
                         pr->det_a.data(), pr->det_b.data(), pr->term_off.data(), pr->term_str.data(),
                         pr->term_coef.data());
    vb_expansion e{n_active, sz.n_alpha_electrons, sz.n_beta_electrons, sz.n_alpha_strings, sz.n_beta_strings,
                   pr->alpha.data(), pr->beta.data(), sz.n_determinants, pr->det_a.data(), pr->det_b.data(),
                   sz.n_structures, pr->term_off.data(), pr->term_str.data(), pr->term_coef.data()};
    st = vb_hs_plan_create(ctx, &e, &pr->plan);
    if (st != VB_OK) {
        delete pr;
        return st;
    }
    pr->n_str = sz.n_structures;
    return VB_OK;
}

}  // namespace

extern "C" {

vb_status vb_scf_problem_create(vb_context* ctx, const vb_scf_input* in, vb_scf_problem** out) {
    if (!ctx || !in || !out) return VB_ERR_INVALID;
    *out = nullptr;
    if (in->n_atoms < 1 || !in->charges || !in->coords || in->n_shells < 1 || !in->shell_atom || !in->shell_nprim ||
        !in->shell_exponents || !in->shell_coefficients || in->n_active < 1 || !in->orbital_offsets ||
        !in->orbital_functions || !in->structures)
        return set_error(ctx, VB_ERR_INVALID, "vb_scf_problem_create: incomplete input");
    for (int s = 0; s < in->n_shells; ++s)
        if (in->shell_atom[s] < 0 || in->shell_atom[s] >= in->n_atoms || in->shell_nprim[s] < 1)
            return set_error(ctx, VB_ERR_INVALID, "vb_scf_problem_create: bad shell");
    auto pr = new vb_scf_problem();
    pr->ctx = ctx;
    pr->basis = make_basis(in->n_shells, in->shell_atom, in->shell_nprim, in->shell_exponents, in->shell_coefficients);
    pr->ao = ao_integrals(pr->basis, in->n_atoms, in->charges, in->coords);
    pr->chol = ao_pair_cholesky(pr->ao, pr->basis.n_bf, 1.0e-15, &pr->n_chol);
    const vb_status st = finish_problem(ctx, pr, in->n_active, in->orbital_offsets, in->orbital_functions,
                                        in->n_electrons, in->multiplicity, in->structures, "vb_scf_problem_create");
    if (st != VB_OK) return st;
    *out = pr;
    return VB_OK;
}

vb_status vb_scf_problem_create_from_integrals(vb_context* ctx, const vb_scf_integral_input* in,
                                               vb_scf_problem** out) {
    const char* who = "vb_scf_problem_create_from_integrals";
    if (!ctx || !in || !out) return VB_ERR_INVALID;
    *out = nullptr;
    const int n = in->n_basis;
    if (n < 1 || !in->S_ao || !in->h_ao || in->n_pairs < 0 || in->n_integrals < 0 ||
        (in->n_pairs > 0 && (!in->pair_first || !in->pair_second)) ||
        (in->n_integrals > 0 && (!in->integral_rows || !in->integral_columns || !in->integral_values)) ||
        in->n_active < 1 || !in->orbital_offsets || !in->orbital_functions || !in->structures)
        return set_error(ctx, VB_ERR_INVALID, std::string(who) + ": incomplete input");
    const int P = n * (n + 1) / 2;
    // AO pair graph -> packed pair index of each graph pair
    std::vector<int> packed((size_t)in->n_pairs);
    for (int64_t p = 0; p < in->n_pairs; ++p) {
        const int a = in->pair_first[p], b = in->pair_second[p];
        if (a < 0 || a >= n || b < 0 || b >= n)
            return set_error(ctx, VB_ERR_INVALID, std::string(who) + ": AO pair index out of range");
        const int hi = std::max(a, b), lo = std::min(a, b);
        packed[p] = hi * (hi + 1) / 2 + lo;
    }
    // dense pair matrix V over packed AO pairs; each unique (left, right) entry once, mirrored
    std::vector<double> V((size_t)P * P, 0.0);
    for (int64_t t = 0; t < in->n_integrals; ++t) {
        const int64_t r = in->integral_rows[t], c = in->integral_columns[t];
        if (r < 0 || r >= in->n_pairs || c < 0 || c >= in->n_pairs)
            return set_error(ctx, VB_ERR_INVALID, std::string(who) + ": integral pair index out of range");
        const size_t p = packed[r], q = packed[c];
        V[p + q * P] = in->integral_values[t];
        V[q + p * P] = in->integral_values[t];
    }
    auto pr = new vb_scf_problem();
    pr->ctx = ctx;
    pr->basis.n_bf = n;
    pr->ao.S.assign(in->S_ao, in->S_ao + (size_t)n * n);
    pr->ao.H.assign(in->h_ao, in->h_ao + (size_t)n * n);
    pr->ao.enuc = in->nuclear_repulsion;
    pr->chol = pair_cholesky(P, [&](int p, int q) { return V[(size_t)p + (size_t)q * P]; }, 1.0e-15, &pr->n_chol);
    const vb_status st = finish_problem(ctx, pr, in->n_active, in->orbital_offsets, in->orbital_functions,
                                        in->n_electrons, in->multiplicity, in->structures, who);
    if (st != VB_OK) return st;
    *out = pr;
    return VB_OK;
}

vb_status vb_ao_integrals_s(const vb_scf_input* in, double* S_ao, double* h_ao, double* eri_ao,
                            double* nuclear_repulsion) {
    if (!in || in->n_atoms < 1 || !in->charges || !in->coords || in->n_shells < 1 || !in->shell_atom ||
        !in->shell_nprim || !in->shell_exponents || !in->shell_coefficients)
        return set_error(nullptr, VB_ERR_INVALID, "vb_ao_integrals_s: incomplete input");
    for (int s = 0; s < in->n_shells; ++s)
        if (in->shell_atom[s] < 0 || in->shell_atom[s] >= in->n_atoms || in->shell_nprim[s] < 1)
            return set_error(nullptr, VB_ERR_INVALID, "vb_ao_integrals_s: bad shell");
    const Basis b = make_basis(in->n_shells, in->shell_atom, in->shell_nprim, in->shell_exponents, in->shell_coefficients);
    const AoIntegrals ao = ao_integrals(b, in->n_atoms, in->charges, in->coords);
    if (S_ao) std::copy(ao.S.begin(), ao.S.end(), S_ao);
    if (h_ao) std::copy(ao.H.begin(), ao.H.end(), h_ao);
    if (eri_ao) std::copy(ao.eri.begin(), ao.eri.end(), eri_ao);
    if (nuclear_repulsion) *nuclear_repulsion = ao.enuc;
    return VB_OK;
}

vb_status vb_scf_problem_destroy(vb_scf_problem* pr) {
    delete pr;
    return VB_OK;
}

vb_status vb_scf_problem_sizes(const vb_scf_problem* pr, int* n_basis, int* n_active, int* n_structures,
                               double* nuclear_repulsion) {
    if (!pr) return VB_ERR_INVALID;
    if (n_basis) *n_basis = pr->basis.n_bf;
    if (n_active) *n_active = pr->n_act;
    if (n_structures) *n_structures = pr->n_str;
    if (nuclear_repulsion) *nuclear_repulsion = pr->ao.enuc;
    return VB_OK;
}

vb_status vb_scf_ao_integrals(const vb_scf_problem* pr, double* S_ao, double* h_ao, double* eri_ao) {
    if (!pr) return VB_ERR_INVALID;
    if (S_ao) std::copy(pr->ao.S.begin(), pr->ao.S.end(), S_ao);
    if (h_ao) std::copy(pr->ao.H.begin(), pr->ao.H.end(), h_ao);
    if (eri_ao && !pr->ao.eri.empty()) std::copy(pr->ao.eri.begin(), pr->ao.eri.end(), eri_ao);
    if (eri_ao && pr->ao.eri.empty()) {
        // a problem built from AO pair integrals: (mu nu|la si) from its pair Cholesky vectors
        const int n = pr->basis.n_bf, nc = pr->n_chol;
        auto pk = [](int a, int b) { return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; };
        for (int m = 0; m < n; ++m)
            for (int v = 0; v < n; ++v)
                for (int l = 0; l < n; ++l)
                    for (int q = 0; q < n; ++q) {
                        const size_t p1 = pk(m, v), p2 = pk(l, q);
                        double acc = 0.0;
                        for (int c = 0; c < nc; ++c) acc += pr->chol[c + (size_t)nc * p1] * pr->chol[c + (size_t)nc * p2];
                        eri_ao[(size_t)m + (size_t)n * (v + (size_t)n * (l + (size_t)n * q))] = acc;
                    }
    }
    return VB_OK;
}

vb_status vb_scf_energy_gradient(vb_scf_problem* pr, const double* coefficients, double* energy, double* gradient,
                                 double* hamiltonian_out, double* overlap_out) {
    if (!pr || !coefficients || !energy) return VB_ERR_INVALID;
    const int nbf = pr->basis.n_bf, na = pr->n_act;
    std::vector<double> C(coefficients, coefficients + (size_t)nbf * na);
    std::vector<double> g, Hs, Ss;
    vb_status st = evaluate(pr, C, energy, gradient ? &g : nullptr, hamiltonian_out ? &Hs : nullptr,
                            overlap_out ? &Ss : nullptr);
    if (st != VB_OK) return st;
    if (gradient) std::copy(g.begin(), g.end(), gradient);
    if (hamiltonian_out) std::copy(Hs.begin(), Hs.end(), hamiltonian_out);
    if (overlap_out) std::copy(Ss.begin(), Ss.end(), overlap_out);
    return VB_OK;
}

vb_status vb_solve_scf(vb_scf_problem* pr, const double* initial_coefficients, const vb_scf_options* opt,
                       vb_scf_result* res, double* coefficients_out) {
    if (!pr || !initial_coefficients || !opt || !res) return VB_ERR_INVALID;
    const int nbf = pr->basis.n_bf, na = pr->n_act;
    // parameters: the allowed entries of C
    std::vector<size_t> where;
    for (int a = 0; a < na; ++a)
        for (int m : pr->pattern[a]) where.push_back(m + (size_t)a * nbf);
    const size_t np_ = where.size();
    std::vector<double> C((size_t)nbf * na, 0.0);
    for (size_t i : where) C[i] = initial_coefficients[i];
    auto pack = [&](const std::vector<double>& full) {
        std::vector<double> x(np_);
        for (size_t i = 0; i < np_; ++i) x[i] = full[where[i]];
        return x;
    };
    auto unpack = [&](const std::vector<double>& x) {
        std::vector<double> full((size_t)nbf * na, 0.0);
        for (size_t i = 0; i < np_; ++i) full[where[i]] = x[i];
        return full;
    };
    auto dot = [](const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0.0;
        for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
        return s;
    };
    auto inf_norm = [](const std::vector<double>& a) {
        double s = 0.0;
        for (double v : a) s = std::max(s, std::fabs(v));
        return s;
    };
    std::vector<double> x = pack(C), gfull;
    double f = 0.0;
    pr->split_evaluations = 0;
    pr->split_now = pr->precision == VB_PRECISION_BF16X3;
    struct SplitOff {  // no split evaluation outlives the solve
        vb_scf_problem* p;
        ~SplitOff() { p->split_now = false; }
    } split_off{pr};
    vb_status st = evaluate(pr, unpack(x), &f, &gfull, nullptr, nullptr);
    if (st != VB_OK) return st;
    std::vector<double> g = pack(gfull);
    int evaluations = 1;
    std::vector<std::vector<double>> S_hist, Y_hist;
    res->converged = 0;
    res->iterations = 0;
    const int history = std::max(1, opt->history_size);
    const double c1 = opt->armijo > 0.0 ? opt->armijo : 1.0e-4;
    for (int it = 0; it < opt->max_iterations; ++it) {
        if (pr->split_now && inf_norm(g) <= std::max(pr->precision_switch, opt->gradient_tolerance)) {
            // leave split precision: the same point in FP64, a fresh secant history
            pr->split_now = false;
            st = evaluate(pr, unpack(x), &f, &gfull, nullptr, nullptr);
            ++evaluations;
            if (st != VB_OK) return st;
            g = pack(gfull);
            S_hist.clear();
            Y_hist.clear();
        }
        if (!pr->split_now && inf_norm(g) <= opt->gradient_tolerance) {
            res->converged = 1;
            break;
        }
        // two-loop recursion with the scaled identity as initial inverse Hessian
        std::vector<double> q = g;
        const int k = (int)S_hist.size();
        std::vector<double> alpha(k);
        for (int i = k - 1; i >= 0; --i) {
            const double rho = 1.0 / dot(Y_hist[i], S_hist[i]);
            alpha[i] = rho * dot(S_hist[i], q);
            for (size_t j = 0; j < np_; ++j) q[j] -= alpha[i] * Y_hist[i][j];
        }
        double gamma = 1.0;
        if (k > 0) gamma = dot(S_hist[k - 1], Y_hist[k - 1]) / dot(Y_hist[k - 1], Y_hist[k - 1]);
        for (double& v : q) v *= gamma;
        for (int i = 0; i < k; ++i) {
            const double rho = 1.0 / dot(Y_hist[i], S_hist[i]);
            const double beta = rho * dot(Y_hist[i], q);
            for (size_t j = 0; j < np_; ++j) q[j] += S_hist[i][j] * (alpha[i] - beta);
        }
        std::vector<double> d(np_);
        for (size_t j = 0; j < np_; ++j) d[j] = -q[j];
        double slope = dot(g, d);
        if (!(slope < 0.0)) {
            S_hist.clear();
            Y_hist.clear();
            for (size_t j = 0; j < np_; ++j) d[j] = -g[j];
            slope = dot(g, d);
        }
        // first step without curvature information: bounded length
        double step = k == 0 ? std::min(1.0, 0.1 / std::max(inf_norm(d), 1e-300)) : 1.0;
        std::vector<double> xn(np_), gn;
        double fn = 0.0;
        bool accepted = false;
        for (int bt = 0; bt < 40; ++bt) {
            for (size_t j = 0; j < np_; ++j) xn[j] = x[j] + step * d[j];
            st = evaluate(pr, unpack(xn), &fn, &gfull, nullptr, nullptr);
            ++evaluations;
            if (st != VB_OK) return st;
            if (std::isfinite(fn) && fn <= f + c1 * step * slope) {
                accepted = true;
                break;
            }
            step *= 0.5;
        }
        res->iterations = it + 1;
        if (!accepted) break;
        gn = pack(gfull);
        std::vector<double> s(np_), y(np_);
        for (size_t j = 0; j < np_; ++j) {
            s[j] = xn[j] - x[j];
            y[j] = gn[j] - g[j];
        }
        if (dot(s, y) > 1.0e-16 * std::sqrt(dot(s, s) * dot(y, y))) {
            S_hist.push_back(s);
            Y_hist.push_back(y);
            if ((int)S_hist.size() > history) {
                S_hist.erase(S_hist.begin());
                Y_hist.erase(Y_hist.begin());
            }
        }
        x = xn;
        g = gn;
        f = fn;
    }
    if (pr->split_now) {
        // stopped while still in split precision: report the FP64 energy and gradient there
        pr->split_now = false;
        st = evaluate(pr, unpack(x), &f, &gfull, nullptr, nullptr);
        ++evaluations;
        if (st != VB_OK) return st;
        g = pack(gfull);
    }
    if (!res->converged && inf_norm(g) <= opt->gradient_tolerance) res->converged = 1;
    res->energy = f;
    res->gradient_inf = inf_norm(g);
    res->evaluations = evaluations;
    if (coefficients_out) {
        std::vector<double> full = unpack(x);
        std::copy(full.begin(), full.end(), coefficients_out);
    }
    return VB_OK;
}

vb_status vb_scf_problem_set_precision(vb_scf_problem* pr, int precision, double switch_gradient) {
    if (!pr) return VB_ERR_INVALID;
    if ((precision != VB_PRECISION_FP64 && precision != VB_PRECISION_BF16X3) || !(switch_gradient >= 0.0))
        return set_error(pr->ctx, VB_ERR_INVALID, "vb_scf_problem_set_precision: bad arguments");
    pr->precision = precision;
    pr->precision_switch = switch_gradient;
    return VB_OK;
}

vb_status vb_scf_problem_split_evaluations(const vb_scf_problem* pr, int32_t* split_evaluations) {
    if (!pr || !split_evaluations) return VB_ERR_INVALID;
    *split_evaluations = pr->split_evaluations;
    return VB_OK;
}

}  // extern "C"
