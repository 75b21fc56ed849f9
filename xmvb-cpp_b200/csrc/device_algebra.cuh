// Exact-semantics determinant-pair algebra for the device (runtime k <= KM, local arrays sized by
// the compile-time bound KM: 16 by default, 8 for kernels instantiated for k <= 8).
//
// This is the path every block takes when the register-resident fast path cannot certify
// that the reference's rank decision would be "full rank": it follows
// src/vbscf/determinants/algebra/overlap.cpp:50-109 (complete-pivoting LU whose rank counts
// pivots |u_ii| > threshold * max pivot, then an SVD for rank-deficient blocks with nullity =
// #{sigma < threshold}), src/vbscf/determinants/pairs/contractions.cpp:172-237 (first
// cofactors, with the closed forms for k <= 3) and :901-983 (second cofactors), and
// src/vbscf/determinants/algebra/hamiltonian.cpp:35-163 (same-spin Hamiltonian).
// Complete pivoting takes the first strict maximum in column-major order.  The SVD is a
// two-sided cyclic Jacobi iteration (bounded sweep count) with singular values sorted in
// decreasing order; every quantity consumed downstream is invariant to the SVD's sign and
// degenerate-subspace choices.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace vbcore {
namespace dev {

constexpr int KMAX = 16;

__host__ __device__ __forceinline__ int pair_index(int a, int b) {
    const int hi = a > b ? a : b;
    const int lo = a > b ? b : a;
    return hi * (hi + 1) / 2 + lo;
}

// index of an unordered pair of distinct orbitals a < b
__host__ __device__ __forceinline__ int anti_index(int a, int b) { return b * (b - 1) / 2 + a; }

__device__ __forceinline__ double eri_packed(const double* eri, int p, int q, int r, int s) {
    const int pq = pair_index(p, q), rs = pair_index(r, s);
    const long long hi = pq > rs ? pq : rs, lo = pq > rs ? rs : pq;
    return __ldg(eri + hi * (hi + 1) / 2 + lo);
}

// Complete-pivoting LU; returns the rank, writes det and (if rank == k and inv != nullptr) the inverse.
template <int KM = KMAX>
__device__ inline int full_pivot_lu(int k, const double* x, double threshold, double* det, double* inv) {
    double lu[KM * KM];
    int rowt[KM], colt[KM];
    for (int i = 0; i < k * k; ++i) lu[i] = x[i];
    int ntrans = 0, nonzero = k;
    double maxpivot = 0.0;
    for (int s = 0; s < k; ++s) {
        double best = -1.0;
        int br = s, bc = s;
        for (int j = s; j < k; ++j)
            for (int i = s; i < k; ++i) {
                const double v = fabs(lu[j * k + i]);
                if (v > best) {
                    best = v;
                    br = i;
                    bc = j;
                }
            }
        if (best == 0.0) {
            nonzero = s;
            for (int t = s; t < k; ++t) rowt[t] = colt[t] = t;
            break;
        }
        if (best > maxpivot) maxpivot = best;
        rowt[s] = br;
        colt[s] = bc;
        if (br != s) {
            for (int j = 0; j < k; ++j) {
                const double t = lu[j * k + s];
                lu[j * k + s] = lu[j * k + br];
                lu[j * k + br] = t;
            }
            ++ntrans;
        }
        if (bc != s) {
            for (int i = 0; i < k; ++i) {
                const double t = lu[s * k + i];
                lu[s * k + i] = lu[bc * k + i];
                lu[bc * k + i] = t;
            }
            ++ntrans;
        }
        const double piv = lu[s * k + s];
        for (int i = s + 1; i < k; ++i) lu[s * k + i] /= piv;
        for (int j = s + 1; j < k; ++j)
            for (int i = s + 1; i < k; ++i) lu[j * k + i] -= lu[s * k + i] * lu[j * k + s];
    }
    int rank = 0;
    const double cut = maxpivot * threshold;
    for (int i = 0; i < nonzero; ++i)
        if (fabs(lu[i * k + i]) > cut) ++rank;
    double d = (ntrans & 1) ? -1.0 : 1.0;
    for (int i = 0; i < k; ++i) d *= lu[i * k + i];
    *det = d;
    if (inv != nullptr && rank == k) {
        double c[KM];
        for (int col = 0; col < k; ++col) {
            for (int i = 0; i < k; ++i) c[i] = (i == col) ? 1.0 : 0.0;
            for (int s = 0; s < k; ++s) {
                const double t = c[s];
                c[s] = c[rowt[s]];
                c[rowt[s]] = t;
            }
            for (int i = 0; i < k; ++i)
                for (int j = 0; j < i; ++j) c[i] -= lu[j * k + i] * c[j];
            for (int i = k - 1; i >= 0; --i) {
                for (int j = i + 1; j < k; ++j) c[i] -= lu[j * k + i] * c[j];
                c[i] /= lu[i * k + i];
            }
            for (int s = k - 1; s >= 0; --s) {
                const double t = c[s];
                c[s] = c[colt[s]];
                c[colt[s]] = t;
            }
            for (int i = 0; i < k; ++i) inv[col * k + i] = c[i];
        }
    }
    return rank;
}

// Two-sided cyclic Jacobi SVD: x = u diag(sv) v^T, sv descending.
template <int KM = KMAX>
__device__ inline void jacobi_svd(int k, const double* x, double* sv, double* u, double* v) {
    double a[KM * KM];
    double scale = 0.0;
    for (int i = 0; i < k * k; ++i) scale = fmax(scale, fabs(x[i]));
    if (scale == 0.0) scale = 1.0;
    for (int i = 0; i < k * k; ++i) {
        a[i] = x[i] / scale;
        u[i] = 0.0;
        v[i] = 0.0;
    }
    for (int i = 0; i < k; ++i) u[i * k + i] = v[i * k + i] = 1.0;
    const double eps2 = 2.0 * 2.220446049250313e-16;
    const double tiny = 2.2250738585072014e-308;
    double maxdiag = 0.0;
    for (int i = 0; i < k; ++i) maxdiag = fmax(maxdiag, fabs(a[i * k + i]));
    for (int sweep = 0; sweep < 64; ++sweep) {
        bool done = true;
        for (int p = 1; p < k; ++p)
            for (int q = 0; q < p; ++q) {
                const double thr = fmax(tiny, eps2 * maxdiag);
                if (!(fabs(a[q * k + p]) > thr || fabs(a[p * k + q]) > thr)) continue;
                done = false;
                const double m00 = a[q * k + q], m01 = a[p * k + q], m10 = a[q * k + p], m11 = a[p * k + p];
                const double t = m00 + m11, d = m10 - m01;
                double c1 = 1.0, s1 = 0.0;
                if (fabs(d) >= tiny) {
                    const double uu = t / d;
                    const double tmp = sqrt(1.0 + uu * uu);
                    s1 = (uu >= 0 ? 1.0 : -1.0) / tmp;
                    c1 = fabs(uu) / tmp;
                }
                const double b00 = c1 * m00 + s1 * m10;
                const double b01 = c1 * m01 + s1 * m11;
                const double b11 = -s1 * m01 + c1 * m11;
                double c2 = 1.0, s2 = 0.0;
                if (b01 != 0.0) {
                    const double tau = (b11 - b00) / (2.0 * b01);
                    const double tt = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                    c2 = 1.0 / sqrt(1.0 + tt * tt);
                    s2 = tt * c2;
                }
                const double l00 = c2 * c1 + s2 * s1, l01 = c2 * s1 - s2 * c1;
                const double l10 = s2 * c1 - c2 * s1, l11 = s2 * s1 + c2 * c1;
                for (int j = 0; j < k; ++j) {
                    const double aq = a[j * k + q], ap = a[j * k + p];
                    a[j * k + q] = l00 * aq + l01 * ap;
                    a[j * k + p] = l10 * aq + l11 * ap;
                }
                for (int i = 0; i < k; ++i) {
                    const double aq = a[q * k + i], ap = a[p * k + i];
                    a[q * k + i] = c2 * aq - s2 * ap;
                    a[p * k + i] = s2 * aq + c2 * ap;
                }
                for (int i = 0; i < k; ++i) {
                    const double u0 = u[q * k + i], u1 = u[p * k + i];
                    u[q * k + i] = l00 * u0 + l01 * u1;
                    u[p * k + i] = l10 * u0 + l11 * u1;
                    const double v0 = v[q * k + i], v1 = v[p * k + i];
                    v[q * k + i] = c2 * v0 - s2 * v1;
                    v[p * k + i] = s2 * v0 + c2 * v1;
                }
                maxdiag = fmax(maxdiag, fmax(fabs(a[p * k + p]), fabs(a[q * k + q])));
            }
        if (done) break;
    }
    for (int i = 0; i < k; ++i) {
        const double di = a[i * k + i];
        sv[i] = fabs(di) * scale;
        if (di < 0)
            for (int r = 0; r < k; ++r) u[i * k + r] = -u[i * k + r];
    }
    // stable insertion sort by decreasing singular value, permuting columns of u and v
    for (int i = 1; i < k; ++i) {
        int j = i;
        while (j > 0 && sv[j] > sv[j - 1]) {
            const double ts = sv[j];
            sv[j] = sv[j - 1];
            sv[j - 1] = ts;
            for (int r = 0; r < k; ++r) {
                double tu = u[j * k + r];
                u[j * k + r] = u[(j - 1) * k + r];
                u[(j - 1) * k + r] = tu;
                double tv = v[j * k + r];
                v[j * k + r] = v[(j - 1) * k + r];
                v[(j - 1) * k + r] = tv;
            }
            --j;
        }
    }
}

template <int KM = KMAX>
__device__ inline double orthogonal_det_sign(int k, const double* q) {
    double det = 0.0;
    full_pivot_lu<KM>(k, q, 1e-300, &det, nullptr);
    return det >= 0.0 ? 1.0 : -1.0;
}

// Resolution of one overlap block with the reference's semantics.
template <int KM>
struct ResolutionT {
    int k;
    double det;
    int nullity;
    double parity;
    bool have_svd;
    double x[KM * KM];
    double inv[KM * KM];
    double sv[KM];
    double u[KM * KM];
    double v[KM * KM];
};

using Resolution = ResolutionT<KMAX>;

template <int KM>
__device__ inline void resolve_exact(int k, const double* x, double threshold, ResolutionT<KM>* r) {
    r->k = k;
    r->parity = 1.0;
    r->have_svd = false;
    for (int i = 0; i < k * k; ++i) r->x[i] = x[i];
    if (k == 0) {
        r->det = 1.0;
        r->nullity = 0;
        return;
    }
    double det = 0.0;
    const int rank = full_pivot_lu<KM>(k, x, threshold, &det, r->inv);
    if (rank == k) {
        r->nullity = 0;
        r->det = det;
        return;
    }
    jacobi_svd<KM>(k, x, r->sv, r->u, r->v);
    r->have_svd = true;
    int nullity = 0;
    for (int i = 0; i < k; ++i)
        if (r->sv[i] < threshold) ++nullity;
    r->nullity = nullity;
    r->parity = orthogonal_det_sign<KM>(k, r->u) * orthogonal_det_sign<KM>(k, r->v);
    if (nullity == 0) {
        double prod = 1.0;
        for (int i = 0; i < k; ++i) prod *= r->sv[i];
        r->det = r->parity * prod;
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) {
                double acc = 0.0;
                for (int t = 0; t < k; ++t) acc += r->v[t * k + rr] * (1.0 / r->sv[t]) * r->u[t * k + c];
                r->inv[c * k + rr] = acc;
            }
    } else {
        r->det = 0.0;
    }
}

template <int KM>
__device__ inline double leading_product(const ResolutionT<KM>& r, int count) {
    double p = 1.0;
    for (int i = 0; i < count; ++i) p *= r.sv[i];
    return p;
}

// First-order cofactor matrix (column-major, rows = right); zero for nullity >= 2.
template <int KM>
__device__ inline void first_cofactor(const ResolutionT<KM>& r, double* cof) {
    const int k = r.k;
    for (int i = 0; i < k * k; ++i) cof[i] = 0.0;
    if (k == 0) return;
    if (k <= 3) {
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) {
                double value = 1.0;
                if (k == 2) {
                    value = r.x[(1 - j) * k + (1 - i)];
                } else if (k == 3) {
                    const int rr = i == 0 ? 1 : 0, s = i == 2 ? 1 : 2;
                    const int c = j == 0 ? 1 : 0, d = j == 2 ? 1 : 2;
                    const double product = r.x[d * k + rr] * r.x[c * k + s];
                    value = fma(r.x[c * k + rr], r.x[d * k + s], -product) - fma(r.x[d * k + rr], r.x[c * k + s], -product);
                }
                cof[j * k + i] = ((i + j) & 1) ? -value : value;
            }
        return;
    }
    if (r.nullity == 0) {
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) cof[c * k + rr] = r.det * r.inv[rr * k + c];
        return;
    }
    if (r.nullity == 1) {
        const int ni = k - 1;
        const double pre = r.parity * leading_product(r, k - 1);
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) cof[c * k + rr] = pre * (r.u[ni * k + rr] * r.v[ni * k + c]);
    }
}

__device__ inline double minor_det(int m, double* a) {
    // partial-pivot determinant of an m x m column-major matrix (destroys a)
    double det = 1.0;
    for (int s = 0; s < m; ++s) {
        int p = s;
        for (int i = s + 1; i < m; ++i)
            if (fabs(a[s * m + i]) > fabs(a[s * m + p])) p = i;
        if (a[s * m + p] == 0.0) return 0.0;
        if (p != s) {
            for (int j = 0; j < m; ++j) {
                const double t = a[j * m + s];
                a[j * m + s] = a[j * m + p];
                a[j * m + p] = t;
            }
            det = -det;
        }
        det *= a[s * m + s];
        for (int i = s + 1; i < m; ++i) {
            const double l = a[s * m + i] / a[s * m + s];
            for (int j = s + 1; j < m; ++j) a[j * m + i] -= l * a[j * m + s];
        }
    }
    return det;
}

template <int KM>
__device__ inline double second_cofactor(const ResolutionT<KM>& r, int r1, int r2, int c1, int c2) {
    const int k = r.k;
    if (r1 == r2 || c1 == c2 || k < 2) return 0.0;
    const double sign = ((r1 + r2 + c1 + c2) & 1) ? -1.0 : 1.0;
    if (k == 2) return sign;
    if (k == 3) return sign * r.x[(3 - c1 - c2) * k + (3 - r1 - r2)];
    if (r.nullity == 0 && r.det != 0.0) {
        const int m = k - 2;
        double minor[KM * KM];
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
        return sign * (m == 0 ? 1.0 : minor_det(m, minor));
    }
    if (!r.have_svd) return 0.0;
    if (r.nullity == 1) {
        const int ni = k - 1;
        const double pre = r.parity * leading_product(r, k - 1);
        const double rn1 = r.u[ni * k + r1], rn2 = r.u[ni * k + r2];
        const double ln1 = r.v[ni * k + c1], ln2 = r.v[ni * k + c2];
        double acc = 0.0;
        for (int s = 0; s < k - 1; ++s) {
            const double rw = r.u[s * k + r1] * rn2 - r.u[s * k + r2] * rn1;
            const double lw = r.v[s * k + c1] * ln2 - r.v[s * k + c2] * ln1;
            acc += (rw * lw) / r.sv[s];
        }
        return pre * acc;
    }
    if (r.nullity == 2) {
        const int a = k - 2, b = k - 1;
        const double pre = r.parity * leading_product(r, k - 2);
        const double rw = r.u[a * k + r1] * r.u[b * k + r2] - r.u[a * k + r2] * r.u[b * k + r1];
        const double lw = r.v[a * k + c1] * r.v[b * k + c2] - r.v[a * k + c2] * r.v[b * k + c1];
        return pre * rw * lw;
    }
    return 0.0;
}

// Same-spin Hamiltonian with the reference's branch structure; h is n x n (symmetric),
// eri is packed.  Returns total and writes the one-electron part.
template <int KM>
__device__ inline double same_spin_exact(int n, int k, const int* occL, const int* occR, const ResolutionT<KM>& r,
                                         const double* cof, const double* h, const double* eri, double* h1_out) {
    *h1_out = 0.0;
    if (r.nullity >= 3) return 0.0;
    double total = 0.0;
    if (r.nullity <= 1) {
        for (int c = 0; c < k; ++c)
            for (int rr = 0; rr < k; ++rr) total += __ldg(h + occL[c] * n + occR[rr]) * cof[c * k + rr];
    }
    *h1_out = total;
    if (k < 2) return total;
    if (r.nullity == 0 && k > 3) {
        const double inv_det = 1.0 / r.det;
        double two = 0.0;
        for (int c1 = 0; c1 < k - 1; ++c1)
            for (int r1 = 0; r1 < k - 1; ++r1) {
                const double c11 = cof[c1 * k + r1];
                for (int c2 = c1 + 1; c2 < k; ++c2) {
                    const double c12 = cof[c2 * k + r1];
                    double ps = 0.0;
                    for (int r2 = r1 + 1; r2 < k; ++r2) {
                        const double minor2 = c11 * cof[c2 * k + r2] - c12 * cof[c1 * k + r2];
                        ps += (eri_packed(eri, occR[r1], occL[c1], occR[r2], occL[c2]) -
                               eri_packed(eri, occR[r1], occL[c2], occR[r2], occL[c1])) *
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
                        total += (eri_packed(eri, occR[r1], occL[c1], occR[r2], occL[c2]) -
                                  eri_packed(eri, occR[r1], occL[c2], occR[r2], occL[c1])) *
                                 c2nd;
                    }
    }
    return total;
}

}  // namespace dev
}  // namespace vbcore
