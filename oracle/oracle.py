"""CPU oracle for the VBSCF determinant-pair hot path.

TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path and the timed
CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg may import this module; the product never does.

Two parts:

* ``vb_oracle.cpp`` (loaded through ctypes) restates the FP64 determinant-pair
  algebra and the structure assembly of Tao-Xia/xmvb-cpp (file:line citations
  are in that file).
* This module restates, in plain Python, the reference's structure-class
  generation (``src/input/loading/generated_structures.cpp:131-167, 181-245,
  249-297, 335-391, 393-433, 475-603``) and the structure-to-determinant
  expansion (``src/vbscf/structures/expansion/expander.cpp:34-70, 130-192,
  287-557``), giving the same structure order, determinant order and +-1
  coefficients.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_vb.so")
_lib = None

THRESHOLD = 1.0e-12  # DeterminantOverlapResolver default (overlap.hpp:166)


def build() -> str:
    """Compile the C++ oracle (make) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        d, i, ll = ctypes.c_double, ctypes.c_int, ctypes.c_longlong
        p = ctypes.c_void_p
        _lib.oracle_full_pivot_lu.argtypes = [i, p, d, p, p]
        _lib.oracle_full_pivot_lu.restype = i
        _lib.oracle_jacobi_svd.argtypes = [i, p, p, p, p]
        _lib.oracle_resolve.argtypes = [i, p, d, p, p]
        _lib.oracle_second_cofactor.argtypes = [i, p, d, i, i, i, i]
        _lib.oracle_second_cofactor.restype = d
        _lib.oracle_spin_pair.argtypes = [i, i, p, p, p, p, p, d, p, p]
        _lib.oracle_full_pair.argtypes = [i, i, p, p, i, p, p, p, p, p, d, p]
        _lib.oracle_determinant_matrices.argtypes = [i, i, i, p, i, p, p, p, p, d, i, p, p]
        _lib.oracle_structure_matrices.argtypes = [i, i, i, p, i, p, p, p, p, i, p, p, p, d, i, ll, p, p]
        _lib.oracle_structure_matrices.restype = ll
        _lib.oracle_ri_transform.argtypes = [i, i, i, p, p, i, p, p]
        _lib.oracle_cached_structure_matrices.argtypes = [i, i, i, p, i, i, p, i, i, p, p, p, p, p, i, p, p, p, d,
                                                          i, i, p, p, p]
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ----------------------------------------------------------------------------------------------
# packed indices (src/core/pair_index.cpp:10-44)


def pair_index(a: int, b: int) -> int:
    hi, lo = (a, b) if a > b else (b, a)
    return hi * (hi + 1) // 2 + lo


def unpack_eri(packed: np.ndarray, n: int) -> np.ndarray:
    """Packed (pq|rs) storage -> full n^4 tensor."""
    g = np.empty((n, n, n, n))
    for p in range(n):
        for q in range(n):
            pq = pair_index(p, q)
            for r in range(n):
                for s in range(n):
                    g[p, q, r, s] = packed[pair_index(pq, pair_index(r, s))]
    return g


# ----------------------------------------------------------------------------------------------
# determinant-pair algebra (C++)


def full_pivot_lu(x: np.ndarray, threshold: float = THRESHOLD):
    """Return (rank, det, inverse-or-None) with Eigen FullPivLU semantics."""
    k = x.shape[0]
    xf = _f64(x.T.reshape(-1))  # column-major
    det = ctypes.c_double()
    inv = np.zeros(k * k)
    rank = lib().oracle_full_pivot_lu(k, _ptr(xf), threshold, ctypes.byref(det), _ptr(inv))
    return rank, det.value, (inv.reshape(k, k).T.copy() if rank == k else None)


def resolve(x: np.ndarray, threshold: float = THRESHOLD):
    """Return (det, nullity, parity, first-cofactor matrix)."""
    k = x.shape[0]
    xf = _f64(x.T.reshape(-1))
    out = np.zeros(3)
    cof = np.zeros(k * k)
    lib().oracle_resolve(k, _ptr(xf), threshold, _ptr(out), _ptr(cof))
    return out[0], int(out[1]), out[2], cof.reshape(k, k).T.copy()


def second_cofactor(x: np.ndarray, r1: int, r2: int, c1: int, c2: int, threshold: float = THRESHOLD) -> float:
    k = x.shape[0]
    xf = _f64(x.T.reshape(-1))
    return lib().oracle_second_cofactor(k, _ptr(xf), threshold, r1, r2, c1, c2)


def spin_pair(n, occ_left, occ_right, S, h, eri, threshold: float = THRESHOLD):
    """One same-spin pair: dict(det, h1, htot, nullity, cof (k x k, rows = right))."""
    k = len(occ_left)
    oL, oR = _i32(occ_left), _i32(occ_right)
    Sf, hf, ef = _f64(np.asarray(S).T.reshape(-1)), _f64(np.asarray(h).T.reshape(-1)), _f64(eri)
    out = np.zeros(4)
    cof = np.zeros(max(1, k * k))
    lib().oracle_spin_pair(n, k, _ptr(oL), _ptr(oR), _ptr(Sf), _ptr(hf), _ptr(ef), threshold, _ptr(out), _ptr(cof))
    return dict(det=out[0], h1=out[1], htot=out[2], nullity=int(out[3]), cof=cof[: k * k].reshape(k, k).T.copy())


def full_pair(n, alpha_left, alpha_right, beta_left, beta_right, S, h, eri, threshold: float = THRESHOLD):
    """One determinant pair <left|H|right>, <left|right>: returns (S_de, H_de)."""
    aL, aR, bL, bR = (_i32(v) for v in (alpha_left, alpha_right, beta_left, beta_right))
    Sf, hf, ef = _f64(np.asarray(S).T.reshape(-1)), _f64(np.asarray(h).T.reshape(-1)), _f64(eri)
    out = np.zeros(2)
    lib().oracle_full_pair(n, len(aL), _ptr(aL), _ptr(aR), len(bL), _ptr(bL), _ptr(bR), _ptr(Sf), _ptr(hf),
                           _ptr(ef), threshold, _ptr(out))
    return out[0], out[1]


def determinant_matrices(n, alpha_occ, beta_occ, S, h, eri, threads: int = 0, threshold: float = THRESHOLD):
    """All determinant pairs: (Hd, Sd) as n_det x n_det arrays."""
    ao, bo = _i32(alpha_occ), _i32(beta_occ)
    n_det = ao.shape[0]
    ka = ao.shape[1] if ao.ndim == 2 else 0
    kb = bo.shape[1] if bo.ndim == 2 else 0
    Sf, hf, ef = _f64(np.asarray(S).T.reshape(-1)), _f64(np.asarray(h).T.reshape(-1)), _f64(eri)
    Hd = np.zeros((n_det, n_det))
    Sd = np.zeros((n_det, n_det))
    lib().oracle_determinant_matrices(n, n_det, ka, _ptr(ao), kb, _ptr(bo), _ptr(Sf), _ptr(hf), _ptr(ef), threshold,
                                      threads, _ptr(Hd), _ptr(Sd))
    return Hd.T.copy(), Sd.T.copy()


def structure_matrices(n, expansion: "Expansion", S, h, eri, threads: int = 0, pair_limit: int = 0,
                       threshold: float = THRESHOLD):
    """Structure H and S (n_str x n_str).  pair_limit > 0 evaluates a bounded prefix of the
    unordered determinant pairs (partial result, for timing); returns (H, S, n_pairs)."""
    ao, bo = _i32(expansion.det_alpha_occ), _i32(expansion.det_beta_occ)
    n_det = ao.shape[0]
    ka = expansion.n_alpha
    kb = expansion.n_beta
    off = np.ascontiguousarray(expansion.offsets, dtype=np.int64)
    ts = _i32(expansion.term_structure)
    tc = _f64(expansion.term_coefficient)
    Sf, hf, ef = _f64(np.asarray(S).T.reshape(-1)), _f64(np.asarray(h).T.reshape(-1)), _f64(eri)
    ns = expansion.n_structures
    Hs = np.zeros((ns, ns))
    Ss = np.zeros((ns, ns))
    npairs = lib().oracle_structure_matrices(n, n_det, ka, _ptr(ao), kb, _ptr(bo), _ptr(off), _ptr(ts), _ptr(tc), ns,
                                             _ptr(Sf), _ptr(hf), _ptr(ef), threshold, threads, int(pair_limit),
                                             _ptr(Hs), _ptr(Ss))
    return Hs.T.copy(), Ss.T.copy(), int(npairs)


def cached_structure_matrices(n, expansion: "Expansion", S, h, eri, threads: int = 0, det_rows: int = 0,
                              threshold: float = THRESHOLD):
    """Structure H and S by the reference's cached CPU algorithm (ordered spin-pair cache with
    projected images, then a sparse dot per ordered determinant pair).  det_rows > 0 evaluates only
    the determinant rows d < det_rows (partial result, for timing).  Returns (H, S, timings) with
    timings = dict(cache_s, cache_entries, pairs_s, pairs)."""
    a_occ = _i32(np.array([_occ(m) for m in expansion.alpha_strings], dtype=np.int32).reshape(
        len(expansion.alpha_strings), expansion.n_alpha))
    b_occ = _i32(np.array([_occ(m) for m in expansion.beta_strings], dtype=np.int32).reshape(
        len(expansion.beta_strings), expansion.n_beta))
    shared = int(expansion.n_alpha == expansion.n_beta and list(expansion.alpha_strings) == list(expansion.beta_strings))
    da, db = _i32(expansion.det_alpha), _i32(expansion.det_beta)
    off = np.ascontiguousarray(expansion.offsets, dtype=np.int64)
    ts = _i32(expansion.term_structure)
    tc = _f64(expansion.term_coefficient)
    Sf, hf, ef = _f64(np.asarray(S).T.reshape(-1)), _f64(np.asarray(h).T.reshape(-1)), _f64(eri)
    ns = expansion.n_structures
    Hs = np.zeros((ns, ns))
    Ss = np.zeros((ns, ns))
    tm = np.zeros(4)
    lib().oracle_cached_structure_matrices(n, expansion.n_alpha, a_occ.shape[0], _ptr(a_occ), expansion.n_beta,
                                           b_occ.shape[0], _ptr(b_occ), shared, len(da), _ptr(da), _ptr(db),
                                           _ptr(off), _ptr(ts), _ptr(tc), ns, _ptr(Sf), _ptr(hf), _ptr(ef),
                                           threshold, threads, int(det_rows), _ptr(Hs), _ptr(Ss), _ptr(tm))
    return Hs.T.copy(), Ss.T.copy(), dict(cache_s=tm[0], cache_entries=int(tm[1]), pairs_s=tm[2], pairs=int(tm[3]))


def ri_transform(B_packed: np.ndarray, C: np.ndarray, threads: int = 0):
    """RI AO->active transform: B_packed [n_aux, n_bf(n_bf+1)/2], C [n_bf, n_act] ->
    (L [n_aux, P], K packed [P(P+1)/2])."""
    n_aux = B_packed.shape[0]
    n_bf, n_act = C.shape
    P = n_act * (n_act + 1) // 2
    Bf = _f64(B_packed.T)  # column-major [n_aux x npair]
    Cf = _f64(C.T)
    L = np.zeros((P, n_aux))
    K = np.zeros(P * (P + 1) // 2)
    lib().oracle_ri_transform(n_aux, n_bf, n_act, _ptr(Bf), _ptr(Cf), threads, _ptr(L), _ptr(K))
    return L.T.copy(), K


def ri_pair_factors_frame(factors, frame, mode=0, factor_direction=None, frame_direction=None):
    """RI pair factors in a new orbital frame, restating transform_ri_pair_factors and its
    directional forms (src/integrals/active/ri_transform.cpp:98-211): rows of `factors`
    [n_aux, n(n+1)/2] pack symmetric n x n factors at i(i+1)/2 + j (i >= j).  mode 0: Q^T B Q;
    mode 1: Q^T dB Q + dQ^T B Q + Q^T B dQ; mode 2 (factors already in the frame, dQ = -Q K):
    Q^T dB Q - K^T Bbar - Bbar K."""
    F = np.asarray(factors, dtype=np.float64)
    n_aux, npair = F.shape
    n = int(round((np.sqrt(8 * npair + 1) - 1) / 2))
    hi, lo = np.tril_indices(n)
    pk = np.zeros((n, n), dtype=np.int64)
    pk[hi, lo] = np.arange(npair)
    pk[lo, hi] = np.arange(npair)

    def expand(M):
        return np.asarray(M)[:, pk]  # [n_aux, n, n]

    Q = np.asarray(frame, dtype=np.float64)
    if mode == 0:
        X = np.einsum("ki,pkl,lj->pij", Q, expand(F), Q)
    elif mode == 1:
        B, dB, dQ = expand(F), expand(factor_direction), np.asarray(frame_direction)
        X = (np.einsum("ki,pkl,lj->pij", Q, dB, Q) + np.einsum("ki,pkl,lj->pij", dQ, B, Q)
             + np.einsum("ki,pkl,lj->pij", Q, B, dQ))
    else:
        Bb, dB, K = expand(F), expand(factor_direction), np.asarray(frame_direction)
        X = np.einsum("ki,pkl,lj->pij", Q, dB, Q) - np.einsum("ki,pkj->pij", K, Bb) - np.einsum("pik,kj->pij", Bb, K)
    return X[:, hi, lo]


def ri_one_index(B_packed: np.ndarray, C: np.ndarray) -> np.ndarray:
    """One-index RI factors T [(n_act n_aux), n_bf], row a*n_aux + P:
    T[(a, P), mu] = sum_nu B_P(mu, nu) C(nu, a) (transform_ri_one_index,
    src/integrals/ao/ri_transform.cpp:10-37, stored as ri_one_index_factors in
    src/integrals/active/ri.cpp:80-90)."""
    n_aux = B_packed.shape[0]
    n_bf, n_act = C.shape
    idx = np.array([[pair_index(m, v) for v in range(n_bf)] for m in range(n_bf)])
    Bfull = B_packed[:, idx]  # [n_aux, mu, nu]
    T = np.einsum("Pmn,na->aPm", Bfull, C)
    return T.reshape(n_act * n_aux, n_bf)


def ri_adjoint(T: np.ndarray, G: np.ndarray, n_act: int) -> np.ndarray:
    """dE/dC from dE/dL for L[P, pair(a,b)] = sum_{mu,nu} C(mu,a) B_P(mu,nu) C(nu,b) (the
    derivative of transform_ri_active_integrals, src/integrals/active/ri.cpp:33-96):
    dE/dC(kappa, c) = sum_{P,b} G[P, pair(c,b)] (1 + delta_cb) T[(b, P), kappa]."""
    n_aux = G.shape[0]
    n_bf = T.shape[1]
    Gs = np.zeros((n_aux, n_act, n_act))
    for c in range(n_act):
        for b in range(n_act):
            Gs[:, c, b] = G[:, pair_index(c, b)] * (2.0 if c == b else 1.0)
    T3 = T.reshape(n_act, n_aux, n_bf)
    return np.einsum("Pcb,bPk->kc", Gs, T3)


# ----------------------------------------------------------------------------------------------
# metric Cholesky and the dense structure eigenproblem


def metric_cholesky(S):
    """Upper Cholesky factor U with S = U^T U (overlap_upper,
    src/vbscf/orbitals/preparation/cholesky.hpp:10-15, an Eigen::LLT): LAPACK dpotrf on the
    upper triangle through SciPy."""
    import scipy.linalg

    return scipy.linalg.cholesky(np.asarray(S, dtype=np.float64), lower=False)


def generalized_eigh(H, S):
    """H C = S C E by LAPACK dsygvd(itype 1, 'V', 'U') -- the routine
    GeneralizedEigensolver::solve_dense calls (src/linalg/eigensolver.cpp:365-388) -- through
    SciPy's LAPACK binding: upper triangles read, eigenvalues ascending, C^T S C = I."""
    import scipy.linalg

    return scipy.linalg.eigh(np.asarray(H, dtype=np.float64), np.asarray(S, dtype=np.float64), lower=False,
                             driver="gvd")


def conditioned_metric(n: int, cond: float, seed: int) -> np.ndarray:
    """Seeded symmetric positive-definite metric with condition number `cond`:
    S = Q diag(logspace(0, -log10 cond, n)) Q^T, Q from the QR factor of a Gaussian matrix."""
    rng = np.random.default_rng(seed)
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    q = q * np.sign(np.diag(r))
    d = np.logspace(0.0, -math.log10(cond), n) if n > 1 else np.ones(1)
    S = (q * d) @ q.T
    return 0.5 * (S + S.T)


# ----------------------------------------------------------------------------------------------
# structure-class generation (src/input/loading/generated_structures.cpp)


def _young_patterns(n_alpha, n_beta, n_orbitals, row_stride):
    """generated_structures.cpp:249-297."""
    if n_alpha <= 0:
        return
    if n_orbitals <= 0 or n_orbitals < n_alpha:
        raise ValueError("invalid orbital count in structure generator")
    row = [0] * row_stride
    for i in range(n_alpha):
        row[i] = i + 1
    mult = n_alpha - n_beta + 1
    maxv = [0] * n_alpha
    if mult == 1:
        maxv[n_beta - 1] = n_orbitals - 1
    else:
        maxv[n_alpha - 1] = n_orbitals
        for idx in range(n_alpha - 1, n_beta, -1):
            maxv[idx - 1] = maxv[idx] - 1
        if n_beta > 0:
            maxv[n_beta - 1] = maxv[n_beta] - 2
    for idx in range(n_beta - 1, 0, -1):
        maxv[idx - 1] = maxv[idx] - 2
    while True:
        yield list(row)
        pivot = n_alpha - 1
        while pivot >= 0 and row[pivot] == maxv[pivot]:
            pivot -= 1
        if pivot < 0:
            break
        row[pivot] += 1
        for s in range(pivot + 1, n_alpha):
            row[s] = row[s - 1] + 1


def _compatible(alpha_row, cand, n_alpha, n_beta):
    """generated_structures.cpp:299-314."""
    for bi in range(n_beta):
        bo = cand[bi]
        if bo < alpha_row[bi]:
            return False
        for ai in range(bi, n_alpha):
            if bo == alpha_row[ai]:
                return False
    return True


def _pad_open_shell(beta_row, n_alpha, n_beta, n_orbitals):
    """generated_structures.cpp:316-328."""
    for idx in range(n_beta, n_alpha):
        beta_row[idx] = n_orbitals + n_alpha - idx


def _covalent_pattern_pairs(n_alpha, n_beta, n_orbitals, row_stride):
    """generated_structures.cpp:330-391."""
    if n_alpha <= 0:
        return
    if n_beta <= 0:
        for a in _young_patterns(n_alpha, 0, n_orbitals, row_stride):
            yield a, [0] * row_stride
        return
    if n_alpha + n_beta == n_orbitals:
        for a in _young_patterns(n_alpha, n_beta, n_orbitals, row_stride):
            b = [0] * row_stride
            nb = 0
            used = set(a[:n_alpha])
            for lab in range(1, n_orbitals + 1):
                if lab not in used:
                    b[nb] = lab
                    nb += 1
            _pad_open_shell(b, n_alpha, n_beta, n_orbitals)
            yield a, b
        return
    for a in _young_patterns(n_alpha, n_beta, n_orbitals, row_stride):
        for cand in _young_patterns(n_beta, 0, n_orbitals, n_beta):
            if not _compatible(a, cand, n_alpha, n_beta):
                continue
            b = [0] * row_stride
            b[:n_beta] = cand[:n_beta]
            _pad_open_shell(b, n_alpha, n_beta, n_orbitals)
            yield a, b


def _reorder_young_bonds(alpha_row, beta_row, n_vector, n_row, n_orbitals):
    """generated_structures.cpp:393-433: pair every alpha label with the smallest remaining
    beta label above it, largest alpha first; returns the alpha row in bond order."""
    left_index = [0] * (3 * n_orbitals)
    right_index = [0] * (3 * n_orbitals)
    rb = list(beta_row[:n_row])
    remaining = n_vector
    for v in range(n_vector):
        right_index[rb[v] - 1] = v + 1
    for _ in range(n_vector, 0, -1):
        left_max = alpha_row[remaining - 1]
        for m in range(remaining):
            if left_max <= rb[m]:
                left_index[left_max - 1] = right_index[rb[m] - 1]
                break
        else:
            m = remaining
        for s in range(m, remaining - 1):
            rb[s] = rb[s + 1]
        remaining -= 1
    for v in range(n_vector):
        rb[left_index[alpha_row[v] - 1] - 1] = alpha_row[v]
    out = list(alpha_row)
    for v in range(n_vector):
        out[v] = rb[v]
    return out


def _binom(n, k):
    return math.comb(n, k) if 0 <= k <= n else 0


def spin_tableau_count(n, spin):
    """generated_structures.cpp:131-143."""
    if n < 0 or spin <= 0 or spin > n + 1:
        return 0
    if n == 0:
        return 1
    if (n - spin + 1) % 2:
        return 0
    beta = (n - spin + 1) // 2
    return _binom(n, beta) - (_binom(n, beta - 1) if beta else 0)


def structure_count_for_class(ionic_class, n_ndb, n_skipped, n_orb, n_el, mult):
    """generated_structures.cpp:145-167."""
    tab = n_orb - 2 * ionic_class - n_skipped + n_ndb
    if tab < 0:
        return 0
    return (_binom(n_orb, ionic_class) * _binom(n_orb - ionic_class, n_skipped + ionic_class - n_ndb)
            * spin_tableau_count(tab, mult))


def parse_structure_classes(keyword: str, n_orb: int, n_el: int, mult: int):
    """generated_structures.cpp:181-245."""
    ndb = max(0, n_el - n_orb)
    reduced_beta = (n_el - 2 * ndb - mult + 1) // 2
    if reduced_beta < 0:
        raise ValueError("negative reduced beta count")
    kw = keyword.upper()
    classes = []
    if "FULL" in kw:
        classes = list(range(0, reduced_beta + 1))
    else:
        if "COV" in kw:
            classes.append(0)
        pos = kw.find("ION(")
        if pos >= 0:
            end = kw.find(")", pos + 4)
            if end < 0:
                raise ValueError("ION( without ')'")
            for tok in kw[pos + 4:end].replace(",", " ").split():
                if "-" in tok:
                    a, b = tok.split("-")
                    classes.extend(range(int(a), int(b) + 1))
                else:
                    classes.append(int(tok))
        elif "ION" in kw:
            classes.extend(range(1, reduced_beta + 1))
    if not classes:
        raise ValueError("empty structure class specification")
    classes = sorted(set(classes))
    if classes[0] < 0 or classes[-1] > reduced_beta:
        raise ValueError("structure class out of range")
    return [c + ndb for c in classes]


def generate_structures(keyword: str, n_orb: int, n_el: int, mult: int = 1, n_inactive: int = 0):
    """Raw structures (1-based orbital labels, n_total_electrons per row), in reference order
    (generated_structures.cpp:475-716)."""
    nb = (n_el - mult + 1) // 2
    na = n_el - nb
    n_total = n_el + 2 * n_inactive
    if (nb == 0 and n_el == mult - 1 and n_el == n_orb) or (nb == n_orb and mult == 1):
        row = [0] * n_total
        tp = n_inactive + nb
        for i in range(tp):
            row[2 * i] = row[2 * i + 1] = i + 1
        for o in range(mult - 1):
            row[2 * tp + o] = tp + o + 1
        return [row]
    out = []
    shift = n_inactive

    def emit(ic, ion_row, remaining, a, b, n_cov_a, n_cov_b):
        row = [0] * n_total
        for i in range(n_inactive):
            row[2 * i] = row[2 * i + 1] = i + 1
        off = 2 * n_inactive
        if ic > 0:
            for ii in range(ic):
                row[off + 2 * ii] = row[off + 2 * ii + 1] = ion_row[ii] + shift
            for bi in range(n_cov_b):
                row[off + 2 * ic + 2 * bi] = remaining[a[bi] - 1] + shift
                row[off + 2 * ic + 2 * bi + 1] = remaining[b[bi] - 1] + shift
            for ai in range(n_cov_b, n_cov_a):
                row[off + 2 * ic + n_cov_b + ai] = remaining[a[ai] - 1] + shift
        else:
            for bi in range(n_cov_b):
                row[off + 2 * bi] = a[bi] + shift
                row[off + 2 * bi + 1] = b[bi] + shift
            for ai in range(n_cov_b, n_cov_a):
                row[off + n_cov_b + ai] = a[ai] + shift
        out.append(row)

    for ic in parse_structure_classes(keyword, n_orb, n_el, mult):
        if ic < 0 or ic > nb:
            raise ValueError("structure class exceeds the active beta count")
        n_cov_a, n_cov_b = na - ic, nb - ic
        if ic > 0:
            for ion_row in _young_patterns(ic, 0, n_orb, ic):
                used = set(ion_row[:ic])
                remaining = [lab for lab in range(1, n_orb + 1) if lab not in used]
                if n_cov_a <= 0:
                    emit(ic, ion_row, remaining, [], [], n_cov_a, n_cov_b)
                    continue
                for a, b in _covalent_pattern_pairs(n_cov_a, n_cov_b, n_orb - ic, na):
                    ra = _reorder_young_bonds(a, b, n_cov_a, na, n_orb) if n_cov_b > 0 else list(a)
                    emit(ic, ion_row, remaining, ra, b, n_cov_a, n_cov_b)
        else:
            for a, b in _covalent_pattern_pairs(na, nb, n_orb, na):
                ra = _reorder_young_bonds(a, b, na, na, n_orb) if nb > 0 else list(a)
                emit(0, [], [], ra, b, n_cov_a, n_cov_b)
    n_skipped = max(0, n_orb - n_el)
    ndb = max(0, n_el - n_orb)
    expected = sum(structure_count_for_class(ic, ndb, n_skipped, n_orb, n_el, mult)
                   for ic in parse_structure_classes(keyword, n_orb, n_el, mult))
    if len(out) != expected:
        raise RuntimeError(f"structure generation count mismatch: {len(out)} != {expected}")
    return out


# ----------------------------------------------------------------------------------------------
# structure -> determinant expansion (src/vbscf/structures/expansion/expander.cpp)


def _sort_sign(orbs):
    """expander.cpp:34-70: parity of earlier-listed orbitals with a higher index."""
    sign = 1
    seen = []
    for o in orbs:
        if o in seen:
            raise ValueError("duplicate orbital in an occupied spin string")
        if sum(1 for s in seen if s > o) & 1:
            sign = -sign
        seen.append(o)
    return sign


def _mask(orbs):
    m = 0
    for o in orbs:
        m |= 1 << o
    return m


def _occ(mask):
    out = []
    i = 0
    while mask:
        if mask & 1:
            out.append(i)
        mask >>= 1
        i += 1
    return out


@dataclass
class Expansion:
    n_structures: int
    n_alpha: int
    n_beta: int
    alpha_strings: list  # sorted masks
    beta_strings: list
    det_alpha: np.ndarray  # string index per determinant
    det_beta: np.ndarray
    offsets: np.ndarray  # CSR by determinant
    term_structure: np.ndarray
    term_coefficient: np.ndarray
    det_alpha_occ: np.ndarray = field(default=None)
    det_beta_occ: np.ndarray = field(default=None)

    @property
    def n_determinants(self):
        return len(self.det_alpha)

    def coefficient_matrix(self) -> np.ndarray:
        """Dense T [n_det x n_str] with T[d, I] = c_dI."""
        T = np.zeros((self.n_determinants, self.n_structures))
        for d in range(self.n_determinants):
            for t in range(self.offsets[d], self.offsets[d + 1]):
                T[d, self.term_structure[t]] += self.term_coefficient[t]
        return T


def expand(structures, n_el_active: int, mult: int = 1, n_inactive: int = 0) -> Expansion:
    """expander.cpp:287-557: unique (alpha, beta) determinants ordered by (alpha rank, beta
    rank), strings ordered by occupation mask, CSR terms per determinant in structure order."""
    n_open = mult - 1
    n_paired = n_el_active - n_open
    nb = n_paired // 2
    per_det = {}
    for s_idx, row in enumerate(structures):
        active = [row[i + 2 * n_inactive] - n_inactive - 1 for i in range(n_el_active)]
        variable = [p for p in range(nb) if active[2 * p] != active[2 * p + 1]]
        for choice in range(1 << len(variable)):
            swapped = {p: (choice >> j) & 1 for j, p in enumerate(variable)}
            alpha = [active[2 * p + swapped.get(p, 0)] for p in range(nb)]
            beta = [active[2 * p + 1 - swapped.get(p, 0)] for p in range(nb)]
            alpha += active[2 * nb:]
            sign = _sort_sign(alpha) * _sort_sign(beta)
            key = (_mask(alpha), _mask(beta))
            per_det.setdefault(key, []).append((s_idx, float(sign)))
    a_masks = sorted({k[0] for k in per_det})
    b_masks = sorted({k[1] for k in per_det})
    a_rank = {m: i for i, m in enumerate(a_masks)}
    b_rank = {m: i for i, m in enumerate(b_masks)}
    keys = sorted(per_det, key=lambda k: (a_rank[k[0]], b_rank[k[1]]))
    offsets = [0]
    ts, tc = [], []
    for key in keys:
        merged = {}
        for s_idx, c in per_det[key]:
            merged[s_idx] = merged.get(s_idx, 0.0) + c
        for s_idx in sorted(merged):
            if merged[s_idx] != 0.0:
                ts.append(s_idx)
                tc.append(merged[s_idx])
        offsets.append(len(ts))
    det_alpha = np.array([a_rank[k[0]] for k in keys], dtype=np.int32)
    det_beta = np.array([b_rank[k[1]] for k in keys], dtype=np.int32)
    n_alpha = nb + n_open
    exp = Expansion(
        n_structures=len(structures), n_alpha=n_alpha, n_beta=nb, alpha_strings=a_masks, beta_strings=b_masks,
        det_alpha=det_alpha, det_beta=det_beta, offsets=np.array(offsets, dtype=np.int64),
        term_structure=np.array(ts, dtype=np.int32), term_coefficient=np.array(tc, dtype=np.float64))
    exp.det_alpha_occ = np.array([_occ(a_masks[i]) for i in det_alpha], dtype=np.int32).reshape(len(keys), n_alpha)
    exp.det_beta_occ = np.array([_occ(b_masks[i]) for i in det_beta], dtype=np.int32).reshape(len(keys), nb)
    return exp


def rumer_pairings(first: int, past_last: int):
    """Non-crossing perfect matchings of sites [first, past_last), as the reference test builds
    them (tests/vbscf/unit/test_structure_tiles.cpp:95-112)."""
    if first == past_last:
        return [[]]
    result = []
    for mate in range(first + 1, past_last, 2):
        for left in rumer_pairings(first + 1, mate):
            for right in rumer_pairings(mate + 1, past_last):
                result.append([(first, mate)] + left + right)
    return result


# ----------------------------------------------------------------------------------------------
# VBSCF on s-type Gaussian molecules (configuration "plain VBSCF": H chains in 6-31G)


def _boys0(t: float) -> float:
    if t < 1e-8:
        return 1.0 - t / 3.0 + t * t / 10.0
    return 0.5 * math.sqrt(math.pi / t) * math.erf(math.sqrt(t))


def s_shell_integrals(charges, coords, shells):
    """Overlap, core Hamiltonian (kinetic + nuclear attraction), (mu nu|la si) and the nuclear
    repulsion for contracted s shells [(atom, exponents, coefficients for normalized
    primitives)], each renormalized to unit self-overlap.  Closed-form s-type Gaussian
    integrals (the Boys function F0); the reference obtains them from libcint."""
    n = len(shells)
    prims = []
    for atom, exps, coefs in shells:
        e = np.asarray(exps, float)
        c = np.asarray(coefs, float) * (2.0 * e / math.pi) ** 0.75
        norm = sum(c[i] * c[j] * (math.pi / (e[i] + e[j])) ** 1.5 for i in range(len(e)) for j in range(len(e)))
        prims.append((np.asarray(coords[atom], float), e, c / math.sqrt(norm)))
    S = np.zeros((n, n))
    H = np.zeros((n, n))
    for m in range(n):
        for v in range(n):
            A, ea, ca = prims[m]
            B, eb, cb = prims[v]
            ab2 = float(np.sum((A - B) ** 2))
            for a, x in zip(ea, ca):
                for b, y in zip(eb, cb):
                    p, mu = a + b, a * b / (a + b)
                    sij = (math.pi / p) ** 1.5 * math.exp(-mu * ab2)
                    S[m, v] += x * y * sij
                    H[m, v] += x * y * mu * (3.0 - 2.0 * mu * ab2) * sij
                    P = (a * A + b * B) / p
                    for Z, Cn in zip(charges, coords):
                        H[m, v] -= x * y * Z * 2.0 * math.pi / p * math.exp(-mu * ab2) * _boys0(
                            p * float(np.sum((P - np.asarray(Cn)) ** 2)))
    eri = np.zeros((n, n, n, n))
    for m in range(n):
        for v in range(m + 1):
            for l in range(n):
                for s in range(l + 1):
                    if m * (m + 1) // 2 + v < l * (l + 1) // 2 + s:
                        continue
                    A, ea, ca = prims[m]
                    B, eb, cb = prims[v]
                    C, ec, cc = prims[l]
                    D, ed, cd = prims[s]
                    val = 0.0
                    for a, xa in zip(ea, ca):
                        for b, xb in zip(eb, cb):
                            p = a + b
                            P = (a * A + b * B) / p
                            kab = xa * xb * math.exp(-a * b / p * float(np.sum((A - B) ** 2)))
                            for c, xc in zip(ec, cc):
                                for d, xd in zip(ed, cd):
                                    q = c + d
                                    Q = (c * C + d * D) / q
                                    kcd = xc * xd * math.exp(-c * d / q * float(np.sum((C - D) ** 2)))
                                    val += kab * kcd * 2.0 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * _boys0(
                                        p * q / (p + q) * float(np.sum((P - Q) ** 2)))
                    for t in ((m, v, l, s), (v, m, l, s), (m, v, s, l), (v, m, s, l), (l, s, m, v), (s, l, m, v),
                              (l, s, v, m), (s, l, v, m)):
                        eri[t] = val
    enuc = 0.0
    for i in range(len(charges)):
        for j in range(i + 1, len(charges)):
            enuc += charges[i] * charges[j] / float(np.linalg.norm(np.asarray(coords[i]) - np.asarray(coords[j])))
    return S, H, eri, enuc


def active_integrals(S_ao, h_ao, eri_ao, C):
    """S_act = C^T S C, h_act = C^T h C, packed (pq|rs) (transform_exact_active_integrals,
    src/integrals/active/exact.cpp:347-557, as a dense four-index transform)."""
    S = C.T @ S_ao @ C
    h = C.T @ h_ao @ C
    full = np.einsum("mnls,mp,nq,lr,st->pqrt", eri_ao, C, C, C, C, optimize=True)
    n = C.shape[1]
    P = n * (n + 1) // 2
    pairs = [(a, b) for a in range(n) for b in range(a + 1)]
    packed = np.zeros(P * (P + 1) // 2)
    for x, (a, b) in enumerate(pairs):
        for y, (c, d) in enumerate(pairs[:x + 1]):
            packed[x * (x + 1) // 2 + y] = full[a, b, c, d]
    return S, h, packed


class VbscfOracle:
    """Energy (lowest structure root + nuclear repulsion, src/vbscf/workflow/evaluator.cpp:
    103-108), its gradient by Richardson-extrapolated central differences over the allowed
    coefficients, and a quasi-Newton solve, all on the CPU restatement above."""

    def __init__(self, charges, coords, shells, pattern, n_electrons, multiplicity=1, keyword="COV"):
        self.S_ao, self.h_ao, self.eri_ao, self.enuc = s_shell_integrals(charges, coords, shells)
        self.pattern = pattern
        self.n = len(pattern)
        self.expansion = expand(generate_structures(keyword, self.n, n_electrons, multiplicity), n_electrons,
                                multiplicity)
        self.where = [(m, a) for a, funcs in enumerate(pattern) for m in funcs]

    def matrices(self, C):
        S, h, eri = active_integrals(self.S_ao, self.h_ao, self.eri_ao, C)
        return structure_matrices(self.n, self.expansion, S, h, eri)[:2]

    def energy(self, C):
        Hs, Ss = self.matrices(C)
        return generalized_eigh(Hs, Ss)[0][0] + self.enuc

    def gradient(self, C, step=1e-4):
        g = np.zeros_like(C)
        for (m, a) in self.where:
            def f(t):
                Ct = C.copy()
                Ct[m, a] += t
                return self.energy(Ct)
            d1 = (f(step) - f(-step)) / (2 * step)
            d2 = (f(step / 2) - f(-step / 2)) / step
            g[m, a] = (4 * d2 - d1) / 3
        return g

    def solve(self, C0, gtol=1e-7, maxiter=500):
        import scipy.optimize

        x0 = np.array([C0[m, a] for (m, a) in self.where])

        def unpack(x):
            C = np.zeros_like(C0)
            for v, (m, a) in zip(x, self.where):
                C[m, a] = v
            return C

        def fun(x):
            C = unpack(x)
            g = self.gradient(C)
            return self.energy(C), np.array([g[m, a] for (m, a) in self.where])

        res = scipy.optimize.minimize(fun, x0, jac=True, method="L-BFGS-B",
                                      options={"maxcor": 100, "gtol": gtol, "ftol": 1e-15, "maxiter": maxiter})
        return res.fun, unpack(res.x), res
