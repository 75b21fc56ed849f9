"""The oracle is pinned before it is trusted: against the golden fixtures (an independent
Fock-space evaluation), the reference's structure counts and Rumer property, and cofactor
identities checked against explicit deleted minors (as the reference's
tests/vbscf/unit/test_cofactor_differential.cpp does)."""

import itertools
import math

import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden

# the reference's structure-test tolerances (test_structure_tiles.cpp:310-319)
H_TOL = 2e-10
S_TOL = 2e-11


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_matches_golden(name):
    z = load_golden(name)
    n, nel, mult, kw = int(z["n"]), int(z["n_el"]), int(z["mult"]), str(z["keyword"])
    structures = O.generate_structures(kw, n, nel, mult)
    assert np.array_equal(np.array(structures), z["structures"])
    exp = O.expand(structures, nel, mult)
    Hs, Ss, _ = O.structure_matrices(n, exp, z["S"], z["h"], z["eri"])
    scale_h = max(1.0, np.linalg.norm(z["Hs"]))
    scale_s = max(1.0, np.linalg.norm(z["Ss"]))
    assert np.linalg.norm(Hs - z["Hs"]) <= H_TOL * scale_h
    assert np.linalg.norm(Ss - z["Ss"]) <= S_TOL * scale_s
    Hd, Sd = O.determinant_matrices(n, exp.det_alpha_occ, exp.det_beta_occ, z["S"], z["h"], z["eri"])
    assert np.abs(Hd - z["Hd"]).max() <= H_TOL * max(1.0, np.abs(z["Hd"]).max())
    assert np.abs(Sd - z["Sd"]).max() <= S_TOL * max(1.0, np.abs(z["Sd"]).max())


@pytest.mark.parametrize("n", [4, 6, 8, 10, 12, 14])
def test_covalent_counts_and_rumer(n):
    structures = O.generate_structures("COV", n, n)
    expected = math.comb(n, n // 2) - math.comb(n, n // 2 - 1)
    assert len(structures) == expected
    rumer = {tuple(sorted(tuple(sorted(b)) for b in p)) for p in O.rumer_pairings(0, n)}
    got = {tuple(sorted(tuple(sorted((row[2 * i] - 1, row[2 * i + 1] - 1))) for i in range(n // 2)))
           for row in structures}
    assert got == rumer
    exp = O.expand(structures, n)
    assert exp.n_determinants == math.comb(n, n // 2)
    assert len(exp.term_structure) == expected * 2 ** (n // 2)


@pytest.mark.parametrize("n", [4, 6, 8, 10, 12])
def test_singly_ionic_counts(n):
    m = n - 2
    ionic = n * (n - 1) * (math.comb(m, m // 2) - math.comb(m, m // 2 - 1))
    assert len(O.generate_structures("ION(1)", n, n)) == ionic


def _adjugate(x):
    k = x.shape[0]
    return np.array([[(-1) ** (i + j) * np.linalg.det(np.delete(np.delete(x, i, 0), j, 1)) for j in range(k)]
                     for i in range(k)])


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 7])
@pytest.mark.parametrize("rank_drop", [0, 1, 2, 3])
def test_first_and_second_cofactors_against_minors(k, rank_drop):
    if rank_drop > k:
        pytest.skip("rank drop larger than the block")
    rng = np.random.default_rng(100 * k + rank_drop)
    x = rng.standard_normal((k, k))
    if rank_drop:
        u, s, vt = np.linalg.svd(x)
        s[k - rank_drop:] = 0.0
        x = (u * s) @ vt
    det, nullity, _, cof = O.resolve(x)
    assert nullity == rank_drop or (k <= 1 and rank_drop == 1)
    scale = max(1.0, np.abs(x).max()) ** max(0, k - 1)
    if k > 1 and nullity <= 1:
        assert np.abs(cof - _adjugate(x)).max() <= 1e-12 * scale
    if k >= 2 and nullity <= 2:
        for r1, r2 in itertools.combinations(range(k), 2):
            for c1, c2 in itertools.combinations(range(k), 2):
                minor = np.delete(np.delete(x, [r1, r2], 0), [c1, c2], 1)
                ref = (-1) ** (r1 + r2 + c1 + c2) * (np.linalg.det(minor) if minor.size else 1.0)
                assert abs(O.second_cofactor(x, r1, r2, c1, c2) - ref) <= 1e-12 * scale


def test_full_pivot_lu_rank_threshold():
    x = np.diag([1.0, 1e-6, 1e-13])
    rank, det, inv = O.full_pivot_lu(x)
    assert rank == 2 and inv is None
    rank, det, inv = O.full_pivot_lu(np.diag([1.0, 1e-6, 1e-11]))
    assert rank == 3 and abs(det - 1e-17) < 1e-30


def test_linalg_oracle_is_dsygvd():
    # the oracle's dense eigenproblem is LAPACK dsygvd; cross-check it against an explicit
    # Cholesky reduction to a standard symmetric problem
    n = 30
    rng = np.random.default_rng(4)
    a = rng.standard_normal((n, n))
    H = 0.5 * (a + a.T)
    S = O.conditioned_metric(n, 1e5, seed=5)
    assert abs(np.linalg.cond(S) / 1e5 - 1) < 1e-6
    U = O.metric_cholesky(S)
    assert np.abs(U.T @ U - S).max() < 1e-14
    w, C = O.generalized_eigh(H, S)
    Ui = np.linalg.inv(U)
    wr = np.linalg.eigvalsh(Ui.T @ H @ Ui)
    assert np.abs(w - wr).max() < 1e-12 * np.abs(w).max()
    assert np.abs(C.T @ S @ C - np.eye(n)).max() < 1e-10


def _ri_inputs(n_aux, n_bf, n_act, seed):
    rng = np.random.default_rng(seed)
    npair = n_bf * (n_bf + 1) // 2
    B = rng.standard_normal((n_aux, npair))
    C = rng.standard_normal((n_bf, n_act)) / np.sqrt(n_bf)
    return B, C


def test_ri_oracle_restatements_agree():
    # the numpy one-index factors reproduce the C++ restatement's L, and the adjoint matches
    # central differences of a linear functional of L (exact up to rounding: L is quadratic in C)
    n_aux, n_bf, n_act = 9, 7, 3
    B, C = _ri_inputs(n_aux, n_bf, n_act, 1)
    L, K = O.ri_transform(B, C)
    T = O.ri_one_index(B, C)
    L2 = np.zeros_like(L)
    T3 = T.reshape(n_act, n_aux, n_bf)
    for a in range(n_act):
        for b in range(a + 1):
            L2[:, O.pair_index(a, b)] = T3[a] @ C[:, b]
    assert np.abs(L - L2).max() < 1e-13
    assert np.abs(K - np.array([L[:, p] @ L[:, q] for p in range(L.shape[1]) for q in range(p + 1)])).max() < 1e-12
    rng = np.random.default_rng(2)
    G = rng.standard_normal(L.shape)
    dC = O.ri_adjoint(T, G, n_act)
    D = rng.standard_normal(C.shape)
    h = 1e-3
    fp = np.sum(G * O.ri_transform(B, C + h * D)[0])
    fm = np.sum(G * O.ri_transform(B, C - h * D)[0])
    assert abs((fp - fm) / (2 * h) - np.sum(dC * D)) < 1e-9


@pytest.mark.parametrize("n,keyword,mult,overlap", [(6, "COV", 1, "random"), (8, "COV ION(1)", 1, "random"),
                                                    (6, "COV", 3, "random"), (8, "COV ION(1)", 1, "identity"),
                                                    (10, "COV", 1, "random")])
def test_cached_algorithm_equals_direct_oracle(n, keyword, mult, overlap):
    """The cached restatement (ordered spin-pair cache with projected images, then a sparse dot per
    determinant pair: the reference's CPU hot-loop shape, used as the timed CPU baseline) gives the
    same structure H/S as the per-pair restatement used as the parity checker."""
    from vbcore import workloads

    S, h, eri = workloads.active_space(n, 3 * n, 17)
    if overlap == "identity":
        S = np.eye(n)
    ex = O.expand(O.generate_structures(keyword, n, n, mult), n, mult)
    H1, S1, _ = O.structure_matrices(n, ex, S, h, eri, threads=4)
    H2, S2, tm = O.cached_structure_matrices(n, ex, S, h, eri, threads=4)
    assert tm["pairs"] == ex.n_determinants ** 2
    assert np.abs(H1 - H2).max() <= 1e-13 * max(1.0, np.abs(H1).max())
    assert np.abs(S1 - S2).max() <= 1e-13 * max(1.0, np.abs(S1).max())
    # a row-limited call evaluates only those determinant rows: the timing sample
    _, _, part = O.cached_structure_matrices(n, ex, S, h, eri, threads=4, det_rows=2)
    assert part["pairs"] == 2 * ex.n_determinants


def test_ri_pair_factor_frame_restatement():
    """The oracle's frame transform of packed RI pair factors: identity frame, an explicit
    single-row check, and the orthogonal directional form equal to the raw one at dQ = -Q K."""
    rng = np.random.default_rng(3)
    n, n_aux = 5, 7
    B = rng.standard_normal((n_aux, n * (n + 1) // 2))
    dB = rng.standard_normal(B.shape)
    Q = np.eye(n) + 0.3 * rng.standard_normal((n, n))
    K = rng.standard_normal((n, n))
    assert np.allclose(O.ri_pair_factors_frame(B, np.eye(n)), B, atol=0, rtol=0)
    hi, lo = np.tril_indices(n)
    M = np.zeros((n, n))
    M[hi, lo] = B[2]
    M[lo, hi] = B[2]
    assert np.allclose(O.ri_pair_factors_frame(B, Q)[2], (Q.T @ M @ Q)[hi, lo], rtol=1e-14, atol=1e-14)
    a = O.ri_pair_factors_frame(O.ri_pair_factors_frame(B, Q), Q, 2, dB, K)
    b = O.ri_pair_factors_frame(B, Q, 1, dB, -Q @ K)
    assert np.abs(a - b).max() < 1e-12
