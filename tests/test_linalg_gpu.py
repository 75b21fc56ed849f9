"""Metric Cholesky and the dense generalized eigenproblem on the device against LAPACK
(dpotrf / dsygvd through SciPy, the routines the reference's Eigen LLT and
GeneralizedEigensolver::solve_dense stand on)."""

import numpy as np
import pytest

import oracle as O
import vbcore
from vbcore import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = vbcore.Context(0)
    yield c
    c.close()


def _random_symmetric(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    return 0.5 * (a + a.T)


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 64, 97, 200, 429, 1000])
@pytest.mark.parametrize("cond", [1e2, 1e6, 1e10])
def test_cholesky_matches_lapack(ctx, n, cond):
    S = O.conditioned_metric(n, cond, seed=n)
    U = vbcore.metric_cholesky(ctx, S)
    assert np.array_equal(U, np.triu(U))
    backward = np.linalg.norm(U.T @ U - S) / np.linalg.norm(S)
    assert backward < 1e-15 * max(1, n) ** 0.5 * 4
    Ur = O.metric_cholesky(S)
    # forward error of a Cholesky factor is bounded by cond(S) eps
    assert np.abs(U - Ur).max() <= 1e-15 * cond * np.abs(Ur).max() * 10


def test_cholesky_reads_upper_triangle_only(ctx):
    S = O.conditioned_metric(40, 1e3, seed=3)
    Sl = np.triu(S) + np.tril(np.full_like(S, 7.0), -1)  # garbage below the diagonal
    assert np.abs(vbcore.metric_cholesky(ctx, Sl) - O.metric_cholesky(S)).max() < 1e-12


@pytest.mark.parametrize("n,bad", [(10, 4), (70, 40), (150, 1), (300, 200)])
def test_cholesky_reports_the_failing_minor(ctx, n, bad):
    S = O.conditioned_metric(n, 1e2, seed=n)
    S[bad - 1, bad - 1] = -1.0  # leading minor of order `bad` is the first that is not positive
    with pytest.raises(vbcore.VbError) as e:
        vbcore.metric_cholesky(ctx, S)
    assert e.value.status == 4 and e.value.info == bad


@pytest.mark.parametrize("n", [1, 2, 3, 5, 14, 42, 97, 132, 429])
def test_generalized_eigh_matches_dsygvd(ctx, n):
    H = _random_symmetric(n, 100 + n)
    S = O.conditioned_metric(n, 1e4, seed=200 + n)
    w, C = vbcore.generalized_eigh(ctx, H, S)
    wr, Cr = O.generalized_eigh(H, S)
    scale = np.abs(wr).max()
    assert np.abs(w - wr).max() < 1e-11 * scale
    assert np.all(np.diff(w) >= 0)
    # C^T S C = I and H C = S C diag(w)
    assert np.abs(C.T @ S @ C - np.eye(n)).max() < 1e-10
    assert np.abs(H @ C - S @ C * w).max() < 1e-10 * scale * max(1.0, np.abs(C).max())
    # lowest root's vector up to sign
    c0, r0 = C[:, 0], Cr[:, 0]
    assert min(np.abs(c0 - r0).max(), np.abs(c0 + r0).max()) < 1e-8 * np.abs(r0).max()


def test_generalized_eigh_uses_upper_triangles(ctx):
    n = 50
    H = _random_symmetric(n, 1)
    S = O.conditioned_metric(n, 1e3, seed=2)
    junk = np.tril(np.full((n, n), 3.0), -1)
    w, _ = vbcore.generalized_eigh(ctx, np.triu(H) + junk, np.triu(S) + junk)
    assert np.abs(w - O.generalized_eigh(H, S)[0]).max() < 1e-11 * np.abs(w).max()


def test_generalized_eigh_rejects_indefinite_overlap(ctx):
    n = 20
    H = _random_symmetric(n, 5)
    S = O.conditioned_metric(n, 1e2, seed=6)
    S[7, 7] = -2.0
    with pytest.raises(vbcore.VbError) as e:
        vbcore.generalized_eigh(ctx, H, S)
    assert e.value.status == 4 and e.value.info == n + 8
    assert "not positive definite" in str(e.value)


def test_degenerate_spectrum(ctx):
    # repeated eigenvalues: the eigenvalues must still match and C must stay S-orthonormal
    n = 60
    rng = np.random.default_rng(9)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.repeat(np.arange(12, dtype=np.float64), 5)
    A = (q * d) @ q.T
    S = O.conditioned_metric(n, 1e2, seed=10)
    Ls = np.linalg.cholesky(S)
    H = Ls @ A @ Ls.T
    H = 0.5 * (H + H.T)
    w, C = vbcore.generalized_eigh(ctx, H, S)
    assert np.abs(w - np.sort(d)).max() < 1e-11 * 12
    assert np.abs(C.T @ S @ C - np.eye(n)).max() < 1e-10


def test_structure_energy_matches_oracle(ctx):
    # lowest root of the structure problem (the VBSCF energy without core and nuclear terms)
    n = 10
    S, h, eri = workloads.active_space(n, 3 * n, 77)
    rows = vbcore.generate_structures("COV", n, n)
    ex = vbcore.expand_structures(rows, n)
    plan = vbcore.HsPlan(ctx, ex, n)
    Hs, Ss = plan.execute(S, h, eri)
    w, C = vbcore.generalized_eigh(ctx, Hs, Ss)
    ex_o = O.expand(O.generate_structures("COV", n, n), n)
    Hr, Sr, _ = O.structure_matrices(n, ex_o, S, h, eri)
    wr, _ = O.generalized_eigh(Hr, Sr)
    assert abs(w[0] - wr[0]) < 1e-9
    plan.close()


def test_batched_matches_single(ctx):
    problems = []
    for i, n in enumerate([1, 2, 5, 14, 42, 60, 33]):
        problems.append((_random_symmetric(n, 300 + i), O.conditioned_metric(n, 1e3, seed=400 + i)))
    out = vbcore.generalized_eigh_batched(ctx, problems)
    for (H, S), (w, C) in zip(problems, out):
        wr, _ = O.generalized_eigh(H, S)
        assert np.abs(w - wr).max() < 1e-11 * np.abs(wr).max()
        assert np.abs(C.T @ S @ C - np.eye(len(w))).max() < 1e-10


@pytest.mark.parametrize("kw,n", [("COV", 8), ("COV ION(1)", 8), ("COV ION(1)", 10)])
def test_lowest_root_matches_dsygvd_on_structure_problems(ctx, kw, n):
    S, h, eri = workloads.active_space(n, 3 * n, 300 + n)
    rows = vbcore.generate_structures(kw, n, n)
    ex = vbcore.expand_structures(rows, n)
    plan = vbcore.HsPlan(ctx, ex, n)
    Hs, Ss = plan.execute(S, h, eri)
    E, c, its = vbcore.lowest_root(ctx, Hs, Ss, tolerance=1e-11)
    wr, Cr = O.generalized_eigh(Hs, Ss)
    assert abs(E - wr[0]) < 1e-9 * max(1.0, abs(wr[0]))
    assert abs(c @ Ss @ c - 1.0) < 1e-10
    r0 = Cr[:, 0]
    assert min(np.abs(c - r0).max(), np.abs(c + r0).max()) < 1e-6 * np.abs(r0).max()
    plan.close()


def test_lowest_root_random(ctx):
    n = 700
    H = _random_symmetric(n, 12)
    S = O.conditioned_metric(n, 1e3, seed=13)
    E, c, its = vbcore.lowest_root(ctx, H, S, tolerance=1e-11, max_iterations=3000)
    assert abs(E - O.generalized_eigh(H, S)[0][0]) < 1e-9 * max(1.0, abs(E))


def test_grid_barrier_timeout_is_reported_and_the_context_stays_usable():
    """The cooperative solver's grid barrier gives up after a bounded number of polls: with a
    one-poll limit the waits run out, the kernel ends and the call returns VB_ERR_TIMEOUT (no
    trap, no hang); after the default limit is restored the same context solves the problem.
    The blocked Cholesky above the one-CTA size has no grid barrier: the limit does not touch it."""
    c = vbcore.Context(0)
    try:
        n = 200  # above the one-CTA size: a grid-wide cooperative launch with a grid barrier
        H = _random_symmetric(n, 7)
        S = O.conditioned_metric(n, 1e3, seed=8)
        c.set_barrier_spin_limit(1)
        with pytest.raises(vbcore.VbError) as e:
            vbcore.generalized_eigh(c, H, S)
        assert e.value.status == 6 and "grid barrier timed out" in str(e.value)
        U = vbcore.metric_cholesky(c, S)
        assert np.abs(U - O.metric_cholesky(S)).max() < 1e-12
        c.set_barrier_spin_limit(0)
        w, _ = vbcore.generalized_eigh(c, H, S)
        wr, _ = O.generalized_eigh(H, S)
        assert np.abs(w - wr).max() < 1e-11 * np.abs(wr).max()
        with pytest.raises(vbcore.VbError):
            c.set_barrier_spin_limit(-1)
    finally:
        c.close()
