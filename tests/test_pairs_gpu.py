"""GPU parity of the determinant-pair path through the C ABI against the oracle.

Tolerances are the north-star bar for structure matrices: 1e-10 relative on every H/S element
(relative to max(1, max |H|)), and the reference's own per-pair closeness for the determinant
level."""

import numpy as np
import pytest

import oracle as O
import vbcore
from vbcore import workloads
from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu
REL = 1e-10


@pytest.fixture(scope="module")
def ctx():
    c = vbcore.Context(0)
    yield c
    c.close()


def _rel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def _plan(ctx, kw, n, nel, mult=1):
    rows = vbcore.generate_structures(kw, n, nel, mult)
    ex = vbcore.expand_structures(rows, nel, mult)
    return vbcore.HsPlan(ctx, ex, n), O.expand(O.generate_structures(kw, n, nel, mult), nel, mult)


@pytest.mark.parametrize("name", golden_cases())
def test_structure_matrices_match_golden(ctx, name):
    z = load_golden(name)
    n, nel, mult, kw = int(z["n"]), int(z["n_el"]), int(z["mult"]), str(z["keyword"])
    plan, _ = _plan(ctx, kw, n, nel, mult)
    H, S = plan.execute(z["S"], z["h"], z["eri"])
    assert _rel(H, z["Hs"]) < REL
    assert _rel(S, z["Ss"]) < REL


@pytest.mark.parametrize("kw,n,seed", [("COV", 8, 1), ("COV", 10, 2), ("COV", 12, 3), ("COV ION(1)", 8, 4),
                                       ("COV ION(1)", 6, 5), ("FULL", 6, 6), ("COV ION(1)", 10, 7)])
def test_structure_matrices_match_oracle(ctx, kw, n, seed):
    S, h, eri = workloads.active_space(n, 3 * n, seed)
    plan, ex = _plan(ctx, kw, n, n)
    H, So = plan.execute(S, h, eri)
    Hr, Sr, _ = O.structure_matrices(n, ex, S, h, eri)
    assert _rel(H, Hr) < REL
    assert _rel(So, Sr) < REL
    assert np.array_equal(H, H.T) and np.array_equal(So, So.T)
    st = plan.stats()
    assert st["spin_pairs"] > 0 and st["kernel_launches"] >= 5
    # (ij|kl) = sum_P B_ij^P B_kl^P with 3n auxiliary functions: the factorization stops at that rank
    assert st["factor_columns"] == min(3 * n, n * (n + 1) // 2)
    if n <= 8:
        # one evaluation per orbit {(d, e), (flip d, flip e)} of unordered pairs (brute force)
        n_det = ex.n_determinants
        index = {(int(a), int(b)): d for d, (a, b) in enumerate(zip(ex.det_alpha, ex.det_beta))}
        flip = [index.get((int(b), int(a))) for a, b in zip(ex.det_alpha, ex.det_beta)]
        orbits = set()
        for d in range(n_det):
            for e in range(d, n_det):
                if None in (flip[d], flip[e]):
                    orbits.add((d, e))
                    continue
                f = tuple(sorted((flip[d], flip[e])))
                orbits.add(min((d, e), f))
        if None in flip:
            assert st["determinant_pairs"] == n_det * (n_det + 1) // 2
        else:
            assert st["determinant_pairs"] == len(orbits)


def test_open_shell_tables(ctx):
    # doublet and triplet: alpha and beta string tables differ
    for n, nel, mult in ((5, 5, 2), (6, 4, 3), (7, 6, 3)):
        S, h, eri = workloads.active_space(n, 2 * n, 11 + n)
        plan, ex = _plan(ctx, "COV", n, nel, mult)
        H, So = plan.execute(S, h, eri)
        Hr, Sr, _ = O.structure_matrices(n, ex, S, h, eri)
        assert _rel(H, Hr) < REL and _rel(So, Sr) < REL


def test_orthogonal_orbitals_take_the_exact_path(ctx):
    z = load_golden("orthogonal_n6")
    plan, _ = _plan(ctx, str(z["keyword"]), int(z["n"]), int(z["n_el"]))
    H, S = plan.execute(z["S"], z["h"], z["eri"])
    assert _rel(H, z["Hs"]) < REL and _rel(S, z["Ss"]) < REL
    st = plan.stats()
    assert st["careful_spin_pairs"] > 0  # singular blocks (nullity 1, 2, ...) present


def test_determinant_pairs_match_oracle(ctx):
    n = 8
    S, h, eri = workloads.active_space(n, 24, 7)
    plan, ex = _plan(ctx, "COV ION(1)", n, n)
    Hd, Sd = O.determinant_matrices(n, ex.det_alpha_occ, ex.det_beta_occ, S, h, eri)
    rng = np.random.default_rng(0)
    pairs = rng.integers(0, ex.n_determinants, size=(4000, 2))
    ho, so = plan.determinant_pairs(S, h, eri, pairs)
    assert np.abs(ho - Hd[pairs[:, 0], pairs[:, 1]]).max() < REL * max(1.0, np.abs(Hd).max())
    assert np.abs(so - Sd[pairs[:, 0], pairs[:, 1]]).max() < REL * max(1.0, np.abs(Sd).max())


def test_determinant_pairs_in_device_memory_use_the_callers_order(ctx):
    # this covalent + ionic list is reordered inside the plan (determinants grouped by the first
    # structure group using them); pair indices in device memory are mapped like host ones
    import ctypes
    import torch
    n = 8
    S, h, eri = workloads.active_space(n, 24, 7)
    plan, ex = _plan(ctx, "COV ION(1)", n, n)
    rng = np.random.default_rng(1)
    pairs = rng.integers(0, ex.n_determinants, size=(3000, 2)).astype(np.int64)
    ho, so = plan.determinant_pairs(S, h, eri, pairs)
    dev = torch.device("cuda", 0)
    dS = torch.tensor(np.ascontiguousarray(S.T), device=dev)
    dh = torch.tensor(np.ascontiguousarray(h.T), device=dev)
    de = torch.tensor(np.ascontiguousarray(eri, dtype=np.float64), device=dev)
    dp = torch.tensor(pairs, device=dev)
    dho = torch.zeros(len(pairs), dtype=torch.float64, device=dev)
    dso = torch.zeros(len(pairs), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    st = vbcore.load_library().vb_hs_plan_determinant_pairs(plan._h, p(dS), p(dh), p(de), len(pairs), p(dp),
                                                            vbcore.VB_MEM_DEVICE, p(dho), p(dso))
    assert st == 0
    assert np.array_equal(dho.cpu().numpy(), ho) and np.array_equal(dso.cpu().numpy(), so)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 6, 7, 9])
def test_resolve_overlaps_reference_semantics(ctx, k):
    rng = np.random.default_rng(k)
    blocks = []
    for drop in range(0, min(k, 3) + 1):
        for _ in range(6):
            x = rng.standard_normal((k, k))
            if drop:
                u, s, vt = np.linalg.svd(x)
                s[k - drop:] = 0.0
                x = (u * s) @ vt
            blocks.append(x)
    blocks.append(np.zeros((k, k)))
    blocks = np.array(blocks)
    det, nul, cof = ctx.resolve_overlaps(blocks)
    for i, x in enumerate(blocks):
        d_ref, n_ref, _, c_ref = O.resolve(x)
        assert nul[i] == n_ref
        assert abs(det[i] - d_ref) <= 1e-12 * max(1.0, abs(d_ref))
        assert np.abs(cof[i] - c_ref).max() <= 1e-11 * max(1.0, np.abs(c_ref).max())


def test_same_spin_pairs_match_oracle(ctx):
    n, k = 10, 5
    S, h, eri = workloads.active_space(n, 30, 3)
    rng = np.random.default_rng(5)
    L = np.array([np.sort(rng.choice(n, k, replace=False)) for _ in range(300)])
    R = np.array([np.sort(rng.choice(n, k, replace=False)) for _ in range(300)])
    R[:20] = L[:20]  # diagonal pairs
    sc, cof = ctx.same_spin_pairs(n, L, R, S, h, eri)
    for i in range(len(L)):
        ref = O.spin_pair(n, L[i], R[i], S, h, eri)
        assert int(sc[i, 3]) == ref["nullity"]
        for j, key in enumerate(("det", "h1", "htot")):
            assert abs(sc[i, j] - ref[key]) <= 1e-11 * max(1.0, abs(ref[key]))


def test_reproducible_and_device_path(ctx):
    import torch
    n = 10
    S, h, eri = workloads.active_space(n, 30, 9)
    plan, _ = _plan(ctx, "COV", n, n)
    H1, S1 = plan.execute(S, h, eri)
    H2, S2 = plan.execute(S, h, eri)
    assert np.array_equal(H1, H2) and np.array_equal(S1, S2)
    dev = torch.device("cuda:0")
    tS = torch.tensor(S.T.copy(), device=dev)
    th = torch.tensor(h.T.copy(), device=dev)
    te = torch.tensor(eri, device=dev)
    ns = plan.n_structures
    tH = torch.empty((ns, ns), dtype=torch.float64, device=dev)
    tSo = torch.empty((ns, ns), dtype=torch.float64, device=dev)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    plan.execute_device(tS.data_ptr(), th.data_ptr(), te.data_ptr(), tH.data_ptr(), tSo.data_ptr())
    torch.cuda.synchronize()
    ctx.set_stream(None)
    assert np.array_equal(tH.cpu().numpy().T, H1) and np.array_equal(tSo.cpu().numpy().T, S1)


def test_full_size_microbenchmark_properties(ctx):
    """n_active = 14, 3432 determinants, 429 structures (the microbenchmark shape): every one of
    the 429 x 429 H and S elements against the oracle (all 5,891,028 unordered determinant pairs,
    all host threads), plus size-independent properties (symmetry, positive metric, linearity of H
    in (h, (ij|kl)))."""
    import os

    n = 14
    S, h, eri = workloads.active_space(n, 42, 2026)
    plan, ex = _plan(ctx, "COV", n, n)
    H, So = plan.execute(S, h, eri)
    assert H.shape == (429, 429)
    ex_o = O.expand(O.generate_structures("COV", n, n), n)
    Hr, Sr, done = O.structure_matrices(n, ex_o, S, h, eri, threads=os.cpu_count() or 1)
    assert done == 3432 * 3433 // 2
    scale_h = max(1.0, np.abs(Hr).max())
    scale_s = max(1.0, np.abs(Sr).max())
    assert np.abs(H - Hr).max() <= REL * scale_h
    assert np.abs(So - Sr).max() <= REL * scale_s
    assert np.array_equal(H, H.T)
    assert np.linalg.eigvalsh(So).min() > 0
    H1, S1 = plan.execute(S, h, np.zeros_like(eri))
    H2, S2 = plan.execute(S, np.zeros_like(h), eri)
    assert np.array_equal(S1, So) and np.array_equal(S2, So)
    assert np.abs(H1 + H2 - H).max() <= 1e-12 * scale_h


@pytest.mark.parametrize("kw,n,nel", [("COV", 8, 6), ("COV", 10, 8), ("COV ION(1)", 6, 2), ("COV", 5, 2),
                                      ("FULL", 5, 4), ("COV ION(1)", 7, 6)])
def test_more_orbitals_than_electrons(ctx, kw, n, nel):
    """Active spaces with n > 2k (complements larger than the strings): every excitation level
    from 0 to min(k, n - k) occurs in the frame kernel."""
    S, h, eri = workloads.active_space(n, 3 * n, 40 + n + nel)
    plan, ex = _plan(ctx, kw, n, nel)
    H, So = plan.execute(S, h, eri)
    Hr, Sr, _ = O.structure_matrices(n, ex, S, h, eri)
    assert _rel(H, Hr) < REL and _rel(So, Sr) < REL


@pytest.mark.parametrize("n,k", [(3, 1), (6, 2), (7, 3), (8, 4), (9, 5), (10, 6), (10, 7), (11, 8), (9, 8)])
def test_spin_pair_records_every_electron_count(n, k):
    """Every spin pair of a complete string table (det, one-electron and total same-spin energy,
    nullity) against the oracle for k = 1 .. 8, through the allocation-free entry point (which
    returns the record scalars of the same kernels); one random and one stretched overlap."""
    import itertools

    import torch

    masks = sorted(sum(1 << o for o in occ) for occ in itertools.combinations(range(n), k))
    N = len(masks)
    n_pairs = N * (N + 1) // 2
    occ = [[o for o in range(n) if (m >> o) & 1] for m in masks]
    S0, h, eri = workloads.active_space(n, 2 * n, 90 + 10 * n + k)
    idx = np.arange(n)
    S1 = np.exp(-0.8 * np.abs(idx[:, None] - idx[None, :]))  # overlaps decaying along a chain
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(n * 100 + k)
    sample = rng.choice(n_pairs, size=min(n_pairs, 3000), replace=False)
    for S in (S0, S1):
        d_masks = torch.tensor(np.array(masks, dtype=np.uint64).view(np.int64), device=dev)
        dS = torch.tensor(np.ascontiguousarray(S.T), device=dev)
        dh = torch.tensor(np.ascontiguousarray(h.T), device=dev)
        de = torch.tensor(eri, device=dev)
        out = torch.full((4 * n_pairs,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        vbcore.spin_pairs_noalloc(torch.cuda.current_stream(dev).cuda_stream, n, k, N, d_masks.data_ptr(),
                                  dS.data_ptr(), dh.data_ptr(), de.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(n_pairs, 4)
        uu = np.repeat(np.arange(N), np.arange(N, 0, -1))
        vv = np.concatenate([np.arange(u, N) for u in range(N)])
        for t in sample:
            ref = O.spin_pair(n, occ[uu[t]], occ[vv[t]], S, h, eri)
            assert int(got[t, 3]) == ref["nullity"]
            for col, key in ((0, "det"), (1, "h1"), (2, "htot")):
                assert abs(got[t, col] - ref[key]) <= REL * max(1.0, abs(ref[key])), (n, k, t, key)


def test_band_reduction_wait_timeout_is_reported_and_the_plan_recovers():
    """The band reduction's tile waits are bounded: with a one-poll limit the first wait gives up,
    the CTAs flag it and leave after their copies in flight land, and the execute returns
    VB_ERR_TIMEOUT (no trap, no hang); with the default limit restored the same plan evaluates
    the structure matrices."""
    n = 8
    S, h, eri = workloads.active_space(n, 3 * n, 21)
    c = vbcore.Context(0)
    try:
        plan, ex = _plan(c, "COV", n, n)
        c.set_barrier_spin_limit(1)
        with pytest.raises(vbcore.VbError) as e:
            plan.execute(S, h, eri)
        assert e.value.status == 6 and "band_reduce" in str(e.value)
        c.set_barrier_spin_limit(0)
        H, So = plan.execute(S, h, eri)
        Hr, Sr, _ = O.structure_matrices(n, ex, S, h, eri)
        assert _rel(H, Hr) < REL and _rel(So, Sr) < REL
        plan.close()
    finally:
        c.close()
