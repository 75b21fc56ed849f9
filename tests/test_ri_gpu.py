"""RI AO -> active transform on the device against the oracle (transform_ri_active_integrals,
src/integrals/active/ri.cpp:33-96), including the one-index factors and the adjoint."""

import numpy as np
import pytest

import oracle as O
import vbcore

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = vbcore.Context(0)
    yield c
    c.close()


def _inputs(n_aux, n_bf, n_act, seed, decay=None):
    rng = np.random.default_rng(seed)
    npair = n_bf * (n_bf + 1) // 2
    B = rng.standard_normal((n_aux, npair))
    if decay:
        idx = np.array([(m, v) for m in range(n_bf) for v in range(m + 1)])
        B *= np.exp(-np.abs(idx[:, 0] - idx[:, 1]) / decay)[None, :]
    C = rng.standard_normal((n_bf, n_act)) / np.sqrt(n_bf)
    return B, C


def _rel(a, b):
    return np.abs(a - b).max() / max(1e-300, np.abs(b).max())


@pytest.mark.parametrize("n_aux,n_bf,n_act", [(1, 1, 1), (10, 7, 3), (37, 20, 6), (129, 50, 1), (130, 33, 16),
                                              (300, 64, 16), (257, 300, 8)])
def test_transform_matches_oracle(ctx, n_aux, n_bf, n_act):
    B, C = _inputs(n_aux, n_bf, n_act, n_aux + n_bf + n_act)
    L, K, T = vbcore.active_transform_ri(ctx, B, C, one_index=True)
    Lr, Kr = O.ri_transform(B, C)
    assert _rel(L, Lr) < 1e-13
    assert _rel(K, Kr) < 1e-13
    if n_aux * n_bf * n_bf <= 300 * 64 * 64:
        assert _rel(T, O.ri_one_index(B, C)) < 1e-13


@pytest.mark.parametrize("n_aux,n_bf,n_act", [(10, 7, 3), (130, 33, 16), (64, 100, 5)])
def test_adjoint_matches_oracle_and_differences(ctx, n_aux, n_bf, n_act):
    B, C = _inputs(n_aux, n_bf, n_act, 5)
    L, _, T = vbcore.active_transform_ri(ctx, B, C, one_index=True)
    rng = np.random.default_rng(6)
    G = rng.standard_normal(L.shape)
    dC = vbcore.active_transform_ri_adjoint(ctx, T, G, n_bf)
    assert _rel(dC, O.ri_adjoint(T, G, n_act)) < 1e-12
    D = rng.standard_normal(C.shape)
    h = 1e-3
    fp = np.sum(G * vbcore.active_transform_ri(ctx, B, C + h * D)[0])
    fm = np.sum(G * vbcore.active_transform_ri(ctx, B, C - h * D)[0])
    assert abs((fp - fm) / (2 * h) - np.sum(dC * D)) < 1e-8 * max(1.0, abs(np.sum(dC * D)))


def test_full_size_precision_workload(ctx):
    # n_bf 400, n_aux 1600, n_act 16 with |mu - nu| decay 20: every output against the oracle
    # on a slice of auxiliary rows (L and its rows are independent per auxiliary function),
    # plus size-independent properties of the whole result
    n_aux, n_bf, n_act = 1600, 400, 16
    B, C = _inputs(n_aux, n_bf, n_act, 20261203, decay=20.0)
    L, K, _ = vbcore.active_transform_ri(ctx, B, C)
    rows = np.arange(0, n_aux, 25)
    Lr, _ = O.ri_transform(B[rows], C)
    assert _rel(L[rows], Lr) < 1e-13
    P = n_act * (n_act + 1) // 2
    Kfull = np.zeros((P, P))
    iu = np.tril_indices(P)
    Kfull[iu] = K
    Kfull = Kfull + np.tril(Kfull, -1).T
    assert _rel(Kfull, L.T @ L) < 1e-13
    # linearity in B
    L2, _, _ = vbcore.active_transform_ri(ctx, 2.0 * B, C)
    assert np.array_equal(L2, 2.0 * L)


# Split precision: the one-index step as three-way BF16 splits on the tensor cores with FP32
# accumulation and FP64 recombination.  Bar: 1e-6 relative to the largest element for the
# one-index factors and L, 2e-6 for K = L^T L (FP32-level: each operand keeps about 24 bits).
SPLIT_REL = 1e-6


@pytest.mark.parametrize("n_aux,n_bf,n_act", [(1, 1, 1), (10, 7, 3), (37, 20, 6), (129, 50, 1), (130, 33, 16),
                                              (300, 64, 16), (257, 300, 8)])
def test_split_precision_transform(ctx, n_aux, n_bf, n_act):
    B, C = _inputs(n_aux, n_bf, n_act, 3 * n_aux + n_bf + n_act)
    L, K, T = vbcore.active_transform_ri(ctx, B, C, one_index=True, precision="bf16x3")
    Lr, Kr = O.ri_transform(B, C)
    assert _rel(L, Lr) < SPLIT_REL
    assert _rel(K, Kr) < 2 * SPLIT_REL
    if n_aux * n_bf * n_bf <= 300 * 64 * 64:
        assert _rel(T, O.ri_one_index(B, C)) < SPLIT_REL
    # and agrees with the FP64 path to the same bar
    L64, _, _ = vbcore.active_transform_ri(ctx, B, C)
    assert _rel(L, L64) < SPLIT_REL


def test_split_precision_full_size(ctx):
    n_aux, n_bf, n_act = 1600, 400, 16
    B, C = _inputs(n_aux, n_bf, n_act, 20261203, decay=20.0)
    L64, K64, T64 = vbcore.active_transform_ri(ctx, B, C, one_index=True)
    L, K, T = vbcore.active_transform_ri(ctx, B, C, one_index=True, precision="bf16x3")
    assert _rel(T, T64) < SPLIT_REL
    assert _rel(L, L64) < SPLIT_REL
    assert _rel(K, K64) < 2 * SPLIT_REL


def test_rejects_too_many_active_orbitals(ctx):
    B, C = _inputs(4, 20, 17, 1)
    with pytest.raises(vbcore.VbError) as e:
        vbcore.active_transform_ri(ctx, B, C)
    assert e.value.status == 5


@pytest.mark.parametrize("n,n_aux", [(1, 3), (6, 40), (14, 42), (16, 257)])
def test_pair_factors_in_a_new_frame(ctx, n, n_aux):
    """transform_ri_pair_factors and its two directional forms (ri_transform.cpp:98-211) against
    the oracle, a non-orthogonal frame; the raw direction against a central difference of the
    forward transform, and the orthogonal form against the raw one with dQ = -Q K."""
    rng = np.random.default_rng(n * 1000 + n_aux)
    npair = n * (n + 1) // 2
    B = rng.standard_normal((n_aux, npair))
    dB = rng.standard_normal((n_aux, npair))
    Q = np.eye(n) + 0.3 * rng.standard_normal((n, n))
    dQ = rng.standard_normal((n, n))
    K = rng.standard_normal((n, n))
    fwd = vbcore.ri_pair_factors_frame(ctx, B, Q)
    ref = O.ri_pair_factors_frame(B, Q)
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(fwd - ref).max() <= 1e-13 * scale
    raw = vbcore.ri_pair_factors_frame(ctx, B, Q, mode=1, factor_direction=dB, frame_direction=dQ)
    assert np.abs(raw - O.ri_pair_factors_frame(B, Q, 1, dB, dQ)).max() <= 1e-13 * max(1.0, np.abs(raw).max())
    # the transform is cubic along the line (B + t dB, Q + t dQ): Richardson's combination of two
    # central differences is exact for a cubic up to rounding
    def central(h):
        return (O.ri_pair_factors_frame(B + h * dB, Q + h * dQ) - O.ri_pair_factors_frame(B - h * dB, Q - h * dQ)) / (2 * h)

    fd = (4.0 * central(5e-4) - central(1e-3)) / 3.0
    assert np.abs(raw - fd).max() <= 1e-9 * max(1.0, np.abs(fd).max())
    orth = vbcore.ri_pair_factors_frame(ctx, fwd, Q, mode=2, factor_direction=dB, frame_direction=K)
    via_raw = vbcore.ri_pair_factors_frame(ctx, B, Q, mode=1, factor_direction=dB, frame_direction=-Q @ K)
    assert np.abs(orth - via_raw).max() <= 1e-12 * max(1.0, np.abs(via_raw).max())


def test_pair_factors_frame_rejects_bad_input(ctx):
    with pytest.raises(vbcore.VbError):
        vbcore.ri_pair_factors_frame(ctx, np.zeros((2, 3)), np.eye(2), mode=1)
