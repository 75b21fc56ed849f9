"""Batched and served work through the engine: every result is the same alone and in the
mix (energies to 1e-10 Eh for the batched instances, 1e-9 Eh for the served solves)."""

import numpy as np
import pytest

import oracle as O
import vbcore
from vbcore import molecules, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = vbcore.Context(0)
    yield c
    c.close()


def _instance(n, seed):
    S, h, _ = workloads.active_space(n, 3 * n, seed)
    rng = np.random.default_rng(seed)
    P = n * (n + 1) // 2
    F = 0.1 * rng.standard_normal((P, 3 * n))
    return S, h, workloads.pack_pair_kernel(F @ F.T), F


def test_batched_instances_match_single_evaluations(ctx):
    eng = vbcore.Engine(0, 0, workers=4)
    specs = [(4, 1), (6, 2), (8, 3), (4, 4), (6, 5), (8, 6), (6, 7), (4, 8)]
    ids, data, exps = [], [], []
    for n, seed in specs:
        rows = vbcore.generate_structures("COV ION(1)", n, n)
        ex = vbcore.expand_structures(rows, n)
        ids.append(eng.add_instance(ex, n))
        data.append(_instance(n, seed))
        exps.append(ex)
    E, G = eng.evaluate(ids, [d[0] for d in data], [d[1] for d in data], [d[2] for d in data], [d[3] for d in data])
    for (n, seed), ex, (S, h, eri, F), e, g in zip(specs, exps, data, E, G):
        plan = vbcore.HsPlan(ctx, ex, n)
        Hs, Ss = plan.execute(S, h, eri)
        w, C = vbcore.generalized_eigh(ctx, Hs, Ss)
        assert abs(e - w[0]) < 1e-10 * max(1.0, abs(w[0]))
        assert abs(e - O.generalized_eigh(Hs, Ss)[0][0]) < 1e-9 * max(1.0, abs(e))
        gr = plan.gradient(S, h, eri, C[:, 0], w[0], packed_eri=False, ri_factors=F)
        assert np.abs(g["S"] - gr["S"]).max() < 1e-9 * max(1.0, np.abs(gr["S"]).max())
        assert np.abs(g["ri"] - gr["ri"]).max() < 1e-9 * max(1.0, np.abs(gr["ri"]).max())
        plan.close()
    eng.close()


def test_served_solves_same_alone_and_in_the_mix():
    eng = vbcore.Engine(0, 0, workers=4)
    reqs = []
    for tag, (n, spacing, seed) in enumerate([(4, 0.9, 1), (6, 1.2, 2), (4, 1.6, 3), (6, 0.8, 4), (8, 1.0, 5),
                                              (4, 2.5, 6)]):
        mol = molecules.h_chain(n, spacing, 0.05, seed=seed)
        pat = molecules.hao_pattern(mol, n)
        reqs.append((mol, pat, n, molecules.hao_guess(mol, pat)))
    for tag, (mol, pat, n, C0) in enumerate(reqs):
        eng.submit_scf(mol, pat, n, C0, gradient_tolerance=1e-7, tag=tag)
    mixed = {}
    while len(mixed) < len(reqs):
        for r in eng.poll(wait=True):
            assert r["status"] == 0 and r["converged"], r
            mixed[r["tag"]] = r
    for tag, (mol, pat, n, C0) in enumerate(reqs):
        eng.submit_scf(mol, pat, n, C0, gradient_tolerance=1e-7, tag=100 + tag)
        alone = eng.poll(wait=True)
        assert len(alone) == 1 and alone[0]["tag"] == 100 + tag
        assert abs(alone[0]["energy"] - mixed[tag]["energy"]) < 1e-9
    eng.close()
