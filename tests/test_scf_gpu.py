"""Plain VBSCF on the device against the oracle: linear H6 (1.00 A spacing, seeded +-0.05 A
jitter), 6-31G, 6 electrons in 6 HAO-local active orbitals, singlet, the 5 covalent Rumer
structures over 20 determinants.  Parity bar: structure H/S 1e-10 relative, energy 1e-9 Eh,
orbital gradient 1e-7."""

import numpy as np
import pytest

import oracle as O
import vbcore
from vbcore import molecules

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = vbcore.Context(0)
    yield c
    c.close()


def _shells(mol):
    offs = np.concatenate([[0], np.cumsum(mol.shell_nprim)[:-1]])
    return [(int(a), mol.shell_exponents[o:o + n], mol.shell_coefficients[o:o + n])
            for a, n, o in zip(mol.shell_atom, mol.shell_nprim, offs)]


@pytest.fixture(scope="module")
def h6():
    mol = molecules.h_chain(6, 1.0, 0.05, seed=20261203)
    pattern = molecules.hao_pattern(mol, 6)
    oracle = O.VbscfOracle(mol.charges, mol.coords, _shells(mol), pattern, 6)
    return mol, pattern, oracle


def test_energy_gradient_and_matrices_at_identical_orbitals(ctx, h6):
    mol, pattern, oracle = h6
    prob = vbcore.ScfProblem(ctx, mol, pattern, 6)
    assert prob.n_structures == 5 and prob.n_basis == 12
    rng = np.random.default_rng(1)
    C = molecules.hao_guess(mol, pattern)
    for trial in range(2):
        E, G, Hs, Ss = prob.energy_gradient(C, with_matrices=True)
        Hr, Sr = oracle.matrices(C)
        assert np.abs(Hs - Hr).max() <= 1e-10 * np.abs(Hr).max()
        assert np.abs(Ss - Sr).max() <= 1e-10 * np.abs(Sr).max()
        assert abs(E - oracle.energy(C)) < 1e-9
        Gr = oracle.gradient(C)
        assert np.abs(G - Gr).max() < 1e-7
        # perturbed orbitals inside the pattern
        mask = np.zeros_like(C)
        for a, funcs in enumerate(pattern):
            mask[funcs, a] = 1.0
        C = C + 0.1 * rng.standard_normal(C.shape) * mask
    prob.close()


def test_solve_converges_to_the_oracle_minimum(ctx, h6):
    mol, pattern, oracle = h6
    prob = vbcore.ScfProblem(ctx, mol, pattern, 6)
    C0 = molecules.hao_guess(mol, pattern)
    res, C = prob.solve(C0, max_iterations=300, gradient_tolerance=1e-7)
    assert res["converged"], res
    Er, Cr, _ = oracle.solve(C0, gtol=1e-9)
    assert abs(res["energy"] - Er) < 1e-9, (res["energy"], Er)
    assert abs(res["energy"] - oracle.energy(C)) < 1e-9
    # orbital gradient at the solution, against the oracle's differences
    E, G = prob.energy_gradient(C)
    assert np.abs(G - oracle.gradient(C)).max() < 1e-7
    assert np.abs(G).max() < 1e-6
    prob.close()


def test_split_precision_solve_reaches_the_fp64_minimum(ctx, h6):
    """The split-precision RI transform layered onto the solve: split-precision evaluations while
    the gradient is above the switch, then an FP64 finish, so the converged energy is the FP64
    solve's (1e-9 Eh) and the split evaluations did part of the work."""
    mol, pattern, oracle = h6
    C0 = molecules.hao_guess(mol, pattern)
    ref = vbcore.ScfProblem(ctx, mol, pattern, 6)
    r64, C64 = ref.solve(C0, max_iterations=300, gradient_tolerance=1e-7)
    ref.close()
    prob = vbcore.ScfProblem(ctx, mol, pattern, 6)
    prob.set_precision("bf16x3", 1e-4)
    res, C = prob.solve(C0, max_iterations=300, gradient_tolerance=1e-7)
    assert res["converged"], res
    assert res["split_evaluations"] > 0 and res["split_evaluations"] < res["evaluations"]
    assert abs(res["energy"] - r64["energy"]) < 1e-9, (res["energy"], r64["energy"])
    assert abs(res["energy"] - oracle.energy(C)) < 1e-9
    # the FP64 evaluation path is restored after the solve
    E, G = prob.energy_gradient(C)
    assert abs(E - res["energy"]) < 1e-12 and np.abs(G).max() < 1e-6
    with pytest.raises(vbcore.VbError):
        prob.set_precision("bf16x3", -1.0)
    prob.close()


@pytest.mark.parametrize("threshold", [0.0, 1e-12])
def test_integral_input_matches_shell_input(ctx, h6, threshold):
    """The problem built from AO integrals the caller already has (an AO pair graph's unique
    integral stream, the reference solve_scf's input) evaluates the same energy and gradient as
    the problem that computes its own integrals, and converges to the same minimum."""
    mol, pattern, oracle = h6
    a = vbcore.ScfProblem(ctx, mol, pattern, 6)
    S, h, eri, enuc = vbcore.ao_integrals_s(mol)
    ints = dict(S_ao=S, h_ao=h, nuclear_repulsion=enuc, **vbcore.ao_pair_graph(eri, threshold))
    b = vbcore.ScfProblem(ctx, None, pattern, 6, integrals=ints)
    assert (b.n_basis, b.n_active, b.n_structures) == (a.n_basis, a.n_active, a.n_structures)
    assert b.nuclear_repulsion == a.nuclear_repulsion
    tol = 1e-12 if threshold == 0.0 else 1e-10
    C = molecules.hao_guess(mol, pattern)
    rng = np.random.default_rng(5)
    mask = np.zeros_like(C)
    for o, funcs in enumerate(pattern):
        mask[funcs, o] = 1.0
    for _ in range(2):
        Ea, Ga = a.energy_gradient(C)
        Eb, Gb = b.energy_gradient(C)
        assert abs(Ea - Eb) < tol
        assert np.abs(Ga - Gb).max() < 100 * tol
        C = C + 0.05 * rng.standard_normal(C.shape) * mask
    C0 = molecules.hao_guess(mol, pattern)
    ra, _ = a.solve(C0, gradient_tolerance=1e-7)
    rb, _ = b.solve(C0, gradient_tolerance=1e-7)
    assert ra["converged"] and rb["converged"]
    assert abs(ra["energy"] - rb["energy"]) < 1e-9
    a.close()
    b.close()
