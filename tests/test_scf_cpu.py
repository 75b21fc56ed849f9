"""Host-side pieces of the VBSCF solver that need no GPU: AO integrals of s shells against the
oracle's restatement, and the hydrogen-chain inputs."""

import numpy as np

import oracle as O
import vbcore
from vbcore import molecules


def _shells(mol):
    offs = np.concatenate([[0], np.cumsum(mol.shell_nprim)[:-1]])
    return [(int(a), mol.shell_exponents[o:o + n], mol.shell_coefficients[o:o + n])
            for a, n, o in zip(mol.shell_atom, mol.shell_nprim, offs)]


def test_ao_integrals_match_oracle():
    for n_atoms, seed in ((2, 0), (4, 3), (6, 1)):
        mol = molecules.h_chain(n_atoms, seed=seed)
        S, h, eri, enuc = vbcore.ao_integrals_s(mol)
        Sr, hr, erir, enr = O.s_shell_integrals(mol.charges, mol.coords, _shells(mol))
        assert np.abs(S - Sr).max() < 1e-14 and np.abs(h - hr).max() < 1e-13
        assert np.abs(eri - erir).max() < 1e-13 and abs(enuc - enr) < 1e-13
        assert np.allclose(np.diag(S), 1.0, atol=1e-14)
        # 8-fold permutational symmetry of the repulsion integrals
        assert np.array_equal(eri, eri.transpose(1, 0, 2, 3)) and np.array_equal(eri, eri.transpose(2, 3, 0, 1))


def test_h2_known_values():
    # H2 at 1.4 bohr with one normalized 1s-like primitive: overlap exp(-a b / (a + b) R^2) (2 sqrt(ab) / (a + b))^1.5
    mol = molecules.Molecule(np.ones(2), np.array([[0, 0, 0], [0, 0, 1.4]], float), np.array([0, 1], np.int32),
                             np.array([1, 1], np.int32), np.array([0.5, 0.8]), np.array([1.0, 1.0]))
    S, h, eri, enuc = vbcore.ao_integrals_s(mol)
    a, b, R = 0.5, 0.8, 1.4
    expect = (2 * np.sqrt(a * b) / (a + b)) ** 1.5 * np.exp(-a * b / (a + b) * R * R)
    assert abs(S[0, 1] - expect) < 1e-15
    assert abs(enuc - 1 / 1.4) < 1e-15
    # one-centre repulsion of a normalized s primitive: 2 sqrt(a / pi) ... (ss|ss) = sqrt(2 a / pi) * 2 / sqrt(2)
    assert abs(eri[0, 0, 0, 0] - 2.0 * np.sqrt(a / np.pi)) < 1e-14


def test_h_chain_geometry():
    mol = molecules.h_chain(6, spacing_angstrom=1.0, jitter_angstrom=0.05, seed=7)
    z = mol.coords[:, 2] / molecules.BOHR_PER_ANGSTROM
    assert np.all(np.abs(z - np.arange(6)) <= 0.05 + 1e-12)
    assert mol.n_basis == 12 and list(mol.shell_nprim) == [3, 1] * 6
