"""Molecular inputs for the VBSCF solver: hydrogen chains in the 6-31G basis.

The 6-31G hydrogen shells are the published basis-set values (the reference ships them in
basis/6-31g.gbs:25-32): one contracted s shell of three primitives and one of a single
primitive per atom.  Coordinates are in bohr.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BOHR_PER_ANGSTROM = 1.0 / 0.529177210903  # CODATA 2018 Bohr radius

H_631G = (
    ((18.7311370, 2.8253937, 0.6401217), (0.03349460, 0.23472695, 0.81375733)),
    ((0.1612778,), (1.0,)),
)


@dataclass
class Molecule:
    charges: np.ndarray          # [n_atoms]
    coords: np.ndarray           # [n_atoms, 3], bohr
    shell_atom: np.ndarray       # [n_shells] int32
    shell_nprim: np.ndarray      # [n_shells] int32
    shell_exponents: np.ndarray  # concatenated
    shell_coefficients: np.ndarray

    @property
    def n_basis(self) -> int:
        return len(self.shell_atom)

    def atom_functions(self, atom: int) -> list[int]:
        return [i for i, a in enumerate(self.shell_atom) if a == atom]


def h_chain(n_atoms: int, spacing_angstrom: float = 1.0, jitter_angstrom: float = 0.05, seed: int = 0) -> Molecule:
    """Linear H_n along z: atom i at i * spacing plus a seeded uniform jitter in
    [-jitter, +jitter] (angstrom), 6-31G basis."""
    rng = np.random.default_rng(seed)
    z = np.arange(n_atoms) * spacing_angstrom + rng.uniform(-jitter_angstrom, jitter_angstrom, n_atoms)
    coords = np.zeros((n_atoms, 3))
    coords[:, 2] = z * BOHR_PER_ANGSTROM
    sa, sn, ex, co = [], [], [], []
    for a in range(n_atoms):
        for exps, coefs in H_631G:
            sa.append(a)
            sn.append(len(exps))
            ex.extend(exps)
            co.extend(coefs)
    return Molecule(np.ones(n_atoms), coords, np.array(sa, np.int32), np.array(sn, np.int32), np.array(ex),
                    np.array(co))


def hao_pattern(mol: Molecule, n_active: int) -> list[list[int]]:
    """One active orbital per atom over that atom's basis functions (the deck's $FRAG pattern)."""
    return [mol.atom_functions(a) for a in range(n_active)]


def hao_guess(mol: Molecule, pattern: list[list[int]]) -> np.ndarray:
    """Initial coefficients [n_basis, n_active]: equal weights on each orbital's functions."""
    C = np.zeros((mol.n_basis, len(pattern)))
    for a, funcs in enumerate(pattern):
        for i, m in enumerate(funcs):
            C[m, a] = 0.7 if i == 0 else 0.4
    return C
