"""Generate the golden structure-matrix fixtures under tests/golden/.

The reference (Tao-Xia/xmvb-cpp) pins its structure Hamiltonian/overlap with an
independent calculation in an orthonormal carrier basis
(tests/vbscf/unit/test_structure_tiles.cpp:245-307, 426-487: orthonormalize the
active orbitals, act with a direct-CI Hamiltonian, map back through the
structure expansion; tolerance 2e-10 on H and 2e-11 on S).  This script does
the same independently of any Loewdin/cofactor algebra:

* orthonormal orbitals chi = phi L^{-T} from S = L L^T; integrals transformed;
* the second-quantized Hamiltonian H = sum h E + 1/2 sum (pq|rs)(E E - delta E)
  is built in the fixed (N_alpha, N_beta) Jordan-Wigner sector;
* every nonorthogonal determinant |alpha occ, beta occ> (alpha creators first,
  ascending orbitals: the reference determinant convention) is built by applying
  b_i^+ = sum_a L_ia a_a^+ to the vacuum;
* H_de = <d|H|e>, S_de = <d|e>, and H_IJ = sum c_dI c_eJ H_de through the
  expansion of the oracle's restated structure generator.

The input fixture "reference_fixture" restates make_fixture() of
test_structure_tiles.cpp:179-227.  Run: python tests/golden/make_golden.py
"""

from __future__ import annotations

import itertools
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def pair_index(a, b):
    hi, lo = (a, b) if a > b else (b, a)
    return hi * (hi + 1) // 2 + lo


def reference_fixture(n):
    """test_structure_tiles.cpp:179-227 (make_fixture)."""
    upper = np.eye(n)
    for j in range(n):
        for i in range(j):
            upper[i, j] = 0.004 * math.cos(0.31 * (i + 2) * (j + 1))
    S = upper.T @ upper
    h = np.zeros((n, n))
    for j in range(n):
        for i in range(j + 1):
            v = -0.8 + 0.06 * i if i == j else 0.015 * math.sin(0.19 * (i + 1) * (j + 3))
            h[i, j] = h[j, i] = v
    npair = n * (n + 1) // 2
    factor = np.zeros((4, npair))
    for j in range(npair):
        for i in range(4):
            factor[i, j] = 0.018 * math.cos(0.13 * (i + 2) * (j + 1))
    kernel = factor.T @ factor
    packed = np.zeros(npair * (npair + 1) // 2)
    for j in range(npair):
        for i in range(j + 1):
            packed[pair_index(i, j)] = kernel[i, j]
    return S, h, packed


def random_fixture(n, n_aux, seed):
    """Seeded synthetic active space with the shapes and distributions of the
    determinant-pair microbenchmark: unit-diagonal S with 0.3 N(0,1)/sqrt(n)
    off-diagonals (eigenvalues floored at 1e-3), symmetric N(0,1) h, and
    (ij|kl) = sum_P B_ij^P B_kl^P with B ~ N(0, 0.1) symmetrized over ij."""
    rng = np.random.default_rng(seed)
    a = 0.3 * rng.standard_normal((n, n)) / math.sqrt(n)
    a = 0.5 * (a + a.T)
    np.fill_diagonal(a, 0.0)
    w, q = np.linalg.eigh(np.eye(n) + a)
    S = (q * np.maximum(w, 1e-3)) @ q.T
    S = 0.5 * (S + S.T)
    g = rng.standard_normal((n, n))
    h = 0.5 * (g + g.T)
    B = 0.1 * rng.standard_normal((n_aux, n, n))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    npair = n * (n + 1) // 2
    Lf = np.zeros((n_aux, npair))
    for i in range(n):
        for j in range(i + 1):
            Lf[:, pair_index(i, j)] = B[:, i, j]
    K = Lf.T @ Lf
    packed = np.zeros(npair * (npair + 1) // 2)
    for p in range(npair):
        for q2 in range(p + 1):
            packed[pair_index(p, q2)] = K[p, q2]
    return S, h, packed


# ------------------------------------------------------------------------------------------
# Jordan-Wigner sector machinery


def sector_basis(n, na, nb):
    states = []
    for A in itertools.combinations(range(n), na):
        for Bs in itertools.combinations(range(n), nb):
            s = 0
            for a in A:
                s |= 1 << a
            for b in Bs:
                s |= 1 << (n + b)
            states.append(s)
    return states, {s: i for i, s in enumerate(states)}


def jw_annihilate(s, p):
    if not (s >> p) & 1:
        return None, 0
    sign = -1 if bin(s & ((1 << p) - 1)).count("1") & 1 else 1
    return s & ~(1 << p), sign


def jw_create(s, p):
    if (s >> p) & 1:
        return None, 0
    sign = -1 if bin(s & ((1 << p) - 1)).count("1") & 1 else 1
    return s | (1 << p), sign


def spin_summed_excitations(n, states, index):
    dim = len(states)
    E = np.zeros((n, n, dim, dim))
    for col, s in enumerate(states):
        for sigma in (0, 1):
            off = sigma * n
            for q in range(n):
                t, s1 = jw_annihilate(s, q + off)
                if t is None:
                    continue
                for p in range(n):
                    u, s2 = jw_create(t, p + off)
                    if u is None:
                        continue
                    E[p, q, index[u], col] += s1 * s2
    return E


def fock_vector(n, L, alpha_occ, beta_occ, index):
    """b^+_{alpha...} b^+_{beta...}|0> with b_i^+ = sum_a L[i, a] a_a^+ (alpha creators leftmost)."""
    vec = {0: 1.0}
    creators = [(i, 0) for i in alpha_occ] + [(j, n) for j in beta_occ]
    for orb, off in reversed(creators):
        nxt = {}
        for s, c in vec.items():
            for a in range(n):
                coeff = L[orb, a]
                if coeff == 0.0:
                    continue
                t, sg = jw_create(s, a + off)
                if t is None:
                    continue
                nxt[t] = nxt.get(t, 0.0) + sg * coeff * c
        vec = nxt
    out = np.zeros(len(index))
    for s, c in vec.items():
        out[index[s]] += c
    return out


def independent_matrices(n, S, h, packed, exp):
    L = np.linalg.cholesky(S)  # S = L L^T; phi_i = sum_a chi_a L[i, a]
    Linv = np.linalg.inv(L)
    g = O.unpack_eri(packed, n)
    hp = Linv @ h @ Linv.T
    gp = np.einsum("pa,qb,rc,sd,abcd->pqrs", Linv, Linv, Linv, Linv, g, optimize=True)
    states, index = sector_basis(n, exp.n_alpha, exp.n_beta)
    E = spin_summed_excitations(n, states, index)
    M = np.einsum("pqrs,rsij->pqij", gp, E, optimize=True)
    H = np.einsum("pq,pqij->ij", hp, E)
    H += 0.5 * np.einsum("pqij,pqjk->ik", E, M, optimize=True)
    H -= 0.5 * np.einsum("pqqs,psij->ij", gp, E, optimize=True)
    vecs = np.array([fock_vector(n, L, exp.det_alpha_occ[d], exp.det_beta_occ[d], index)
                     for d in range(exp.n_determinants)])
    Hd = vecs @ H @ vecs.T
    Sd = vecs @ vecs.T
    T = exp.coefficient_matrix()
    return Hd, Sd, T.T @ Hd @ T, T.T @ Sd @ T


CASES = [
    # name, n_orb, n_el, mult, keyword, fixture
    ("rumer_n4", 4, 4, 1, "COV", ("reference", None)),
    ("rumer_n6", 6, 6, 1, "COV", ("reference", None)),
    ("ionic_n4", 4, 4, 1, "COV ION(1)", ("reference", None)),
    ("ionic_n6", 6, 6, 1, "COV ION(1)", ("reference", None)),
    ("orthogonal_n4", 4, 4, 1, "FULL", ("orthogonal", None)),
    ("orthogonal_n6", 6, 6, 1, "COV ION(1)", ("orthogonal", None)),
    ("triplet_n5", 5, 4, 3, "COV", ("reference", None)),
    ("random_n6", 6, 6, 1, "COV", ("random", 20260101)),
    ("random_n8", 8, 8, 1, "COV", ("random", 20260102)),
]


def make_case(name, n, n_el, mult, keyword, fixture):
    kind, seed = fixture
    if kind == "reference":
        S, h, packed = reference_fixture(n)
    elif kind == "orthogonal":
        _, h, packed = reference_fixture(n)
        S = np.eye(n)
    else:
        S, h, packed = random_fixture(n, 3 * n, seed)
    structures = O.generate_structures(keyword, n, n_el, mult)
    exp = O.expand(structures, n_el, mult)
    Hd, Sd, Hs, Ss = independent_matrices(n, S, h, packed, exp)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez(path, n=n, n_el=n_el, mult=mult, keyword=keyword, S=S, h=h, eri=packed,
             structures=np.array(structures, dtype=np.int32), Hd=Hd, Sd=Sd, Hs=Hs, Ss=Ss)
    return path, exp.n_structures, exp.n_determinants


def main():
    meta = {}
    for case in CASES:
        path, ns, nd = make_case(*case)
        meta[case[0]] = dict(n_structures=ns, n_determinants=nd, keyword=case[4], n_orb=case[1],
                             n_el=case[2], mult=case[3], fixture=case[5][0])
        print(f"{case[0]}: {ns} structures, {nd} determinants -> {os.path.basename(path)}")
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
