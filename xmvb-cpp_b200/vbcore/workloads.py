"""Seeded synthetic inputs with the shapes and distributions of the benchmark workloads.

No public benchmark data is involved: every workload is generated here from a seed.

* ``active_space``: the determinant-pair microbenchmark's active space (n_active orbitals,
  unit-diagonal overlap with 0.3 N(0,1)/sqrt(n) off-diagonals made positive definite by an
  eigenvalue floor of 1e-3, symmetric N(0,1) one-electron integrals, and
  (ij|kl) = sum_P B_ij^P B_kl^P with B ~ N(0, 0.1) of shape [n_aux, n, n] symmetrized over ij,
  stored in the packed pair-of-pairs layout).
"""

from __future__ import annotations

import math

import numpy as np


def pair_index(a: int, b: int) -> int:
    hi, lo = (a, b) if a > b else (b, a)
    return hi * (hi + 1) // 2 + lo


def pack_pair_kernel(K: np.ndarray) -> np.ndarray:
    """Dense symmetric P x P pair kernel -> packed P(P+1)/2 storage (pair-of-pairs index)."""
    P = K.shape[0]
    iu = np.tril_indices(P)
    # packed[hi*(hi+1)/2 + lo] for hi >= lo; tril_indices enumerates rows (hi) then cols (lo)
    return np.ascontiguousarray(K[iu[0], iu[1]])


def ri_factor_to_packed(B: np.ndarray) -> np.ndarray:
    """B [n_aux, n, n] (symmetric in the last two) -> packed (ij|kl) = sum_P B_ij^P B_kl^P."""
    n_aux, n, _ = B.shape
    rows, cols = np.tril_indices(n)  # rows >= cols: pair index rows*(rows+1)/2 + cols in order
    L = B[:, rows, cols]  # [n_aux, P]
    K = L.T @ L
    return pack_pair_kernel(K)


def active_space(n: int, n_aux: int, seed: int):
    """(S, h, eri_packed) for the determinant-pair microbenchmark distribution."""
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
    return S, h, ri_factor_to_packed(B)
