"""Python host mirror of the vbcore C ABI (include/vbcore.h).

The names follow the reference's (Tao-Xia/xmvb-cpp) interfaces for the determinant-pair
path: structure generation (``build_generated_raw_structures_from_structure_class``),
expansion (``StructureExpander::expand``), the structure H/S builder
(``FullDeterminantStructureHamiltonianOverlapBuilder::build``), overlap resolution
(``DeterminantOverlapResolver::resolve_matrix``) and same-spin pair evaluation
(``DeterminantPairEvaluator::evaluate_same_spin_pair``).  Errors raise ``VbError`` with the
library's message, as the reference raises ``std::invalid_argument`` / ``std::runtime_error``.

The numerical entry points run CUDA kernels only; there is no CPU path.  Loading the library
needs no GPU (structure generation and expansion are host work), but creating a ``Context``
on a machine without an sm_100 device raises.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "lib", "libvbcore.so")

VB_MEM_HOST = 0
VB_MEM_DEVICE = 1

_STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "HBM budget exceeded", 4: "numerical failure",
           5: "unsupported", 6: "timeout"}


class VbError(RuntimeError):
    def __init__(self, status: int, message: str, info: int = 0):
        super().__init__(f"vbcore {_STATUS.get(status, status)}: {message}")
        self.status = status
        self.info = info


class _ExpansionSizes(ctypes.Structure):
    _fields_ = [("n_structures", ctypes.c_int32), ("n_alpha_electrons", ctypes.c_int32),
                ("n_beta_electrons", ctypes.c_int32), ("n_alpha_strings", ctypes.c_int32),
                ("n_beta_strings", ctypes.c_int32), ("n_determinants", ctypes.c_int64),
                ("n_terms", ctypes.c_int64)]


class _Expansion(ctypes.Structure):
    _fields_ = [("n_orbitals", ctypes.c_int32), ("n_alpha_electrons", ctypes.c_int32),
                ("n_beta_electrons", ctypes.c_int32), ("n_alpha_strings", ctypes.c_int32),
                ("n_beta_strings", ctypes.c_int32), ("alpha_strings", ctypes.c_void_p),
                ("beta_strings", ctypes.c_void_p), ("n_determinants", ctypes.c_int64),
                ("det_alpha", ctypes.c_void_p), ("det_beta", ctypes.c_void_p), ("n_structures", ctypes.c_int32),
                ("term_offsets", ctypes.c_void_p), ("term_structure", ctypes.c_void_p),
                ("term_coefficient", ctypes.c_void_p)]


class _ScfInput(ctypes.Structure):
    _fields_ = [("n_atoms", ctypes.c_int32), ("charges", ctypes.c_void_p), ("coords", ctypes.c_void_p),
                ("n_shells", ctypes.c_int32), ("shell_atom", ctypes.c_void_p), ("shell_nprim", ctypes.c_void_p),
                ("shell_exponents", ctypes.c_void_p), ("shell_coefficients", ctypes.c_void_p),
                ("n_active", ctypes.c_int32), ("orbital_offsets", ctypes.c_void_p),
                ("orbital_functions", ctypes.c_void_p), ("n_electrons", ctypes.c_int32),
                ("multiplicity", ctypes.c_int32), ("structures", ctypes.c_char_p)]


class _ScfIntegralInput(ctypes.Structure):
    _fields_ = [("n_basis", ctypes.c_int32), ("S_ao", ctypes.c_void_p), ("h_ao", ctypes.c_void_p),
                ("n_pairs", ctypes.c_int64), ("pair_first", ctypes.c_void_p), ("pair_second", ctypes.c_void_p),
                ("n_integrals", ctypes.c_int64), ("integral_rows", ctypes.c_void_p),
                ("integral_columns", ctypes.c_void_p), ("integral_values", ctypes.c_void_p),
                ("nuclear_repulsion", ctypes.c_double), ("n_active", ctypes.c_int32),
                ("orbital_offsets", ctypes.c_void_p), ("orbital_functions", ctypes.c_void_p),
                ("n_electrons", ctypes.c_int32), ("multiplicity", ctypes.c_int32), ("structures", ctypes.c_char_p)]


class _ScfOptions(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_int32), ("gradient_tolerance", ctypes.c_double),
                ("history_size", ctypes.c_int32), ("armijo", ctypes.c_double)]


class _ScfResult(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("gradient_inf", ctypes.c_double), ("iterations", ctypes.c_int32),
                ("evaluations", ctypes.c_int32), ("converged", ctypes.c_int32)]


class _HsStats(ctypes.Structure):
    _fields_ = [("spin_pairs", ctypes.c_int64), ("careful_spin_pairs", ctypes.c_int64),
                ("determinant_pairs", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("factor_columns", ctypes.c_int64)]


# every symbol include/vbcore.h declares
EXPORTED_SYMBOLS = (
    "vb_context_create", "vb_context_destroy", "vb_context_set_stream", "vb_context_synchronize",
    "vb_context_set_barrier_spin_limit", "vb_last_error",
    "vb_context_memory", "vb_generate_structures", "vb_expand_structures", "vb_hs_plan_create",
    "vb_hs_plan_destroy", "vb_hs_plan_execute", "vb_hs_plan_stats", "vb_resolve_overlaps", "vb_same_spin_pairs",
    "vb_hs_plan_determinant_pairs", "vb_hs_plan_enable_phase_timing", "vb_hs_plan_phase_times",
    "vb_spin_pairs_noalloc", "vb_metric_cholesky", "vb_generalized_eigh", "vb_generalized_eigh_batched",
    "vb_active_transform_ri", "vb_active_transform_ri_precision", "vb_active_transform_ri_adjoint",
    "vb_hs_plan_gradient", "vb_hs_plan_root_gradient",
    "vb_lowest_root", "vb_engine_create", "vb_engine_destroy", "vb_engine_last_error", "vb_engine_add_instance",
    "vb_engine_evaluate_instances", "vb_engine_submit_scf", "vb_engine_poll", "vb_engine_pending",
    "vb_ao_integrals_s", "vb_scf_problem_create", "vb_scf_problem_create_from_integrals", "vb_scf_problem_destroy",
    "vb_scf_problem_sizes", "vb_scf_ao_integrals", "vb_scf_energy_gradient", "vb_solve_scf",
    "vb_scf_problem_set_precision", "vb_scf_problem_split_evaluations",
    "vb_autotune_report", "vb_autotune_clear", "vb_ri_pair_factors_frame",
)

PHASES = ("tables", "spin_pairs", "determinant_pairs", "band_reduce", "structure_reduce", "exact_pairs")

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libvbcore.so (raises when the extension has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise VbError(2, f"native library missing: {path} (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    c = ctypes
    P = c.c_void_p
    lib.vb_context_create.argtypes = [c.c_int, c.c_size_t, c.POINTER(P)]
    lib.vb_context_destroy.argtypes = [P]
    lib.vb_context_set_stream.argtypes = [P, P]
    lib.vb_context_synchronize.argtypes = [P]
    lib.vb_context_set_barrier_spin_limit.argtypes = [P, c.c_longlong]
    lib.vb_autotune_report.argtypes = [c.c_char_p, c.c_size_t, c.POINTER(c.c_size_t)]
    lib.vb_ri_pair_factors_frame.argtypes = [P, c.c_int, P, P, c.c_int, c.c_int, P, P, c.c_int, P]
    lib.vb_autotune_clear.argtypes = []
    lib.vb_last_error.argtypes = [P]
    lib.vb_last_error.restype = c.c_char_p
    lib.vb_context_memory.argtypes = [P, c.POINTER(c.c_size_t), c.POINTER(c.c_size_t)]
    lib.vb_generate_structures.argtypes = [c.c_char_p, c.c_int, c.c_int, c.c_int, c.c_int, c.POINTER(c.c_int64), P,
                                           c.c_int64]
    lib.vb_expand_structures.argtypes = [P, c.c_int64, c.c_int, c.c_int, c.c_int, c.POINTER(_ExpansionSizes)] + [P] * 7
    lib.vb_hs_plan_create.argtypes = [P, c.POINTER(_Expansion), c.POINTER(P)]
    lib.vb_hs_plan_destroy.argtypes = [P]
    lib.vb_hs_plan_execute.argtypes = [P, P, P, P, c.c_int, P, P]
    lib.vb_hs_plan_stats.argtypes = [P, c.POINTER(_HsStats)]
    lib.vb_hs_plan_determinant_pairs.argtypes = [P, P, P, P, c.c_int64, P, c.c_int, P, P]
    lib.vb_hs_plan_enable_phase_timing.argtypes = [P, c.c_int]
    lib.vb_hs_plan_phase_times.argtypes = [P, P, c.c_int]
    lib.vb_resolve_overlaps.argtypes = [P, c.c_int, c.c_int64, P, c.c_int, P, P, P]
    lib.vb_spin_pairs_noalloc.argtypes = [P, c.c_int, c.c_int, c.c_int, P, P, P, P, P]
    lib.vb_metric_cholesky.argtypes = [P, P, c.c_int, c.c_int, P, c.POINTER(c.c_int)]
    lib.vb_generalized_eigh.argtypes = [P, P, P, c.c_int, c.c_int, P, P, c.POINTER(c.c_int)]
    lib.vb_generalized_eigh_batched.argtypes = [P, c.c_int, P, P, P, P, c.c_int, P, P, P, P]
    lib.vb_engine_create.argtypes = [c.c_int, c.c_size_t, c.c_int, c.POINTER(P)]
    lib.vb_engine_destroy.argtypes = [P]
    lib.vb_engine_last_error.argtypes = [P]
    lib.vb_engine_last_error.restype = c.c_char_p
    lib.vb_engine_add_instance.argtypes = [P, c.POINTER(_Expansion), c.POINTER(c.c_int64)]
    lib.vb_engine_evaluate_instances.argtypes = [P, c.c_int, P, P, P, P, P, P, P, P, P, P]
    lib.vb_engine_submit_scf.argtypes = [P, c.POINTER(_ScfInput), P, c.POINTER(_ScfOptions), c.c_int64]
    lib.vb_engine_poll.argtypes = [P, c.c_int, c.c_int, P, P, P, P, P, P, P, P, c.POINTER(c.c_int)]
    lib.vb_engine_pending.argtypes = [P, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_size_t)]
    lib.vb_lowest_root.argtypes = [P, P, P, c.c_int, c.c_int, c.c_double, c.c_int, c.POINTER(c.c_double), P,
                                   c.POINTER(c.c_int)]
    lib.vb_ao_integrals_s.argtypes = [c.POINTER(_ScfInput), P, P, P, c.POINTER(c.c_double)]
    lib.vb_scf_problem_create.argtypes = [P, c.POINTER(_ScfInput), c.POINTER(P)]
    lib.vb_scf_problem_create_from_integrals.argtypes = [P, c.POINTER(_ScfIntegralInput), c.POINTER(P)]
    lib.vb_scf_problem_destroy.argtypes = [P]
    lib.vb_scf_problem_sizes.argtypes = [P, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int),
                                         c.POINTER(c.c_double)]
    lib.vb_scf_ao_integrals.argtypes = [P, P, P, P]
    lib.vb_scf_energy_gradient.argtypes = [P, P, c.POINTER(c.c_double), P, P, P]
    lib.vb_solve_scf.argtypes = [P, P, c.POINTER(_ScfOptions), c.POINTER(_ScfResult), P]
    lib.vb_scf_problem_set_precision.argtypes = [P, c.c_int, c.c_double]
    lib.vb_scf_problem_split_evaluations.argtypes = [P, c.POINTER(c.c_int32)]
    lib.vb_hs_plan_gradient.argtypes = [P, P, P, P, c.c_int, P, c.c_double, P, P, P, P, c.c_int, P]
    lib.vb_active_transform_ri.argtypes = [P, P, c.c_int, c.c_int, P, c.c_int, c.c_int, P, P, P]
    lib.vb_active_transform_ri_precision.argtypes = [P, P, c.c_int, c.c_int, P, c.c_int, c.c_int, c.c_int, P, P, P]
    lib.vb_active_transform_ri_adjoint.argtypes = [P, P, P, c.c_int, c.c_int, c.c_int, c.c_int, P]
    lib.vb_hs_plan_root_gradient.argtypes = [P, P, P, P, c.c_double, P, P, P, P, P, c.c_int, P]
    lib.vb_same_spin_pairs.argtypes = [P, c.c_int, c.c_int, c.c_int64, P, P, P, P, P, c.c_int, P, P]
    for name in EXPORTED_SYMBOLS:
        fn = getattr(lib, name)
        if name != "vb_last_error" and fn.restype is not c.c_char_p:
            fn.restype = c.c_int
    _lib = lib
    return lib


def _check(status: int, ctx_handle=None, info: int = 0):
    if status != 0:
        msg = load_library().vb_last_error(ctx_handle)
        raise VbError(status, msg.decode() if msg else "", info)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# ---------------------------------------------------------------------------------------------
# host-side structure setup (no GPU needed)


def generate_structures(keyword: str, n_active_orbitals: int, n_active_electrons: int,
                        spin_multiplicity: int = 1, n_inactive: int = 0) -> np.ndarray:
    """Raw structures, one row per structure of 1-based orbital labels (reference row layout)."""
    lib = load_library()
    n = ctypes.c_int64()
    _check(lib.vb_generate_structures(keyword.encode(), n_active_orbitals, n_active_electrons, spin_multiplicity,
                                      n_inactive, ctypes.byref(n), None, 0))
    width = n_active_electrons + 2 * n_inactive
    rows = np.zeros((n.value, width), dtype=np.int32)
    _check(lib.vb_generate_structures(keyword.encode(), n_active_orbitals, n_active_electrons, spin_multiplicity,
                                      n_inactive, ctypes.byref(n), _ptr(rows), rows.size))
    return rows


@dataclass
class Expansion:
    """Structure -> determinant expansion (StructureExpansion of the reference)."""
    n_structures: int
    n_alpha_electrons: int
    n_beta_electrons: int
    alpha_strings: np.ndarray  # uint64 occupation masks, ascending
    beta_strings: np.ndarray
    det_alpha: np.ndarray  # int32 string index per determinant
    det_beta: np.ndarray
    term_offsets: np.ndarray  # int64 CSR by determinant
    term_structure: np.ndarray  # int32
    term_coefficient: np.ndarray  # float64

    @property
    def n_determinants(self) -> int:
        return len(self.det_alpha)

    def occupations(self, beta: bool = False) -> np.ndarray:
        strings = self.beta_strings if beta else self.alpha_strings
        ids = self.det_beta if beta else self.det_alpha
        k = self.n_beta_electrons if beta else self.n_alpha_electrons
        occ = np.zeros((len(ids), k), dtype=np.int32)
        for d, s in enumerate(ids):
            m = int(strings[s])
            occ[d] = [i for i in range(64) if (m >> i) & 1]
        return occ


def expand_structures(rows: np.ndarray, n_active_electrons: int, spin_multiplicity: int = 1,
                      n_inactive: int = 0) -> Expansion:
    lib = load_library()
    rows = _c(rows, np.int32)
    sizes = _ExpansionSizes()
    _check(lib.vb_expand_structures(_ptr(rows), rows.shape[0], n_active_electrons, spin_multiplicity, n_inactive,
                                    ctypes.byref(sizes), None, None, None, None, None, None, None))
    a = np.zeros(sizes.n_alpha_strings, dtype=np.uint64)
    b = np.zeros(sizes.n_beta_strings, dtype=np.uint64)
    da = np.zeros(sizes.n_determinants, dtype=np.int32)
    db = np.zeros(sizes.n_determinants, dtype=np.int32)
    off = np.zeros(sizes.n_determinants + 1, dtype=np.int64)
    ts = np.zeros(sizes.n_terms, dtype=np.int32)
    tc = np.zeros(sizes.n_terms, dtype=np.float64)
    _check(lib.vb_expand_structures(_ptr(rows), rows.shape[0], n_active_electrons, spin_multiplicity, n_inactive,
                                    ctypes.byref(sizes), _ptr(a), _ptr(b), _ptr(da), _ptr(db), _ptr(off), _ptr(ts),
                                    _ptr(tc)))
    return Expansion(sizes.n_structures, sizes.n_alpha_electrons, sizes.n_beta_electrons, a, b, da, db, off, ts, tc)


# ---------------------------------------------------------------------------------------------
# device context and the H/S plan


_LIVE_CONTEXTS = None


def _close_live_contexts():
    """At interpreter exit: close every open context and the objects built on it, children first,
    while the native library and the CUDA runtime are still up."""
    for ctx in list(_LIVE_CONTEXTS or ()):
        try:
            ctx.close()
        except Exception:
            pass


class Context:
    """One device, one stream, an HBM budget (xmvb::cuda::Context of the reference)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        global _LIVE_CONTEXTS
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.vb_context_create(device, hbm_budget_bytes, ctypes.byref(h)))
        self._h = h
        self.device = device
        if _LIVE_CONTEXTS is None:
            import atexit
            import weakref

            _LIVE_CONTEXTS = weakref.WeakSet()
            atexit.register(_close_live_contexts)
        _LIVE_CONTEXTS.add(self)

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_handle: int | None):
        """Run this context's work on a caller stream (a cudaStream_t handle as an int).  None
        restores the context's own stream; 0 (torch's default stream) means the legacy default
        stream (cudaStreamLegacy)."""
        if stream_handle is None:
            handle = None
        elif stream_handle == 0:
            handle = 1  # cudaStreamLegacy
        else:
            handle = stream_handle
        _check(load_library().vb_context_set_stream(self._h, ctypes.c_void_p(handle)), self._h)

    def synchronize(self):
        _check(load_library().vb_context_synchronize(self._h), self._h)

    def set_barrier_spin_limit(self, polls: int):
        """Polls a grid-barrier wait of the cooperative eigensolver kernels makes before the call
        gives up with VB_ERR_TIMEOUT (0: the built-in default)."""
        _check(load_library().vb_context_set_barrier_spin_limit(self._h, int(polls)), self._h)

    def memory(self):
        cur, peak = ctypes.c_size_t(), ctypes.c_size_t()
        _check(load_library().vb_context_memory(self._h, ctypes.byref(cur), ctypes.byref(peak)), self._h)
        return cur.value, peak.value

    def _adopt(self, child):
        """Track an object whose native handle depends on this context (closed first)."""
        import weakref

        if not hasattr(self, "_children"):
            self._children = weakref.WeakSet()
        self._children.add(child)

    def close(self):
        for child in list(getattr(self, "_children", ())):
            child.close()
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().vb_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- determinant-pair level entry points ---------------------------------------------------

    def resolve_overlaps(self, blocks: np.ndarray):
        """blocks: (batch, k, k) -> (det, nullity, cofactor (batch, k, k)), reference semantics."""
        blocks = np.asarray(blocks, dtype=np.float64)
        batch, k, _ = blocks.shape
        colmajor = _c(np.transpose(blocks, (0, 2, 1)), np.float64)
        det = np.zeros(batch)
        nul = np.zeros(batch, dtype=np.int32)
        cof = np.zeros((batch, k, k))
        _check(load_library().vb_resolve_overlaps(self._h, k, batch, _ptr(colmajor), VB_MEM_HOST, _ptr(det), _ptr(nul),
                                                  _ptr(cof)), self._h)
        return det, nul, np.transpose(cof, (0, 2, 1)).copy()

    def same_spin_pairs(self, n_orbitals, occ_left, occ_right, S, h, eri):
        """Explicit same-spin pairs -> (scalars (batch, 4) = det, h1, htot, nullity; cofactors)."""
        occ_left = _c(occ_left, np.int32)
        occ_right = _c(occ_right, np.int32)
        batch, k = occ_left.shape
        sc = np.zeros((batch, 4))
        cof = np.zeros((batch, k, k))
        Sf = _c(np.asarray(S).T, np.float64)
        hf = _c(np.asarray(h).T, np.float64)
        ef = _c(eri, np.float64)
        _check(load_library().vb_same_spin_pairs(self._h, n_orbitals, k, batch, _ptr(occ_left), _ptr(occ_right),
                                                 _ptr(Sf), _ptr(hf), _ptr(ef), VB_MEM_HOST, _ptr(sc), _ptr(cof)),
               self._h)
        return sc, np.transpose(cof, (0, 2, 1)).copy()


def spin_pairs_noalloc(stream_handle: int, n_orbitals: int, k: int, n_strings: int, strings_ptr: int, S_ptr: int,
                       h_ptr: int, eri_ptr: int, out_ptr: int):
    """Allocation-free evaluation of every unordered pair of one spin-string table (device
    pointers; see vb_spin_pairs_noalloc in include/vbcore.h).  Raises VbError on failure."""
    _check(load_library().vb_spin_pairs_noalloc(ctypes.c_void_p(stream_handle), n_orbitals, k, n_strings,
                                                ctypes.c_void_p(strings_ptr), ctypes.c_void_p(S_ptr),
                                                ctypes.c_void_p(h_ptr), ctypes.c_void_p(eri_ptr),
                                                ctypes.c_void_p(out_ptr)))


def metric_cholesky(ctx: "Context", S) -> np.ndarray:
    """Upper Cholesky factor U of a symmetric positive-definite metric, S = U^T U (host
    arrays; overlap_upper of the reference).  Raises VbError (info = failing minor order)."""
    S = np.asarray(S, dtype=np.float64)
    n = S.shape[0]
    Sf = _c(S.T, np.float64)
    U = np.empty(n * n, dtype=np.float64)
    info = ctypes.c_int(0)
    st = load_library().vb_metric_cholesky(ctx.handle, _ptr(Sf), n, VB_MEM_HOST, _ptr(U), ctypes.byref(info))
    _check(st, ctx.handle, info.value)
    return U.reshape(n, n).T.copy()


def generalized_eigh(ctx: "Context", H, S):
    """(eigenvalues ascending, eigenvectors as columns) of H C = S C E with dsygvd semantics
    (GeneralizedEigensolver::solve_dense of the reference); host arrays."""
    H = np.asarray(H, dtype=np.float64)
    S = np.asarray(S, dtype=np.float64)
    n = H.shape[0]
    Hf = _c(H.T, np.float64)
    Sf = _c(S.T, np.float64)
    w = np.empty(n, dtype=np.float64)
    C = np.empty(n * n, dtype=np.float64)
    info = ctypes.c_int(0)
    st = load_library().vb_generalized_eigh(ctx.handle, _ptr(Hf), _ptr(Sf), n, VB_MEM_HOST, _ptr(w), _ptr(C),
                                            ctypes.byref(info))
    _check(st, ctx.handle, info.value)
    return w, C.reshape(n, n).T.copy()


def lowest_root(ctx: "Context", H, S, tolerance: float = 1e-10, max_iterations: int = 1000):
    """(E, c, iterations): lowest root of H c = E S c by the device Davidson iteration."""
    H = np.asarray(H, dtype=np.float64)
    S = np.asarray(S, dtype=np.float64)
    n = H.shape[0]
    Hf = _c(H.T, np.float64)
    Sf = _c(S.T, np.float64)
    c = np.empty(n)
    e = ctypes.c_double()
    its = ctypes.c_int()
    _check(load_library().vb_lowest_root(ctx.handle, _ptr(Hf), _ptr(Sf), n, VB_MEM_HOST, tolerance, max_iterations,
                                         ctypes.byref(e), _ptr(c), ctypes.byref(its)), ctx.handle)
    return e.value, c, its.value


def generalized_eigh_batched(ctx: "Context", problems, device=None):
    """Batched dense eigenproblems [(H, S), ...] (host arrays in, host results out), solved
    on the device one CTA per problem; returns [(eigenvalues, eigenvectors), ...]."""
    import torch

    dev = torch.device("cuda", ctx.device) if device is None else device
    dims = np.array([np.asarray(H).shape[0] for H, _ in problems], dtype=np.int32)
    sizes = dims.astype(np.int64) ** 2
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    voff = np.concatenate([[0], np.cumsum(dims.astype(np.int64))[:-1]]).astype(np.int64)
    Hcat = np.concatenate([np.asarray(H, dtype=np.float64).T.ravel() for H, _ in problems])
    Scat = np.concatenate([np.asarray(S, dtype=np.float64).T.ravel() for _, S in problems])
    dH = torch.tensor(Hcat, device=dev)
    dS = torch.tensor(Scat, device=dev)
    dw = torch.empty(int(dims.sum()), dtype=torch.float64, device=dev)
    dC = torch.empty(int(sizes.sum()), dtype=torch.float64, device=dev)
    info = np.zeros(len(problems), dtype=np.int32)
    torch.cuda.synchronize(dev)
    st = load_library().vb_generalized_eigh_batched(ctx.handle, len(problems), _ptr(dims), _ptr(offsets),
                                                    ctypes.c_void_p(dH.data_ptr()), ctypes.c_void_p(dS.data_ptr()),
                                                    VB_MEM_DEVICE, ctypes.c_void_p(dw.data_ptr()), _ptr(voff),
                                                    ctypes.c_void_p(dC.data_ptr()), _ptr(info))
    _check(st, ctx.handle, int(info[info != 0][0]) if np.any(info != 0) else 0)
    w = dw.cpu().numpy()
    C = dC.cpu().numpy()
    out = []
    for b, n in enumerate(dims):
        out.append((w[voff[b]:voff[b] + n].copy(), C[offsets[b]:offsets[b] + n * n].reshape(n, n).T.copy()))
    return out


PRECISIONS = {"fp64": 0, "bf16x3": 1}


def active_transform_ri(ctx: "Context", B_packed, C, one_index: bool = False, precision: str = "fp64"):
    """RI AO -> active transform (transform_ri_active_integrals of the reference), host arrays:
    B_packed [n_aux, n_bf(n_bf+1)/2], C [n_bf, n_act] -> (L [n_aux, P], K packed, T or None)
    with T [(n_act n_aux), n_bf] the one-index factors (row a*n_aux + P).  precision "bf16x3"
    runs the one-index step as split-BF16 tensor-core products (about 1e-7 relative)."""
    B = np.asarray(B_packed, dtype=np.float64)
    C = np.asarray(C, dtype=np.float64)
    n_aux = B.shape[0]
    n_bf, n_act = C.shape
    P = n_act * (n_act + 1) // 2
    Bf = _c(B.T, np.float64)  # column-major
    Cf = _c(C.T, np.float64)
    L = np.empty(n_aux * P, dtype=np.float64)
    K = np.empty(P * (P + 1) // 2, dtype=np.float64)
    T = np.empty(n_act * n_aux * n_bf, dtype=np.float64) if one_index else None
    st = load_library().vb_active_transform_ri_precision(ctx.handle, _ptr(Bf), n_aux, n_bf, _ptr(Cf), n_act,
                                                         PRECISIONS[precision], VB_MEM_HOST,
                                                         _ptr(T) if one_index else None, _ptr(L), _ptr(K))
    _check(st, ctx.handle)
    Lm = L.reshape(P, n_aux).T.copy()
    Tm = T.reshape(n_bf, n_act * n_aux).T.copy() if one_index else None
    return Lm, K, Tm


def active_transform_ri_adjoint(ctx: "Context", T, dL, n_bf: int):
    """dE/dC [n_bf, n_act] from dE/dL [n_aux, P] and the one-index factors T of the forward call."""
    T = np.asarray(T, dtype=np.float64)
    dL = np.asarray(dL, dtype=np.float64)
    n_aux, P = dL.shape
    n_act = int(round((np.sqrt(8 * P + 1) - 1) / 2))
    Tf = _c(T.T, np.float64)
    Gf = _c(dL.T, np.float64)
    dC = np.empty(n_bf * n_act, dtype=np.float64)
    st = load_library().vb_active_transform_ri_adjoint(ctx.handle, _ptr(Tf), _ptr(Gf), n_aux, n_bf, n_act,
                                                       VB_MEM_HOST, _ptr(dC))
    _check(st, ctx.handle)
    return dC.reshape(n_act, n_bf).T.copy()


def _scf_input(mol, pattern, n_electrons, multiplicity, structures, keep):
    arrays = [_c(mol.charges, np.float64), _c(mol.coords, np.float64), _c(mol.shell_atom, np.int32),
              _c(mol.shell_nprim, np.int32), _c(mol.shell_exponents, np.float64),
              _c(mol.shell_coefficients, np.float64)]
    offsets = np.concatenate([[0], np.cumsum([len(p) for p in pattern])]).astype(np.int32)
    funcs = np.array([m for p in pattern for m in p], dtype=np.int32)
    arrays += [offsets, funcs]
    keep.extend(arrays)
    kw = structures.encode()
    keep.append(kw)
    return _ScfInput(len(mol.charges), _ptr(arrays[0]).value, _ptr(arrays[1]).value, len(mol.shell_atom),
                     _ptr(arrays[2]).value, _ptr(arrays[3]).value, _ptr(arrays[4]).value, _ptr(arrays[5]).value,
                     len(pattern), _ptr(offsets).value, _ptr(funcs).value if funcs.size else None, n_electrons,
                     multiplicity, kw)


def _scf_integral_input(ints, pattern, n_electrons, multiplicity, structures, keep):
    S = _c(np.asarray(ints["S_ao"]).T, np.float64)
    hh = _c(np.asarray(ints["h_ao"]).T, np.float64)
    pf = _c(ints["pair_first"], np.int32)
    ps = _c(ints["pair_second"], np.int32)
    rows = _c(ints["rows"], np.int64)
    cols = _c(ints["columns"], np.int64)
    vals = _c(ints["values"], np.float64)
    offsets = np.concatenate([[0], np.cumsum([len(p) for p in pattern])]).astype(np.int32)
    funcs = np.array([m for p in pattern for m in p], dtype=np.int32)
    kw = structures.encode()
    keep.extend([S, hh, pf, ps, rows, cols, vals, offsets, funcs, kw])
    return _ScfIntegralInput(S.shape[0], _ptr(S).value, _ptr(hh).value, pf.size, _ptr(pf).value, _ptr(ps).value,
                             vals.size, _ptr(rows).value, _ptr(cols).value, _ptr(vals).value,
                             float(ints["nuclear_repulsion"]), len(pattern), _ptr(offsets).value,
                             _ptr(funcs).value if funcs.size else None, n_electrons, multiplicity, kw)


def ri_pair_factors_frame(ctx: "Context", factors, frame, mode: int = 0, factor_direction=None,
                          frame_direction=None):
    """RI pair factors [n_aux, n(n+1)/2] in the frame Q (mode 0: Q^T B Q; mode 1: the raw
    directional derivative; mode 2: the direction from factors already in the frame); host arrays."""
    F = np.asarray(factors, dtype=np.float64)
    n_aux, npair = F.shape
    n = int(round((np.sqrt(8 * npair + 1) - 1) / 2))
    Ff = _c(F.T, np.float64)  # column-major [n_aux x np]
    Qf = _c(np.asarray(frame).T, np.float64)
    Gf = _c(np.asarray(factor_direction).T, np.float64) if factor_direction is not None else None
    Df = _c(np.asarray(frame_direction).T, np.float64) if frame_direction is not None else None
    out = np.empty(n_aux * npair)
    _check(load_library().vb_ri_pair_factors_frame(ctx.handle, mode, _ptr(Ff), _ptr(Gf) if Gf is not None else None,
                                                   n_aux, n, _ptr(Qf), _ptr(Df) if Df is not None else None,
                                                   VB_MEM_HOST, _ptr(out)), ctx.handle)
    return out.reshape(npair, n_aux).T.copy()


def autotune_report() -> str:
    """The autotuner's cached choices, one line per (kernel, shape, device) key."""
    lib = load_library()
    need = ctypes.c_size_t(0)
    lib.vb_autotune_report(None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(max(1, need.value))
    lib.vb_autotune_report(buf, need.value, ctypes.byref(need))
    return buf.value.decode()


def autotune_clear():
    load_library().vb_autotune_clear()


def ao_pair_graph(eri, threshold: float = 0.0):
    """The unique-integral stream of an AO pair graph from a dense (mu nu|la si) [n,n,n,n]: pairs
    (mu >= nu), and each unordered pair of pairs once with |value| > threshold."""
    n = eri.shape[0]
    first, second = np.tril_indices(n)
    P = first.size
    V = eri[first[:, None], second[:, None], first[None, :], second[None, :]]
    r, c = np.tril_indices(P)
    keep = np.abs(V[r, c]) > threshold
    return dict(pair_first=first.astype(np.int32), pair_second=second.astype(np.int32),
                rows=r[keep].astype(np.int64), columns=c[keep].astype(np.int64), values=V[r, c][keep])


def ao_integrals_s(mol):
    """(S_ao, h_ao, eri_ao [n,n,n,n], nuclear repulsion) of an s-shell molecule (host only)."""
    keep = []
    inp = _scf_input(mol, [], 0, 1, "COV", keep)
    n = mol.n_basis
    S = np.empty(n * n)
    h = np.empty(n * n)
    eri = np.empty(n ** 4)
    enuc = ctypes.c_double(0.0)
    _check(load_library().vb_ao_integrals_s(ctypes.byref(inp), _ptr(S), _ptr(h), _ptr(eri), ctypes.byref(enuc)))
    return (S.reshape(n, n).T.copy(), h.reshape(n, n).T.copy(), eri.reshape(n, n, n, n).transpose(3, 2, 1, 0).copy(),
            enuc.value)


class ScfProblem:
    """A VBSCF problem (molecule, HAO pattern, structure class) with its plan on the device."""

    def __init__(self, ctx: "Context", mol, pattern, n_electrons: int, multiplicity: int = 1,
                 structures: str = "COV", integrals=None):
        """mol: an s-shell molecule (its AO integrals are computed by the library), or None with
        `integrals` = dict(S_ao, h_ao, pair_first, pair_second, rows, columns, values,
        nuclear_repulsion): AO integrals the caller already has, as an AO pair graph's unique
        integral stream (vb_scf_problem_create_from_integrals)."""
        self.ctx = ctx
        self.mol = mol
        self.pattern = pattern
        self._keep = []
        h = ctypes.c_void_p()
        if integrals is None:
            inp = _scf_input(mol, pattern, n_electrons, multiplicity, structures, self._keep)
            _check(load_library().vb_scf_problem_create(ctx.handle, ctypes.byref(inp), ctypes.byref(h)), ctx.handle)
        else:
            inp = _scf_integral_input(integrals, pattern, n_electrons, multiplicity, structures, self._keep)
            _check(load_library().vb_scf_problem_create_from_integrals(ctx.handle, ctypes.byref(inp), ctypes.byref(h)),
                   ctx.handle)
        self._h = h
        ctx._adopt(self)
        nb, na, ns, en = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        load_library().vb_scf_problem_sizes(h, ctypes.byref(nb), ctypes.byref(na), ctypes.byref(ns), ctypes.byref(en))
        self.n_basis, self.n_active, self.n_structures, self.nuclear_repulsion = nb.value, na.value, ns.value, en.value

    def energy_gradient(self, C, with_matrices: bool = False):
        """Total energy, dE/dC [n_basis, n_active] (zero outside the pattern) and, optionally,
        the structure H and S at coefficients C."""
        Cf = _c(np.asarray(C).T, np.float64)
        e = ctypes.c_double()
        g = np.empty(self.n_basis * self.n_active)
        ns = self.n_structures
        H = np.empty(ns * ns) if with_matrices else None
        S = np.empty(ns * ns) if with_matrices else None
        _check(load_library().vb_scf_energy_gradient(self._h, _ptr(Cf), ctypes.byref(e), _ptr(g),
                                                     _ptr(H) if with_matrices else None,
                                                     _ptr(S) if with_matrices else None), self.ctx.handle)
        out = (e.value, g.reshape(self.n_active, self.n_basis).T.copy())
        if with_matrices:
            out += (H.reshape(ns, ns).T.copy(), S.reshape(ns, ns).T.copy())
        return out

    def solve(self, C0, max_iterations: int = 200, gradient_tolerance: float = 1e-6, history_size: int = 100,
              armijo: float = 1e-4):
        """Quasi-Newton orbital optimization from C0; returns (result dict, final C)."""
        Cf = _c(np.asarray(C0).T, np.float64)
        out = np.empty(self.n_basis * self.n_active)
        opt = _ScfOptions(max_iterations, gradient_tolerance, history_size, armijo)
        res = _ScfResult()
        _check(load_library().vb_solve_scf(self._h, _ptr(Cf), ctypes.byref(opt), ctypes.byref(res), _ptr(out)),
               self.ctx.handle)
        split = ctypes.c_int32()
        _check(load_library().vb_scf_problem_split_evaluations(self._h, ctypes.byref(split)), self.ctx.handle)
        return ({"energy": res.energy, "gradient_inf": res.gradient_inf, "iterations": res.iterations,
                 "evaluations": res.evaluations, "split_evaluations": split.value, "converged": bool(res.converged)},
                out.reshape(self.n_active, self.n_basis).T.copy())

    def set_precision(self, precision: str = "fp64", switch_gradient: float = 1e-4):
        """RI transform precision of solve(): "bf16x3" evaluates in split precision until the
        gradient's infinity norm falls to switch_gradient, then finishes in FP64."""
        _check(load_library().vb_scf_problem_set_precision(self._h, PRECISIONS[precision], switch_gradient),
               self.ctx.handle)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().vb_scf_problem_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """Batched and served work on one GPU: `workers` host workers with their own contexts."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, workers: int = 8):
        h = ctypes.c_void_p()
        lib = load_library()
        _check(lib.vb_engine_create(device, hbm_budget_bytes, workers, ctypes.byref(h)))
        self._h = h
        self.workers = workers
        self._keep = []
        self._n = {}

    def _err(self, status):
        if status != 0:
            raise VbError(status, load_library().vb_engine_last_error(self._h).decode())

    def add_instance(self, expansion: "Expansion", n_orbitals: int) -> int:
        e = expansion
        keep = [_c(e.alpha_strings, np.uint64), _c(e.beta_strings, np.uint64), _c(e.det_alpha, np.int32),
                _c(e.det_beta, np.int32), _c(e.term_offsets, np.int64), _c(e.term_structure, np.int32),
                _c(e.term_coefficient, np.float64)]
        a, b, da, db, off, ts, tc = keep
        desc = _Expansion(n_orbitals, e.n_alpha_electrons, e.n_beta_electrons, len(a), len(b), _ptr(a).value,
                          _ptr(b).value, len(da), _ptr(da).value, _ptr(db).value, e.n_structures, _ptr(off).value,
                          _ptr(ts).value, _ptr(tc).value)
        iid = ctypes.c_int64()
        self._err(load_library().vb_engine_add_instance(self._h, ctypes.byref(desc), ctypes.byref(iid)))
        self._n[iid.value] = n_orbitals
        return iid.value

    def evaluate(self, ids, S_list, h_list, eri_list, F_list=None, gradient: bool = True):
        """Energies (lowest roots) and, if `gradient`, per-instance dicts {S, h, ri} of the gradient."""
        count = len(ids)
        P = ctypes.c_void_p
        keep = []

        def ptrs(arrays):
            arr = (P * count)()
            for i, x in enumerate(arrays):
                if x is None:
                    arr[i] = None
                else:
                    keep.append(x)
                    arr[i] = _ptr(x).value
            return arr

        Sf = [_c(np.asarray(S).T, np.float64) for S in S_list]
        hf = [_c(np.asarray(h).T, np.float64) for h in h_list]
        ef = [_c(e, np.float64) for e in eri_list]
        Ff = [None if (F_list is None or F is None) else _c(np.asarray(F).T, np.float64)
              for F in (F_list or [None] * count)]
        naux = np.array([0 if F is None else np.asarray(F_list[i]).shape[1] for i, F in enumerate(Ff)], np.int32)
        energies = np.empty(count)
        gS = [np.empty(self._n[i] ** 2) for i in ids] if gradient else None
        gh = [np.empty(self._n[i] ** 2) for i in ids] if gradient else None
        gF = [None if F is None else np.empty(F.size) for F in Ff] if gradient else None
        idarr = np.asarray(ids, np.int64)
        st = load_library().vb_engine_evaluate_instances(
            self._h, count, _ptr(idarr), ptrs(Sf), ptrs(hf), ptrs(ef), ptrs(Ff), _ptr(naux), _ptr(energies),
            ptrs(gS) if gradient else None, ptrs(gh) if gradient else None, ptrs(gF) if gradient else None)
        self._err(st)
        if not gradient:
            return energies, None
        grads = []
        for i, iid in enumerate(ids):
            n = self._n[iid]
            g = {"S": gS[i].reshape(n, n).T.copy(), "h": gh[i].reshape(n, n).T.copy()}
            if gF[i] is not None:
                g["ri"] = gF[i].reshape(naux[i], -1).T.copy()
            grads.append(g)
        return energies, grads

    def submit_scf(self, mol, pattern, n_electrons, C0, multiplicity: int = 1, structures: str = "COV",
                   max_iterations: int = 200, gradient_tolerance: float = 1e-6, history_size: int = 100,
                   tag: int = 0):
        keep = []
        inp = _scf_input(mol, pattern, n_electrons, multiplicity, structures, keep)
        Cf = _c(np.asarray(C0).T, np.float64)
        opt = _ScfOptions(max_iterations, gradient_tolerance, history_size, 1e-4)
        self._err(load_library().vb_engine_submit_scf(self._h, ctypes.byref(inp), _ptr(Cf), ctypes.byref(opt), tag))

    def poll(self, wait: bool = True, capacity: int = 256):
        tags = np.empty(capacity, np.int64)
        e = np.empty(capacity)
        g = np.empty(capacity)
        it = np.empty(capacity, np.int32)
        cv = np.empty(capacity, np.int32)
        st = np.empty(capacity, np.int32)
        ws = np.empty(capacity)
        lat = np.empty(capacity)
        n = ctypes.c_int()
        self._err(load_library().vb_engine_poll(self._h, capacity, 1 if wait else 0, _ptr(tags), _ptr(e), _ptr(g),
                                                _ptr(it), _ptr(cv), _ptr(st), _ptr(ws), _ptr(lat), ctypes.byref(n)))
        return [{"tag": int(tags[i]), "energy": float(e[i]), "gradient_inf": float(g[i]), "iterations": int(it[i]),
                 "converged": bool(cv[i]), "status": int(st[i]), "wait_s": float(ws[i]), "latency_s": float(lat[i])}
                for i in range(n.value)]

    def pending(self):
        q, r, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        self._err(load_library().vb_engine_pending(self._h, ctypes.byref(q), ctypes.byref(r), ctypes.byref(b)))
        return q.value, r.value, b.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().vb_engine_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HsPlan:
    """Structure Hamiltonian/overlap builder with the topology resident on the device."""

    def __init__(self, ctx: Context, expansion: Expansion, n_orbitals: int):
        self.ctx = ctx
        self.expansion = expansion
        self.n_orbitals = n_orbitals
        e = expansion
        self._keep = [_c(e.alpha_strings, np.uint64), _c(e.beta_strings, np.uint64), _c(e.det_alpha, np.int32),
                      _c(e.det_beta, np.int32), _c(e.term_offsets, np.int64), _c(e.term_structure, np.int32),
                      _c(e.term_coefficient, np.float64)]
        a, b, da, db, off, ts, tc = self._keep
        desc = _Expansion(n_orbitals, e.n_alpha_electrons, e.n_beta_electrons, len(a), len(b), _ptr(a).value,
                          _ptr(b).value, len(da), _ptr(da).value, _ptr(db).value, e.n_structures, _ptr(off).value,
                          _ptr(ts).value, _ptr(tc).value)
        h = ctypes.c_void_p()
        _check(load_library().vb_hs_plan_create(ctx.handle, ctypes.byref(desc), ctypes.byref(h)), ctx.handle)
        self._h = h
        ctx._adopt(self)
        self.n_structures = e.n_structures

    def execute(self, S, h, eri):
        """Host arrays in (S, h as n x n; eri packed), host H and S out."""
        n = self.n_orbitals
        Sf = _c(np.asarray(S).T, np.float64)
        hf = _c(np.asarray(h).T, np.float64)
        ef = _c(eri, np.float64)
        if Sf.size != n * n or hf.size != n * n:
            raise VbError(1, "S and h must be n_orbitals x n_orbitals")
        np_ = n * (n + 1) // 2
        if ef.size != np_ * (np_ + 1) // 2:
            raise VbError(1, "eri must hold P(P+1)/2 packed values")
        ns = self.n_structures
        H = np.zeros((ns, ns))
        So = np.zeros((ns, ns))
        _check(load_library().vb_hs_plan_execute(self._h, _ptr(Sf), _ptr(hf), _ptr(ef), VB_MEM_HOST, _ptr(H), _ptr(So)),
               self.ctx.handle)
        return H.T.copy(), So.T.copy()

    def execute_device(self, S_ptr: int, h_ptr: int, eri_ptr: int, H_ptr: int, S_out_ptr: int):
        """Device pointers (column-major S/h; packed eri); stream-ordered, no synchronization."""
        _check(load_library().vb_hs_plan_execute(self._h, ctypes.c_void_p(S_ptr), ctypes.c_void_p(h_ptr),
                                                 ctypes.c_void_p(eri_ptr), VB_MEM_DEVICE, ctypes.c_void_p(H_ptr),
                                                 ctypes.c_void_p(S_out_ptr)), self.ctx.handle)

    def execute_host_pointers(self, S_ptr: int, h_ptr: int, eri_ptr: int, H_ptr: int, S_out_ptr: int):
        """Host pointers (ideally pinned; column-major S/h; packed eri): copies in, evaluates,
        copies H and S out, and returns when the results are on the host."""
        _check(load_library().vb_hs_plan_execute(self._h, ctypes.c_void_p(S_ptr), ctypes.c_void_p(h_ptr),
                                                 ctypes.c_void_p(eri_ptr), VB_MEM_HOST, ctypes.c_void_p(H_ptr),
                                                 ctypes.c_void_p(S_out_ptr)), self.ctx.handle)

    def root_gradient(self, S, h, eri, ri_factors=None, tolerance: float = 1e-11, gradient: bool = True):
        """Lowest root of the structure problem at host inputs with H and S kept on the device,
        and (gradient=True) its gradient: (E, c, {"S": dS, "h": dh, "ri": dF or None})."""
        n = self.n_orbitals
        Sf = _c(np.asarray(S).T, np.float64)
        hf = _c(np.asarray(h).T, np.float64)
        ef = _c(eri, np.float64)
        ns = self.n_structures
        E = ctypes.c_double()
        c = np.empty(ns)
        gS = np.empty(n * n) if gradient else None
        gh = np.empty(n * n) if gradient else None
        Ff = dF = None
        n_aux = 0
        if gradient and ri_factors is not None:
            F = np.asarray(ri_factors, dtype=np.float64)
            n_aux = F.shape[1]
            Ff = _c(F.T, np.float64)
            dF = np.empty(F.size)
        _check(load_library().vb_hs_plan_root_gradient(
            self._h, _ptr(Sf), _ptr(hf), _ptr(ef), tolerance, ctypes.byref(E), _ptr(c),
            _ptr(gS) if gradient else None, _ptr(gh) if gradient else None, _ptr(Ff) if Ff is not None else None,
            n_aux, _ptr(dF) if dF is not None else None), self.ctx.handle)
        g = None
        if gradient:
            g = {"S": gS.reshape(n, n).T.copy(), "h": gh.reshape(n, n).T.copy(),
                 "ri": dF.reshape(n_aux, -1).T.copy() if dF is not None else None}
        return E.value, c, g

    def gradient(self, S, h, eri, coefficients, eigenvalue, packed_eri: bool = True, ri_factors=None):
        """Gradient of the structure root (eigenvalue, S-normalized coefficients) with respect to
        S, h (symmetric n x n) and the packed integrals (if packed_eri) or RI factors
        F [n(n+1)/2, n_aux] with (ij|kl) = F[pair(i,j)] . F[pair(k,l)] (if given).
        Returns a dict with keys S, h and eri / ri."""
        n = self.n_orbitals
        Sf = _c(np.asarray(S).T, np.float64)
        hf = _c(np.asarray(h).T, np.float64)
        ef = _c(eri, np.float64)
        cf = _c(coefficients, np.float64)
        gS = np.empty(n * n)
        gh = np.empty(n * n)
        ge = np.empty(ef.size) if packed_eri else None
        F = None if ri_factors is None else _c(np.asarray(ri_factors).T, np.float64)
        n_aux = 0 if ri_factors is None else np.asarray(ri_factors).shape[1]
        gF = None if ri_factors is None else np.empty(F.size)
        st = load_library().vb_hs_plan_gradient(self._h, _ptr(Sf), _ptr(hf), _ptr(ef), VB_MEM_HOST, _ptr(cf),
                                                float(eigenvalue), _ptr(gS), _ptr(gh),
                                                _ptr(ge) if packed_eri else None, _ptr(F) if F is not None else None,
                                                n_aux, _ptr(gF) if gF is not None else None)
        _check(st, self.ctx.handle)
        out = {"S": gS.reshape(n, n).T.copy(), "h": gh.reshape(n, n).T.copy()}
        if packed_eri:
            out["eri"] = ge
        if gF is not None:
            out["ri"] = gF.reshape(n_aux, -1).T.copy()
        return out

    def determinant_pairs(self, S, h, eri, pairs):
        """<d|H|e>, <d|e> for an (m, 2) array of determinant index pairs."""
        pairs = _c(pairs, np.int64)
        m = pairs.shape[0]
        ho = np.zeros(m)
        so = np.zeros(m)
        Sf = _c(np.asarray(S).T, np.float64)
        hf = _c(np.asarray(h).T, np.float64)
        ef = _c(eri, np.float64)
        _check(load_library().vb_hs_plan_determinant_pairs(self._h, _ptr(Sf), _ptr(hf), _ptr(ef), m, _ptr(pairs),
                                                           VB_MEM_HOST, _ptr(ho), _ptr(so)), self.ctx.handle)
        return ho, so

    def stats(self) -> dict:
        st = _HsStats()
        _check(load_library().vb_hs_plan_stats(self._h, ctypes.byref(st)), self.ctx.handle)
        return dict(spin_pairs=st.spin_pairs, careful_spin_pairs=st.careful_spin_pairs,
                    determinant_pairs=st.determinant_pairs, kernel_launches=st.kernel_launches,
                    factor_columns=st.factor_columns)

    def enable_phase_timing(self, enable: bool = True):
        _check(load_library().vb_hs_plan_enable_phase_timing(self._h, int(enable)), self.ctx.handle)

    def phase_times(self) -> dict:
        """Milliseconds per phase of the last execute (CUDA events on the context stream)."""
        out = np.zeros(len(PHASES))
        _check(load_library().vb_hs_plan_phase_times(self._h, _ptr(out), len(PHASES)), self.ctx.handle)
        return dict(zip(PHASES, out.tolist()))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().vb_hs_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
