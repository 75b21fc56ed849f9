"""CPU-side checks of the product library: it loads, exports every symbol include/vbcore.h
declares, and its host-side structure generation and expansion match the oracle's
restatement of the reference (generated_structures.cpp, expander.cpp) exactly."""

import os
import re

import numpy as np
import pytest

import oracle as O
import vbcore
from conftest import ROOT


def test_header_symbols_exported():
    lib = vbcore.load_library()
    header = open(os.path.join(ROOT, "include", "vbcore.h")).read()
    declared = set(re.findall(r"\b(vb_[a-z_]+)\s*\(", header))
    assert declared == set(vbcore.EXPORTED_SYMBOLS)
    for name in declared:
        assert hasattr(lib, name), name


@pytest.mark.parametrize("kw,n,nel,mult", [
    ("COV", 4, 4, 1), ("COV", 6, 6, 1), ("COV", 14, 14, 1), ("COV ION(1)", 6, 6, 1), ("COV ION(1)", 8, 8, 1),
    ("FULL", 4, 4, 1), ("COV", 5, 4, 3), ("COV", 6, 4, 1), ("COV", 5, 5, 2), ("ION(1-2)", 6, 6, 1),
])
def test_generation_and_expansion_match_oracle(kw, n, nel, mult):
    rows = vbcore.generate_structures(kw, n, nel, mult)
    ref_rows = O.generate_structures(kw, n, nel, mult)
    assert np.array_equal(rows, np.array(ref_rows))
    ex = vbcore.expand_structures(rows, nel, mult)
    ref = O.expand(ref_rows, nel, mult)
    assert ex.n_structures == ref.n_structures
    assert list(ex.alpha_strings) == ref.alpha_strings
    assert list(ex.beta_strings) == ref.beta_strings
    assert np.array_equal(ex.det_alpha, ref.det_alpha)
    assert np.array_equal(ex.det_beta, ref.det_beta)
    assert np.array_equal(ex.term_offsets, ref.offsets)
    assert np.array_equal(ex.term_structure, ref.term_structure)
    assert np.array_equal(ex.term_coefficient, ref.term_coefficient)


def test_generation_errors_are_reported():
    with pytest.raises(vbcore.VbError, match="structure class"):
        vbcore.generate_structures("ION(9)", 6, 6, 1)
    with pytest.raises(vbcore.VbError):
        vbcore.generate_structures("BOGUS", 6, 6, 1)


def test_context_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(vbcore.VbError):
        vbcore.Context(0)
