"""The reference-side C++ shim (tests/shim/cuvbscf_shim.cpp: the `cuvbscf` solve entry routed to
vb_scf_problem_create_from_integrals + vb_solve_scf, with std::vector stand-ins for the reference's
types) compiled against include/vbcore.h and linked with libvbcore.so; on the GPU it solves H6
from AO integrals passed as an AO pair graph, and its energy equals the library's own solve."""

import os
import subprocess

import numpy as np
import pytest

import vbcore
from vbcore import molecules

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "xmvb-cpp_b200", "lib")


def _build(tmp_path):
    exe = str(tmp_path / "cuvbscf_shim")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "shim", "cuvbscf_shim.cpp"), "-L", LIBDIR, "-lvbcore",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
    return exe


def test_shim_compiles_and_links(tmp_path):
    vbcore.load_library()
    assert os.path.exists(_build(tmp_path))


def _write_problem(path, S, h, graph, enuc, pattern, n_el, mult, keyword, C0):
    with open(path, "w") as f:
        n = S.shape[0]
        f.write(f"{n}\n")
        f.write(" ".join(repr(float(x)) for x in S.T.reshape(-1)) + "\n")
        f.write(" ".join(repr(float(x)) for x in h.T.reshape(-1)) + "\n")
        f.write(f"{len(graph['pair_first'])}\n")
        for a, b in zip(graph["pair_first"], graph["pair_second"]):
            f.write(f"{a} {b}\n")
        f.write(f"{len(graph['values'])}\n")
        for r, c, v in zip(graph["rows"], graph["columns"], graph["values"]):
            f.write(f"{r} {c} {float(v)!r}\n")
        f.write(f"{float(enuc)!r} {len(pattern)}\n")
        for funcs in pattern:
            f.write(f"{len(funcs)} " + " ".join(str(m) for m in funcs) + "\n")
        f.write(f"{n_el} {mult} {keyword}\n")
        f.write(" ".join(repr(float(x)) for x in C0.T.reshape(-1)) + "\n")


@pytest.mark.gpu
def test_shim_solves_h6_from_an_ao_pair_graph(tmp_path):
    exe = _build(tmp_path)
    mol = molecules.h_chain(6, 1.0, 0.05, seed=20261203)
    pattern = molecules.hao_pattern(mol, 6)
    C0 = molecules.hao_guess(mol, pattern)
    S, h, eri, enuc = vbcore.ao_integrals_s(mol)
    graph = vbcore.ao_pair_graph(eri, threshold=1e-14)
    path = str(tmp_path / "h6.txt")
    _write_problem(path, S, h, graph, enuc, pattern, 6, 1, "COV", C0)
    proc = subprocess.run([exe, path], capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    out = dict(line.split() for line in proc.stdout.strip().splitlines())
    assert out["converged"] == "1"
    ctx = vbcore.Context(0)
    try:
        prob = vbcore.ScfProblem(ctx, mol, pattern, 6)
        res, _ = prob.solve(C0, gradient_tolerance=1e-7)
        prob.close()
    finally:
        ctx.close()
    assert abs(float(out["energy"]) - res["energy"]) < 1e-9
