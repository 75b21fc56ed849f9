"""The launch-schedule autotuner: the first evaluation of a shape times the spin-pair kernel's
pair-to-warp schedules (2, 4 or 8 warps per CTA) and the determinant-pair kernel's block shapes,
keeps the fastest, and every schedule gives bitwise the same structure matrices (each pair's
arithmetic does not depend on which warp or CTA evaluates it)."""

import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
import vbcore
from vbcore import workloads

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import sys
sys.path[:0] = [{pkg!r}]
import numpy as np
import vbcore
from vbcore import workloads
ctx = vbcore.Context(0)
n = 10
S, h, eri = workloads.active_space(n, 30, 77)
ex = vbcore.expand_structures(vbcore.generate_structures("COV ION(1)", n, n), n)
plan = vbcore.HsPlan(ctx, ex, n)
H, So = plan.execute(S, h, eri)
np.save({out!r}, np.stack([H, So]))
print(vbcore.autotune_report())
"""


def test_tuned_schedules_are_cached_and_do_not_change_results(tmp_path):
    n = 10
    S, h, eri = workloads.active_space(n, 30, 77)
    ctx = vbcore.Context(0)
    try:
        ex = vbcore.expand_structures(vbcore.generate_structures("COV ION(1)", n, n), n)
        plan = vbcore.HsPlan(ctx, ex, n)
        H1, S1 = plan.execute(S, h, eri)  # tunes (first time this shape is seen)
        report = vbcore.autotune_report()
        H2, S2 = plan.execute(S, h, eri)  # cached choices
        plan.close()
    finally:
        ctx.close()
    assert "spin_pairs_frame k=5 n=10" in report and "full_pairs_kernel" in report
    for line in report.strip().splitlines():
        ms = [float(x) for x in line.split("(ms:")[1].rstrip(")").split()]
        assert len(ms) >= 2 and all(m > 0 for m in ms)
        assert int(line.split("->")[1].split()[0]) == int(np.argmin(ms))
    assert np.array_equal(H1, H2) and np.array_equal(S1, S2)
    ex_o = O.expand(O.generate_structures("COV ION(1)", n, n), n)
    Hr, Sr, _ = O.structure_matrices(n, ex_o, S, h, eri)
    assert np.abs(H1 - Hr).max() <= 1e-10 * max(1.0, np.abs(Hr).max())
    # the default schedules (tuning off) in a fresh process: bitwise the same matrices
    out = str(tmp_path / "untuned.npy")
    env = dict(os.environ, VBCORE_AUTOTUNE="0")
    code = _CHILD.format(pkg=os.path.join(ROOT, "xmvb-cpp_b200"), out=out)
    proc = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-3000:]
    assert proc.stdout.strip() == ""  # nothing tuned
    HS = np.load(out)
    assert np.array_equal(HS[0], H1) and np.array_equal(HS[1], S1)
