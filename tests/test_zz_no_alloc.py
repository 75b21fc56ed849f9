"""The allocation-free spin-pair entry point, vb_spin_pairs_noalloc.

It exists for callers that cannot allocate device memory where they need these numbers: a
serving loop that reserves all of its HBM up front and forbids allocation on the request
path, or an application whose own allocator already owns the whole device budget.  It takes
all scratch from a static device array instead.  These checks call it through the C ABI,
twice in a row with different tables and inputs (the array keeps the previous call's
contents in between), and compare every pair with the oracle's same-spin pair restatement and
with the existing same-spin entry point, vb_same_spin_pairs, at the tolerance the other parity
tests use.  One check runs in a fresh process that never creates a vb_context, so the entry
point's own first-call set-up is what reserves the exact-path kernels' stack and loads its
kernels; there the device's free memory must not change across any later call.  This file is
collected last on purpose."""

import itertools
import os
import subprocess
import sys

import numpy as np
import pytest

import vbcore
from vbcore import workloads

REL = 1e-10
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _masks(n, k):
    return sorted(sum(1 << o for o in occ) for occ in itertools.combinations(range(n), k))


def _occ(mask):
    return [o for o in range(64) if (mask >> o) & 1]


def _cases():
    cases = [(10, 5, workloads.active_space(10, 30, 31)), (8, 4, workloads.active_space(8, 24, 32))]
    # the second call's overlap is the identity: most pairs are singular and take the exact path
    _, h8, e8 = cases[1][2]
    cases[1] = (8, 4, (np.eye(8), h8, e8))
    return cases


def _call_noalloc(n, k, S, h, eri):
    """One call through the C ABI with torch-owned device buffers; returns (n_pairs x 4) scalars."""
    import torch

    dev = torch.device("cuda:0")
    masks = _masks(n, k)
    N = len(masks)
    d_masks = torch.tensor(np.array(masks, dtype=np.uint64).view(np.int64), device=dev)
    dS = torch.tensor(np.ascontiguousarray(S.T), device=dev)
    dh = torch.tensor(np.ascontiguousarray(h.T), device=dev)
    de = torch.tensor(eri, device=dev)
    n_pairs = N * (N + 1) // 2
    out = torch.full((4 * n_pairs,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    stream = torch.cuda.current_stream(dev).cuda_stream
    vbcore.spin_pairs_noalloc(stream, n, k, N, d_masks.data_ptr(), dS.data_ptr(), dh.data_ptr(), de.data_ptr(),
                              out.data_ptr())
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(0)[0]
    return masks, out.cpu().numpy().reshape(n_pairs, 4), (free_before, free_after)


def _check_against_oracle(n, masks, got, S, h, eri):
    import oracle as O

    N = len(masks)
    t = 0
    for u in range(N):
        for v in range(u, N):
            ref = O.spin_pair(n, _occ(masks[u]), _occ(masks[v]), S, h, eri)
            assert int(got[t, 3]) == ref["nullity"], f"nullity differs at pair {t}"
            for col, key in ((0, "det"), (1, "h1"), (2, "htot")):
                assert abs(got[t, col] - ref[key]) <= REL * max(1.0, abs(ref[key])), f"{key} differs at pair {t}"
            t += 1


def test_noalloc_rejects_tables_beyond_the_static_scratch():
    # 3432 strings of 7 electrons need far more than the 32 MiB static array; the size check
    # runs before any CUDA call, so this needs no GPU
    with pytest.raises(vbcore.VbError, match="static scratch"):
        vbcore.spin_pairs_noalloc(0, 14, 7, 3432, 1, 1, 1, 1, 1)


@pytest.mark.gpu
def test_noalloc_matches_oracle_and_existing_entry_point_on_two_calls():
    results = []
    for n, k, (S, h, eri) in _cases():
        masks, got, _ = _call_noalloc(n, k, S, h, eri)
        results.append((n, masks, got, S, h, eri))
    for n, masks, got, S, h, eri in results:
        _check_against_oracle(n, masks, got, S, h, eri)
    ctx = vbcore.Context(0)
    try:
        for n, masks, got, S, h, eri in results:
            N = len(masks)
            left, right = [], []
            for u in range(N):
                for v in range(u, N):
                    left.append(_occ(masks[u]))
                    right.append(_occ(masks[v]))
            ref, _ = ctx.same_spin_pairs(n, np.array(left), np.array(right), S, h, eri)
            assert np.array_equal(got[:, 3], ref[:, 3]), "nullity differs"
            for col in range(3):
                scale = np.maximum(1.0, np.abs(ref[:, col]))
                assert np.all(np.abs(got[:, col] - ref[:, col]) <= REL * scale), f"column {col} differs"
    finally:
        ctx.close()


_FRESH = r"""
import sys
sys.path[:0] = [{pkg!r}, {ora!r}, {tests!r}]
import torch
import test_zz_no_alloc as T
random_case, identity_case = T._cases()
free = []
# first call on the device (the set-up call): identity overlap, so the exact path runs too
for n, k, (S, h, eri) in (identity_case, random_case, identity_case):
    masks, got, (before, after) = T._call_noalloc(n, k, S, h, eri)
    free.append((before, after))
    T._check_against_oracle(n, masks, got, S, h, eri)
# after the set-up call, no call may change the device's free memory
for before, after in free[1:]:
    assert before == after, f"free device memory changed across a call: {{free}}"
print("fresh-process noalloc ok", free)
"""


@pytest.mark.gpu
def test_noalloc_in_a_fresh_process_without_a_context():
    code = _FRESH.format(pkg=os.path.join(ROOT, "xmvb-cpp_b200"), ora=os.path.join(ROOT, "oracle"),
                         tests=os.path.join(ROOT, "tests"))
    proc = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stdout[-2000:] + proc.stderr[-4000:]
    assert "fresh-process noalloc ok" in proc.stdout
