"""The allocation-free spin-pair entry point, vb_spin_pairs_noalloc.

It exists for callers that cannot allocate device memory where they need these numbers: a
serving loop that reserves all of its HBM up front and forbids allocation on the request
path, or an application whose own allocator already owns the whole device budget.  It takes
all scratch from a static device array instead.  These checks call it through the C ABI,
twice in a row with different tables and inputs (the array keeps the previous call's
contents in between), and compare every pair with the existing same-spin entry point,
vb_same_spin_pairs, at the tolerance the other parity tests use.  This file is collected
last on purpose."""

import itertools

import numpy as np
import pytest

import vbcore
from vbcore import workloads

REL = 1e-10


def _masks(n, k):
    return sorted(sum(1 << o for o in occ) for occ in itertools.combinations(range(n), k))


def _occ(mask):
    return [o for o in range(64) if (mask >> o) & 1]


def test_noalloc_rejects_tables_beyond_the_static_scratch():
    # 3432 strings of 7 electrons need far more than the 32 MiB static array; the size check
    # runs before any CUDA call, so this needs no GPU
    with pytest.raises(vbcore.VbError, match="static scratch"):
        vbcore.spin_pairs_noalloc(0, 14, 7, 3432, 1, 1, 1, 1, 1)


@pytest.mark.gpu
def test_noalloc_matches_existing_entry_point_on_two_calls():
    import torch

    ctx = vbcore.Context(0)
    dev = torch.device("cuda:0")
    cases = [(10, 5, workloads.active_space(10, 30, 31)), (8, 4, workloads.active_space(8, 24, 32))]
    # the second call's overlap is the identity: most pairs are singular and take the exact path
    S8, h8, e8 = cases[1][2]
    cases[1] = (8, 4, (np.eye(8), h8, e8))
    for n, k, (S, h, eri) in cases:
        masks = _masks(n, k)
        N = len(masks)
        d_masks = torch.tensor(np.array(masks, dtype=np.uint64).view(np.int64), device=dev)
        dS = torch.tensor(np.ascontiguousarray(S.T), device=dev)
        dh = torch.tensor(np.ascontiguousarray(h.T), device=dev)
        de = torch.tensor(eri, device=dev)
        n_pairs = N * (N + 1) // 2
        out = torch.full((4 * n_pairs,), float("nan"), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        vbcore.spin_pairs_noalloc(stream, n, k, N, d_masks.data_ptr(), dS.data_ptr(), dh.data_ptr(), de.data_ptr(),
                                  out.data_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(n_pairs, 4)
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
    ctx.close()
