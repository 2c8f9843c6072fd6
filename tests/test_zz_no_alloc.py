"""The allocation-free grouped-moments entry point.

cs_b200_group_moments_blocked_ell_noalloc serves callers that may not call
cudaMalloc (a plugin inside a process whose device memory another allocator
owns or caps): it works in a fixed static scratch array inside the library.
These tests call it through the C ABI and check it against the regular entry
point with caller-provided scratch, within the tolerance the moments tests
use (1e-6 relative), on two calls in a row with different inputs -- the
second call runs over the first call's leftover scratch contents.  This file
is collected last so that a run stopping at its first failure has already
run every other test; it also passes on its own in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

from cases import random_csr, to_device_csr

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def _inputs(rows, cols, B, G, seed):
    import torch

    from cellshard_b200.device import blocked_ell_from_csr

    ptr, idx, val = random_csr(rows, cols, 0.06, seed, 0.1, integer=(seed % 2 == 0))
    bell = blocked_ell_from_csr(to_device_csr(rows, cols, ptr, idx, val), B)
    rng = np.random.default_rng(seed)
    rk = torch.from_numpy((rng.random(rows) < 0.7).astype(np.uint8)).cuda()
    fk = torch.from_numpy((rng.random(cols) < 0.8).astype(np.uint8)).cuda()
    lab = torch.from_numpy(rng.integers(0, G, rows).astype(np.uint32).view(np.int32)).cuda()
    return bell, rk, fk, lab


def _outputs(G, cols):
    import torch

    out = {k: torch.full((G, cols), -1.0, dtype=torch.float32, device="cuda") for k in ("sum", "sumsq", "mean", "var")}
    out["group_rows"] = torch.zeros(G, dtype=torch.int32, device="cuda")
    out["status"] = torch.zeros(1, dtype=torch.int32, device="cuda")
    return out


def _noalloc(bell, G, rk, fk, lab, out, chunk_rows=0):
    import torch

    from cellshard_b200 import _abi
    from cellshard_b200.device import ptr

    lib = _abi.load()
    p = _abi.GroupMomentsParams(G, 2, 1, chunk_rows)
    o = _abi.GroupMomentsOut(ptr(out["sum"]), ptr(out["sumsq"]), ptr(out["mean"]), ptr(out["var"]), None, None,
                             ptr(out["group_rows"]), ptr(out["status"]))
    v = bell.view()
    ok = lib.cs_b200_group_moments_blocked_ell_noalloc(C.byref(v), ptr(rk), ptr(fk), ptr(lab), C.byref(p),
                                                       C.byref(o), torch.cuda.current_stream().cuda_stream)
    _abi.check(ok, "group_moments_blocked_ell_noalloc")


def _close(a, b):
    a = a.cpu().numpy().astype(np.float64)
    b = b.cpu().numpy().astype(np.float64)
    err = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    return bool(np.all((err <= RTOL) | (np.abs(a - b) <= 1e-30)))


def test_noalloc_matches_caller_scratch_entry_point_on_two_calls(cuda):
    import torch

    from cellshard_b200 import runtime

    cases = [(3000, 700, 16, 9, 1), (4100, 1500, 8, 31, 2)]
    for n, (rows, cols, B, G, seed) in enumerate(cases):
        bell, rk, fk, lab = _inputs(rows, cols, B, G, seed)
        ref = runtime.compute_sparse_group_moments(bell, G, rk, fk, lab, ddof=1)
        out = _outputs(G, cols)
        torch.cuda.synchronize()
        free = [torch.cuda.mem_get_info()[0]]
        for _ in range(3 if n > 0 else 1):
            _noalloc(bell, G, rk, fk, lab, out)
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
        if n > 0:
            # once the first call has located the static scratch, repeated calls allocate nothing:
            # the device's free memory stays the same across all of them
            assert len(set(free)) == 1, free
        assert int(out["status"].item()) == 0
        assert torch.equal(out["group_rows"], ref["group_rows"])
        for k in ("sum", "sumsq", "mean", "var"):
            assert _close(out[k], ref[k]), (n, k)


def test_noalloc_rejects_partitions_beyond_the_static_scratch(cuda):
    from cellshard_b200 import _abi

    lib = _abi.load()
    v = _abi.BlockedEllView()
    v.rows, v.cols, v.block_size, v.ell_cols = 500_000, 32768, 16, 32768
    p = _abi.GroupMomentsParams(64, 2, 1, 0)
    o = _abi.GroupMomentsOut()
    assert lib.cs_b200_group_moments_blocked_ell_noalloc(C.byref(v), None, None, None, C.byref(p), C.byref(o),
                                                         None) == 0
    msg = lib.cs_b200_last_error().decode()
    assert "static scratch" in msg and str(64 * 1024 * 1024) in msg
