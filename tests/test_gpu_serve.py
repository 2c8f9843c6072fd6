"""Serving loop (device-resident persistent kernel, HBM-budget admission,
continuous batching) vs the FP64 oracle on the concatenated partitions.

Tolerance: the FP64-combine scheme within 1e-6 relative of FP64 (sum,
sumsq, mean; variance relative to max(var, 1e-12 * sumsq / n)), as the
single-partition moments tests.  A request gives the same bits alone and in
a mix of concurrent requests.
"""

import time

import numpy as np
import pytest

from cases import random_csr, to_device_csr

pytestmark = pytest.mark.gpu

RTOL = 1e-6
CUTS = [0, 3000, 3000, 4234, 4251, 10251]  # 5 partitions, one of them empty
COLS = 300


@pytest.fixture(scope="module")
def staged(cuda):
    from cellshard_b200.device import blocked_ell_from_csr

    rows = CUTS[-1]
    ptr, idx, val = random_csr(rows, COLS, 0.06, 77, 0.1, integer=False)
    parts = []
    for a, b in zip(CUTS[:-1], CUTS[1:]):
        pp = (ptr[a:b + 1] - ptr[a]).astype(np.uint32)
        parts.append(blocked_ell_from_csr(to_device_csr(b - a, COLS, pp, idx[ptr[a]:ptr[b]], val[ptr[a]:ptr[b]]), 16))
    return rows, ptr, idx, val, parts


def _inputs(rows, G, seed, keep=0.7, fkeep=None, bad_labels=True):
    rng = np.random.default_rng(seed)
    rk = (rng.random(rows) < keep).astype(np.uint8)
    lab = rng.integers(0, G + (2 if bad_labels else 0), rows).astype(np.uint32)
    fk = None if fkeep is None else (rng.random(COLS) < fkeep).astype(np.uint8)
    return rk, lab, fk


def _check(res, ref, rtol=RTOL):
    n = res["group_rows"].astype(np.int64)
    assert np.array_equal(n, ref["group_rows"].astype(np.int64))
    for k in ("sum", "sumsq", "mean"):
        got, exp = res[k].astype(np.float64), ref[k]
        err = np.abs(got - exp) / np.maximum(np.abs(exp), 1e-30)
        assert np.all((err <= rtol) | (np.abs(got - exp) <= 1e-30)), (k, float(err.max()))
    got, exp = res["var"].astype(np.float64), ref["var"]
    scale = np.maximum(np.abs(exp), 1e-12 * ref["sumsq"] / np.maximum(n, 1)[:, None])
    err = np.abs(got - exp) / np.maximum(scale, 1e-30)
    assert np.all((err <= rtol) | (np.abs(got - exp) == 0)), ("var", float(err.max()))


def test_serve_matches_oracle(staged, orc):
    from cellshard_b200.serve import Request, Server

    rows, ptr, idx, val, parts = staged
    srv = Server(parts, scratch_budget_bytes=1 << 30, chunk_rows=64)
    try:
        reqs = []
        for k, G in enumerate([1, 5, 37, 300]):
            rk, lab, fk = _inputs(rows, G, 10 + k, fkeep=0.8 if k % 2 else None)
            reqs.append((Request(G, rk, lab, fk, COLS), rk, lab, fk, G))
        tickets = [srv.submit(r[0]) for r in reqs]
        for t in tickets:
            srv.wait(t)
        for req, rk, lab, fk, G in reqs:
            ref = orc.group_moments_csr(rows, COLS, ptr, idx, val, rk, fk, lab, G, ddof=1, nthreads=4)
            _check(req.results(), ref)
        st = srv.stats()
        assert st["completed"] == 4 and st["scratch_in_use"] == 0 and st["device_error"] == 0
    finally:
        srv.close()


def test_serve_same_alone_and_in_mix(staged, orc):
    from cellshard_b200.serve import Request, Server

    rows, ptr, idx, val, parts = staged
    srv = Server(parts, scratch_budget_bytes=2 << 30, chunk_rows=128)
    try:
        rk, lab, fk = _inputs(rows, 17, 5, fkeep=0.9)
        alone = Request(17, rk, lab, fk, COLS)
        srv.wait(srv.submit(alone))
        a_res = alone.results()
        mix = []
        for k in range(12):
            G = [2, 64, 300, 9][k % 4]
            rki, labi, fki = _inputs(rows, G, 100 + k, keep=0.2 + 0.06 * k)
            mix.append((Request(G, rki, labi, fki, COLS), rki, labi, fki, G))
        again = Request(17, rk, lab, fk, COLS)
        tickets = [srv.submit(m[0]) for m in mix[:6]] + [srv.submit(again)] + [srv.submit(m[0]) for m in mix[6:]]
        for t in tickets:
            srv.wait(t)
        b_res = again.results()
        for key in ("sum", "sumsq", "mean", "var"):
            assert np.array_equal(a_res[key].view(np.uint32), b_res[key].view(np.uint32)), key
        for req, rki, labi, fki, G in mix[::3]:
            ref = orc.group_moments_csr(rows, COLS, ptr, idx, val, rki, fki, labi, G, ddof=1, nthreads=4)
            _check(req.results(), ref)
        _check(a_res, orc.group_moments_csr(rows, COLS, ptr, idx, val, rk, fk, lab, 17, ddof=1, nthreads=4))
    finally:
        srv.close()


def test_serve_budget_admission_queues_requests(staged, orc):
    from cellshard_b200.serve import Request, Server

    rows, ptr, idx, val, parts = staged
    # a budget that admits about two of these requests at a time
    srv = Server(parts, scratch_budget_bytes=1 << 30, max_inflight=4)
    try:
        reqs = [Request(8, *_inputs(rows, 8, 200 + k)[:2], None, COLS) for k in range(10)]
        tickets = [srv.submit(r) for r in reqs]
        lat = [srv.wait(t) for t in tickets]
        st = srv.stats()
        assert st["admitted"] == 10 and st["completed"] == 10 and st["pending"] == 0 and st["scratch_in_use"] == 0
        assert all(x > 0 for x in lat)
        rk, lab = _inputs(rows, 8, 209)[:2]
        _check(reqs[9].results(), orc.group_moments_csr(rows, COLS, ptr, idx, val, rk, None, lab, 8, ddof=1))
    finally:
        srv.close()
    # a request larger than the whole budget is refused at submit
    small = Server(parts, scratch_budget_bytes=1 << 20)
    try:
        with pytest.raises(Exception):
            small.submit(Request(300, *_inputs(rows, 300, 1)[:2], None, COLS))
    finally:
        small.close()


@pytest.mark.parametrize("scheme,rtol", [(0, 1e-5), (1, 1e-6)])
def test_serve_fp32_schemes(staged, orc, scheme, rtol):
    from cellshard_b200.serve import Request, Server

    rows, ptr, idx, val, parts = staged
    srv = Server(parts, scratch_budget_bytes=1 << 30)
    try:
        rk, lab, fk = _inputs(rows, 6, 31, fkeep=0.5)
        req = Request(6, rk, lab, fk, COLS, scheme=scheme)
        srv.wait(srv.submit(req))
        res = req.results()
        ref = orc.group_moments_csr(rows, COLS, ptr, idx, val, rk, fk, lab, 6, ddof=1)
        for k in ("sum", "sumsq"):
            got, exp = res[k].astype(np.float64), ref[k]
            assert np.allclose(got, exp, rtol=rtol, atol=0), k
        assert np.all(res["sum"][:, fk == 0] == 0)
    finally:
        srv.close()


def test_serve_idle_exit_and_relaunch(staged, orc):
    from cellshard_b200.serve import Request, Server

    rows, ptr, idx, val, parts = staged
    srv = Server(parts, scratch_budget_bytes=1 << 30, idle_exit_us=2000)
    try:
        rk, lab, _ = _inputs(rows, 3, 41)
        a = Request(3, rk, lab, None, COLS)
        srv.wait(srv.submit(a))
        time.sleep(0.1)  # the loop exits after 2 ms idle
        b = Request(3, rk, lab, None, COLS)
        srv.wait(srv.submit(b))
        assert srv.stats()["kernel_launches"] >= 2
        assert np.array_equal(a.results()["sum"], b.results()["sum"])
    finally:
        srv.close()


def test_serve_device_inputs_and_outputs(staged, orc):
    import ctypes as C

    import torch

    from cellshard_b200 import _abi
    from cellshard_b200.serve import Server

    rows, ptr, idx, val, parts = staged
    srv = Server(parts, scratch_budget_bytes=1 << 30)
    try:
        G = 4
        rk, lab, fk = _inputs(rows, G, 51, fkeep=0.7)
        d_rk = torch.from_numpy(rk).cuda()
        d_lab = torch.from_numpy(lab.view(np.int32)).cuda()
        d_fk = torch.from_numpy(fk).cuda()
        out = {k: torch.empty((G, COLS), dtype=torch.float32, device="cuda") for k in ("sum", "sumsq", "mean", "var")}
        gr = torch.empty(G, dtype=torch.int32, device="cuda")
        req = _abi.ServeRequest(G, 2, 1, _abi.SERVE_DEVICE_INPUTS | _abi.SERVE_DEVICE_OUTPUTS, d_rk.data_ptr(),
                                d_lab.data_ptr(), d_fk.data_ptr(), out["sum"].data_ptr(), out["sumsq"].data_ptr(),
                                out["mean"].data_ptr(), out["var"].data_ptr(), gr.data_ptr())
        t = _abi.u64()
        _abi.check(srv.lib.cs_b200_serve_submit(srv.handle, C.byref(req), C.byref(t)), "submit")
        srv.wait(t.value)
        res = {k: v.cpu().numpy() for k, v in out.items()}
        res["group_rows"] = gr.cpu().numpy().view(np.uint32)
        _check(res, orc.group_moments_csr(rows, COLS, ptr, idx, val, rk, fk, lab, G, ddof=1))
    finally:
        srv.close()
