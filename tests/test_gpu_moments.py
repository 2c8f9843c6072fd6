"""Grouped per-feature moments on the GPU vs the FP64 oracle (oracle/cs_oracle.c).

Tolerance: the compensated schemes must match the FP64 oracle within 1e-6
relative (sum, sumsq, mean, variance; variance relative to max(var, 1e-12 *
sumsq / n) so that exact zeros compare absolutely).  Integer-valued data
makes sum and sumsq exact in FP64, so those must match to the fp32 rounding
of the exact value.
"""

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def _bell(cuda, rows, cols, B, density=0.1, seed=0, integer=True, empty=0.1):
    from cellshard_b200.device import blocked_ell_from_csr

    ptr, idx, val = random_csr(rows, cols, density, seed, empty, integer)
    csr = to_device_csr(rows, cols, ptr, idx, val)
    return blocked_ell_from_csr(csr, B)


def _host(bell):
    return np_u32(bell.bci), np_u16(bell.val)


def _masks(rows, cols, G, seed, keep=0.7, fkeep=0.8):
    rng = np.random.default_rng(seed)
    rk = (rng.random(rows) < keep).astype(np.uint8)
    fk = (rng.random(cols) < fkeep).astype(np.uint8)
    lab = rng.integers(0, G, rows).astype(np.uint32)
    return rk, fk, lab


def _dev(a):
    import torch

    if a is None:
        return None
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    return torch.from_numpy(a.copy()).cuda()


def _check(res, ref, G, cols, rtol=RTOL):
    import torch

    torch.cuda.synchronize()
    assert int(res["status"].item()) == 0
    n = res["group_rows"].cpu().numpy().astype(np.int64)
    assert np.array_equal(n, ref["group_rows"].astype(np.int64))
    for k in ("sum", "sumsq", "mean"):
        got = res[k].cpu().numpy().astype(np.float64)
        exp = ref[k]
        err = np.abs(got - exp) / np.maximum(np.abs(exp), 1e-30)
        assert np.all((err <= rtol) | (np.abs(got - exp) <= 1e-30)), (k, float(err.max()))
    got = res["var"].cpu().numpy().astype(np.float64)
    exp = ref["var"]
    scale = np.maximum(np.abs(exp), 1e-12 * ref["sumsq"] / np.maximum(n, 1)[:, None])
    err = np.abs(got - exp) / np.maximum(scale, 1e-30)
    assert np.all((err <= rtol) | (np.abs(got - exp) == 0)), ("var", float(err.max()))


@pytest.mark.parametrize("B", [1, 2, 3, 4, 8, 16, 32])
def test_moments_block_sizes(cuda, orc, B):
    from cellshard_b200 import runtime

    rows, cols, G = 301, 203, 5
    bell = _bell(cuda, rows, cols, B, 0.08, seed=B)
    rk, fk, lab = _masks(rows, cols, G, B)
    bci, val = _host(bell)
    ref = orc.group_moments_bell(rows, cols, B, bell.ell_cols, bci, val, rk, fk, lab, G, ddof=1)
    for scheme in (runtime.TWOSUM_F32, runtime.TWOSUM_F64_COMBINE):
        res = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), scheme=scheme, ddof=1)
        _check(res, ref, G, cols)


def test_moments_many_chunks_and_determinism(cuda, orc):
    from cellshard_b200 import runtime

    rows, cols, G = 5000, 257, 7
    bell = _bell(cuda, rows, cols, 16, 0.05, seed=42, integer=False)
    rk, fk, lab = _masks(rows, cols, G, 7)
    bci, val = _host(bell)
    ref = orc.group_moments_bell(rows, cols, 16, bell.ell_cols, bci, val, rk, fk, lab, G, ddof=0, nthreads=4)
    a = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), ddof=0, chunk_rows=64)
    _check(a, ref, G, cols)
    b = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), ddof=0, chunk_rows=64)
    for k in ("sum", "sumsq", "mean", "var"):
        assert np.array_equal(a[k].cpu().numpy().view(np.uint32), b[k].cpu().numpy().view(np.uint32)), k
    c = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), ddof=0)
    _check(c, ref, G, cols)


def test_moments_edge_cases(cuda, orc):
    import torch

    from cellshard_b200 import runtime

    rows, cols, G = 200, 100, 3
    bell = _bell(cuda, rows, cols, 16, 0.1, seed=5)
    bci, val = _host(bell)
    # all rows masked out
    rk = np.zeros(rows, np.uint8)
    res = runtime.compute_sparse_group_moments(bell, G, _dev(rk), None, None)
    torch.cuda.synchronize()
    assert float(res["sum"].abs().sum()) == 0.0 and int(res["group_rows"].sum()) == 0
    # labels >= G are ignored; no masks at all; one group
    lab = np.random.default_rng(1).integers(0, G + 2, rows).astype(np.uint32)
    ref = orc.group_moments_bell(rows, cols, 16, bell.ell_cols, bci, val, None, None, lab, G, ddof=1)
    res = runtime.compute_sparse_group_moments(bell, G, None, None, _dev(lab))
    _check(res, ref, G, cols)
    ref1 = orc.group_moments_bell(rows, cols, 16, bell.ell_cols, bci, val, None, None, None, 1, ddof=1)
    res1 = runtime.compute_sparse_group_moments(bell, 1)
    _check(res1, ref1, 1, cols)
    # feature mask all zero
    res0 = runtime.compute_sparse_group_moments(bell, G, None, _dev(np.zeros(cols, np.uint8)), _dev(lab))
    torch.cuda.synchronize()
    assert float(res0["sumsq"].abs().sum()) == 0.0


def test_moments_empty_matrix(cuda):
    import torch

    from cellshard_b200 import runtime
    from cellshard_b200.device import BlockedELL

    e = BlockedELL(0, 50, 16, 0, torch.zeros(0, dtype=torch.int32, device="cuda"),
                   torch.zeros(0, dtype=torch.float16, device="cuda"))
    res = runtime.compute_sparse_group_moments(e, 4)
    torch.cuda.synchronize()
    assert float(res["sum"].abs().sum()) == 0.0 and int(res["group_rows"].sum()) == 0


def test_moments_plain_scheme_close_to_fp64(cuda, orc):
    from cellshard_b200 import runtime

    rows, cols, G = 3000, 64, 4
    bell = _bell(cuda, rows, cols, 16, 0.3, seed=9)
    rk, fk, lab = _masks(rows, cols, G, 3)
    bci, val = _host(bell)
    ref = orc.group_moments_bell(rows, cols, 16, bell.ell_cols, bci, val, rk, fk, lab, G, ddof=1)
    res = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), scheme=runtime.PLAIN_F32)
    s = res["sum"].cpu().numpy()
    assert np.allclose(s, ref["sum"], rtol=1e-5)


def test_moments_generated_matrix(cuda, orc):
    """Seeded NB/Zipf matrix generated on the GPU, 2,048 x 2,000 at block 16."""
    from cellshard_b200 import runtime, synth
    from cellshard_b200.device import blocked_ell_from_csr

    spec = synth.plain_conversion_spec()
    spec.rows = 2048
    csr = synth.make_csr(spec)
    bell = blocked_ell_from_csr(csr, 16)
    G = 64
    rk, fk, lab = synth.masks_and_labels(spec.rows, spec.cols, G, kept_features=1500)
    bci, val = _host(bell)
    ref = orc.group_moments_bell(spec.rows, spec.cols, 16, bell.ell_cols, bci, val, rk, fk, lab, G, ddof=1,
                                 nthreads=4)
    res = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab))
    _check(res, ref, G, spec.cols)


@pytest.mark.parametrize("parts", [0, 1, 2, 3, 7])
def test_moments_to_host_matches_device_call(cuda, orc, parts):
    """The host-delivery entry point (groups in `parts` ranges, each range's rows copied
    while the next computes) returns the device-only call's results bit for bit, in
    pinned host memory, and both match the FP64 oracle."""
    import torch

    from cellshard_b200 import runtime

    rows, cols, G = 3000, 203, 7
    bell = _bell(cuda, rows, cols, 16, 0.06, seed=parts + 3, integer=False)
    rk, fk, lab = _masks(rows, cols, G, parts + 11)
    bci, val = _host(bell)
    ref = orc.group_moments_bell(rows, cols, 16, bell.ell_cols, bci, val, rk, fk, lab, G, ddof=1)
    want = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), ddof=1, chunk_rows=128,
                                                want_f64=True)
    host = {k: torch.empty((G, cols), dtype=torch.float32).pin_memory() for k in ("sum", "sumsq", "mean", "var")}
    host["mean64"] = torch.empty((G, cols), dtype=torch.float64).pin_memory()
    host["group_rows"] = torch.empty(G, dtype=torch.int32).pin_memory()
    host["status"] = torch.full((1,), -1, dtype=torch.int32).pin_memory()
    runtime.compute_sparse_group_moments_to_host(bell, G, host, _dev(rk), _dev(fk), _dev(lab), ddof=1,
                                                 chunk_rows=128, parts=parts)
    torch.cuda.synchronize()
    for k in ("sum", "sumsq", "mean", "var", "mean64", "group_rows"):
        a, b = host[k].numpy(), want[k].cpu().numpy()
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
    assert int(host["status"][0]) == 0
    _check(host, ref, G, cols)


@pytest.mark.parametrize("chunk_rows", [64, 0])
def test_moments_headline_layout(cuda, orc, chunk_rows):
    """The headline workload's layout on 20,000 rows: 32,768 columns at ~4 % density as
    Blocked-ELL-16 (ell_width near the 2,048 block columns), 64 uniform groups, a
    Bernoulli(0.7) row mask and 20,000 kept features.  Chunks of 64 rows give every group
    three or more chunks, so the fp64 cross-chunk combine is exercised; 0 is the library's
    default chunking, as the headline runs it."""
    from cellshard_b200 import runtime, synth
    from cellshard_b200.device import blocked_ell_from_csr

    G = 64
    spec = synth.grouped_reduction_spec(20000)
    csr = synth.make_csr(spec)
    bell = blocked_ell_from_csr(csr, 16)
    del csr
    assert bell.cols == 32768 and bell.ell_width >= 1900
    rk, fk, lab = synth.masks_and_labels(spec.rows, spec.cols, G, 0.7, 20000)
    per_group = np.bincount(lab[rk == 1], minlength=G)
    if chunk_rows:
        assert int(per_group.min()) > 2 * chunk_rows
    bci, val = _host(bell)
    ref = orc.group_moments_bell(spec.rows, spec.cols, 16, bell.ell_cols, bci, val, rk, fk, lab, G, ddof=1,
                                 nthreads=orc.cpu_count())
    res = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), ddof=1, chunk_rows=chunk_rows)
    _check(res, ref, G, spec.cols)
    err = orc.moments_max_rel({k: res[k].cpu().numpy() for k in ("sum", "sumsq", "mean", "var")}, ref)
    assert max(err.values()) <= RTOL, err



def test_moments_prebuilt_index_matches(cuda, orc):
    """A column-block index built once for the partition (build_moments_index) gives the
    same bits as the index each call builds, for the one-shot call, the phases and the
    host-delivery call, over repeated requests."""
    import torch

    from cellshard_b200 import runtime

    rows, cols, G = 3000, 203, 7
    bell = _bell(cuda, rows, cols, 16, 0.06, seed=21, integer=False)
    idx = runtime.build_moments_index(bell)
    for seed in (1, 2):
        rk, fk, lab = _masks(rows, cols, G, seed)
        a = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), chunk_rows=128)
        b = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), chunk_rows=128, index=idx)
        ws = runtime.MomentsWorkspace()
        c = None
        for ph in (runtime.PHASE_PREPARE, runtime.PHASE_ACCUMULATE, runtime.PHASE_COMBINE):
            c = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), chunk_rows=128,
                                                     index=idx, workspace=ws, out=c, phases=ph)
        host = {k: torch.empty((G, cols), dtype=torch.float32).pin_memory() for k in ("sum", "sumsq", "mean", "var")}
        runtime.compute_sparse_group_moments_to_host(bell, G, host, _dev(rk), _dev(fk), _dev(lab), chunk_rows=128,
                                                     index=idx)
        torch.cuda.synchronize()
        for k in ("sum", "sumsq", "mean", "var"):
            want = a[k].cpu().numpy().view(np.uint32)
            assert np.array_equal(b[k].cpu().numpy().view(np.uint32), want), k
            assert np.array_equal(c[k].cpu().numpy().view(np.uint32), want), k
            assert np.array_equal(host[k].numpy().view(np.uint32), want), k
        bci, val = _host(bell)
        ref = orc.group_moments_bell(rows, cols, 16, bell.ell_cols, bci, val, rk, fk, lab, G, ddof=1)
        _check(b, ref, G, cols)


@pytest.mark.parametrize("prebuilt", [False, True])
def test_moments_over_shard_partitions(cuda, orc, prebuilt):
    """One call over a shard of uneven partitions (rows not multiples of the block size,
    different ell_cols): the FP64 oracle over the partitions stacked row-wise; prebuilt
    per-partition indexes give the same bits as indexes built by the call."""
    import torch

    from cellshard_b200 import runtime

    cols, G, B = 203, 6, 16
    rows = [301, 64, 17, 540]
    parts = [_bell(cuda, r, cols, B, 0.03 + 0.02 * k, seed=50 + k, integer=(k % 2 == 0)) for k, r in enumerate(rows)]
    R = sum(rows)
    rk, fk, lab = _masks(R, cols, G, 9)
    idx = [runtime.build_moments_index(q) for q in parts] if prebuilt else None
    res = runtime.compute_sparse_group_moments_parts(parts, G, _dev(rk), _dev(fk), _dev(lab), chunk_rows=64,
                                                     indexes=idx)
    # the oracle over the stacked partitions: FP64 sums per partition, added
    s = np.zeros((G, cols))
    q = np.zeros((G, cols))
    n = np.zeros(G, np.int64)
    r0 = 0
    for part, r in zip(parts, rows):
        bci, val = _host(part)
        o = orc.group_moments_bell(r, cols, B, part.ell_cols, bci, val, rk[r0:r0 + r], None, lab[r0:r0 + r], G)
        s += o["sum"]
        q += o["sumsq"]
        n += o["group_rows"].astype(np.int64)
        r0 += r
    keep = fk.astype(bool)
    s[:, ~keep] = 0.0
    q[:, ~keep] = 0.0
    nn = n[:, None].astype(np.float64)
    mean = np.where(nn > 0, s / np.maximum(nn, 1), 0.0)
    var = np.where(nn > 1, np.maximum(q - s * mean, 0.0) / np.maximum(nn - 1, 1), 0.0)
    mean[:, ~keep] = 0.0
    var[:, ~keep] = 0.0
    ref = {"sum": s, "sumsq": q, "mean": mean, "var": var, "group_rows": n.astype(np.uint32)}
    _check(res, ref, G, cols)
    again = runtime.compute_sparse_group_moments_parts(parts, G, _dev(rk), _dev(fk), _dev(lab), chunk_rows=64,
                                                       indexes=[runtime.build_moments_index(q_) for q_ in parts])
    torch.cuda.synchronize()
    for k in ("sum", "sumsq", "mean", "var"):
        assert np.array_equal(res[k].cpu().numpy().view(np.uint32), again[k].cpu().numpy().view(np.uint32)), k


def test_moments_one_partition_shard_matches_single_call(cuda):
    """A shard of one partition is the single-partition reduction, bit for bit."""
    from cellshard_b200 import runtime

    rows, cols, G = 1000, 150, 5
    bell = _bell(cuda, rows, cols, 16, 0.05, seed=77, integer=False)
    rk, fk, lab = _masks(rows, cols, G, 4)
    a = runtime.compute_sparse_group_moments(bell, G, _dev(rk), _dev(fk), _dev(lab), chunk_rows=128)
    b = runtime.compute_sparse_group_moments_parts([bell], G, _dev(rk), _dev(fk), _dev(lab), chunk_rows=128)
    for k in ("sum", "sumsq", "mean", "var", "group_rows"):
        assert np.array_equal(a[k].cpu().numpy().view(np.uint32), b[k].cpu().numpy().view(np.uint32)), k
