"""The FP64 grouped-moments oracle itself (CPU): numpy restatement agreement,
thread-count independence, unsorted rows, and the Blocked-ELL and CSR forms
agreeing on the same matrix."""

import numpy as np
import pytest

from cases import random_csr


def _numpy_moments(rows, cols, ptr, idx, val, rk, fk, lab, G, ddof):
    x = val.view(np.float16).astype(np.float64)
    s = np.zeros((G, cols))
    q = np.zeros((G, cols))
    n = np.zeros(G, np.int64)
    for r in range(rows):
        if rk is not None and not rk[r]:
            continue
        g = int(lab[r]) if lab is not None else 0
        if g >= G:
            continue
        n[g] += 1
        a, b = int(ptr[r]), int(ptr[r + 1])
        for i in range(a, b):
            s[g, idx[i]] += x[i]
            q[g, idx[i]] += x[i] * x[i]
    if fk is not None:
        s[:, fk == 0] = 0
        q[:, fk == 0] = 0
    nn = n[:, None].astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        m = np.where(nn > 0, s / np.maximum(nn, 1), 0.0)
        m2 = np.maximum(q - s * m, 0.0)
        v = np.where(nn > ddof, m2 / np.maximum(nn - ddof, 1), 0.0)
    if fk is not None:
        m[:, fk == 0] = 0
        v[:, fk == 0] = 0
    return s, q, m, v, n


@pytest.mark.parametrize("unsorted", [0, 7])
def test_csr_oracle_vs_numpy_and_thread_count(orc, unsorted):
    rows, cols, G = 400, 97, 6
    ptr, idx, val = random_csr(rows, cols, 0.1, 11, 0.1, integer=False, unsorted_rows=unsorted)
    rng = np.random.default_rng(2)
    rk = (rng.random(rows) < 0.8).astype(np.uint8)
    fk = (rng.random(cols) < 0.9).astype(np.uint8)
    lab = rng.integers(0, G + 1, rows).astype(np.uint32)
    s, q, m, v, n = _numpy_moments(rows, cols, ptr, idx, val, rk, fk, lab, G, 1)
    one = orc.group_moments_csr(rows, cols, ptr, idx, val, rk, fk, lab, G, ddof=1, nthreads=1)
    many = orc.group_moments_csr(rows, cols, ptr, idx, val, rk, fk, lab, G, ddof=1, nthreads=5)
    assert np.array_equal(one["group_rows"], n.astype(np.uint32))
    for k, ref in (("sum", s), ("sumsq", q), ("mean", m), ("var", v)):
        assert np.array_equal(one[k], many[k]), k
        assert np.array_equal(one[k], ref), k  # same order of additions -> identical doubles


def test_bell_oracle_matches_csr_oracle(orc):
    rows, cols, G, B = 333, 150, 4, 16
    ptr, idx, val = random_csr(rows, cols, 0.07, 5, 0.1, integer=True)
    bell = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
    bci, bval, ell_cols = bell["bci"], bell["val"], bell["ell_cols"]
    rng = np.random.default_rng(9)
    rk = (rng.random(rows) < 0.7).astype(np.uint8)
    lab = rng.integers(0, G, rows).astype(np.uint32)
    a = orc.group_moments_csr(rows, cols, ptr, idx, val, rk, None, lab, G, ddof=0, nthreads=3)
    b = orc.group_moments_bell(rows, cols, B, ell_cols, bci, bval, rk, None, lab, G, ddof=0, nthreads=4)
    for k in ("sum", "sumsq", "mean", "var", "group_rows"):
        assert np.array_equal(a[k], b[k]), k


def test_moments_slab_oracle_matches_one_call(orc):
    """The slab-accumulated FP64 oracle the benchmark uses over its full partition equals
    one oracle call over all rows (integer counts: exact sums)."""
    rows, cols, B, G = 301, 70, 16, 4
    ptr, idx, val = random_csr(rows, cols, 0.2, 3, 0.1, True)
    oracle = orc
    b = oracle.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
    W = b["ell_cols"] // B
    rng = np.random.default_rng(1)
    rk = (rng.random(rows) < 0.7).astype(np.uint8)
    fk = (rng.random(cols) < 0.8).astype(np.uint8)
    lab = rng.integers(0, G, rows).astype(np.uint32)
    one = oracle.group_moments_bell(rows, cols, B, b["ell_cols"], b["bci"], b["val"], rk, fk, lab, G, ddof=1)
    fetch = lambda r0, r1: (b["bci"][(r0 // B) * W:((r1 + B - 1) // B) * W], b["val"][r0 * b["ell_cols"]:
                                                                                     r1 * b["ell_cols"]])
    slabs = oracle.group_moments_bell_slabs(fetch, rows, cols, B, b["ell_cols"], rk, fk, lab, G, ddof=1, slab_rows=64)
    for k in ("sum", "sumsq", "mean", "var"):
        assert np.allclose(slabs[k], one[k], rtol=1e-15, atol=0), k
    assert np.array_equal(slabs["group_rows"], one["group_rows"])
    assert max(oracle.moments_max_rel(slabs, one).values()) <= 1e-15
