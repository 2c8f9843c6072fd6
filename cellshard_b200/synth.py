"""Seeded synthetic cell x gene matrices.

Row nnz ~ round(lognormal(mu = ln(mean) - sigma^2 / 2, sigma)), clipped; the
row's columns are drawn without replacement from Zipf(s) gene popularity (a
seeded rank -> column permutation spreads popular genes over the column
range) and sorted; values are zero-truncated negative-binomial counts
(mean 2, dispersion 0.5, i.e. size 2) rounded to fp16, optionally scaled per
row.  The host computes the per-row counts and the integer CDF tables; the
column and value draws run on the GPU (cs_b200_synth_csr), so large
matrices are generated in HBM.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SEED_BASE = 20261203


def row_nnz(rows: int, mean: float, sigma: float, lo: int, hi: int, rng: np.random.Generator) -> np.ndarray:
    mu = math.log(mean) - sigma * sigma / 2.0
    x = np.rint(rng.lognormal(mu, sigma, size=rows))
    return np.clip(x, lo, hi).astype(np.uint32)


def _cdf_u53(p: np.ndarray) -> np.ndarray:
    c = np.cumsum(p / p.sum(), dtype=np.float64)
    t = np.minimum(np.rint(c * 2.0 ** 53), 2.0 ** 53).astype(np.uint64)
    t = np.maximum.accumulate(t)
    t[-1] = np.uint64(1 << 53)
    return t


def zipf_cdf_u53(cols: int, s: float = 1.1) -> np.ndarray:
    ranks = np.arange(1, cols + 1, dtype=np.float64)
    return _cdf_u53(ranks ** (-s))


def nb_cdf_u53(mean: float = 2.0, dispersion: float = 0.5, max_count: int = 256) -> np.ndarray:
    """CDF of the zero-truncated NB on counts 1..max_count (bucket i -> count i+1)."""
    r = 1.0 / dispersion
    p = r / (r + mean)
    k = np.arange(0, max_count + 1, dtype=np.float64)
    logpmf = (np.array([math.lgamma(x + r) - math.lgamma(r) - math.lgamma(x + 1.0) for x in k])
              + r * math.log(p) + k * math.log1p(-p))
    pmf = np.exp(logpmf)[1:]
    return _cdf_u53(pmf)


@dataclass
class MatrixSpec:
    rows: int
    cols: int
    mean_nnz: float
    lo: int
    hi: int
    sigma: float = 0.6
    zipf_s: float = 1.1
    outlier_frac: float = 0.0
    outlier_scale: float = 100.0
    seed: int = SEED_BASE


def plain_conversion_spec() -> MatrixSpec:
    """8,192 x 2,000, nnz/row lognormal mean 120 (sigma 0.6) clipped to [10, 1000]."""
    return MatrixSpec(8192, 2000, 120.0, 10, 1000, seed=SEED_BASE + 1)


def grouped_reduction_spec(rows: int = 500_000) -> MatrixSpec:
    """500,000 x 32,768 at ~4 % density (mean 1,311 nnz/row)."""
    cols = 32768
    return MatrixSpec(rows, cols, 0.04 * cols, 1, cols // 2, seed=SEED_BASE + 2)


def precision_spec(rows: int = 1_000_000) -> MatrixSpec:
    """1,000,000 x 32,768 at ~3 %, 1 % of rows scaled x100."""
    cols = 32768
    return MatrixSpec(rows, cols, 0.03 * cols, 1, cols // 2, outlier_frac=0.01, seed=SEED_BASE + 4)


def host_tables(spec: MatrixSpec):
    """(row_nnz, row_ptr, col_cdf, col_of_rank, val_cdf, row_scale|None) as numpy arrays."""
    rng = np.random.default_rng(spec.seed)
    nnz = row_nnz(spec.rows, spec.mean_nnz, spec.sigma, spec.lo, min(spec.hi, spec.cols), rng)
    ptr = np.zeros(spec.rows + 1, dtype=np.uint64)
    np.cumsum(nnz, out=ptr[1:])
    if ptr[-1] >= 2 ** 32:
        raise ValueError("nnz exceeds the u32 index range of one partition")
    col_cdf = zipf_cdf_u53(spec.cols, spec.zipf_s)
    col_of_rank = rng.permutation(spec.cols).astype(np.uint32)
    val_cdf = nb_cdf_u53()
    scale = None
    if spec.outlier_frac > 0:
        scale = np.ones(spec.rows, dtype=np.float32)
        pick = rng.random(spec.rows) < spec.outlier_frac
        scale[pick] = np.float32(spec.outlier_scale)
    return nnz, ptr.astype(np.uint32), col_cdf, col_of_rank, val_cdf, scale


_COL_SALT = 0x636F6C756D6E73
_VAL_SALT = 0x76616C7565737321


def _splitmix64(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _draw_u53(key: np.uint64, row: int, j: np.ndarray) -> np.ndarray:
    return _splitmix64(key ^ ((np.uint64(row) << np.uint64(32)) | j.astype(np.uint64))) >> np.uint64(11)


def host_rows(spec: MatrixSpec, tables, r0: int, r1: int):
    """Rows [r0, r1) of the matrix cs_b200_synth_csr generates, computed on the host
    with the same draws (bit-identical); returns (ptr, idx, val_bits)."""
    nnz, rp, col_cdf, col_of_rank, val_cdf, scale = tables
    cols = spec.cols
    col_key = _splitmix64(np.array([spec.seed ^ _COL_SALT], np.uint64))[0]
    val_key = _splitmix64(np.array([spec.seed ^ _VAL_SALT], np.uint64))[0]
    max_draws = ((64 * cols + 1024) // 32) * 32
    base = int(rp[r0])
    ptr = (rp[r0:r1 + 1].astype(np.int64) - base).astype(np.uint32)
    idx = np.empty(int(ptr[-1]), np.uint32)
    val = np.empty(int(ptr[-1]), np.uint16)
    for r in range(r0, r1):
        need = min(int(nnz[r]), cols)
        chosen = np.zeros(cols, bool)
        count, j0 = 0, 0
        while count < need and j0 < max_draws:
            batch = min(max(256, 4 * (need - count)), max_draws - j0)
            j = np.arange(j0, j0 + batch, dtype=np.uint64)
            c = col_of_rank[np.searchsorted(col_cdf, _draw_u53(col_key, r, j), side="right")]
            first = np.zeros(batch, bool)
            first[np.unique(c, return_index=True)[1]] = True
            acc = np.flatnonzero(first & ~chosen[c])[:need - count]
            chosen[c[acc]] = True
            count += len(acc)
            j0 += batch
        if count < need:
            chosen[np.flatnonzero(~chosen)[:need - count]] = True
        cs = np.flatnonzero(chosen).astype(np.uint32)
        k = np.searchsorted(val_cdf, _draw_u53(val_key, r, np.arange(need, dtype=np.uint64)), side="right") + 1
        sc = np.float32(scale[r]) if scale is not None else np.float32(1.0)
        a, b = int(ptr[r - r0]), int(ptr[r - r0 + 1])
        idx[a:b] = cs
        val[a:b] = (k.astype(np.float32) * sc).astype(np.float16).view(np.uint16)
    return ptr, idx, val


def make_csr(spec: MatrixSpec, stream=None):
    """Generates the matrix on the current CUDA device; returns device.CSR."""
    import torch

    from . import _abi
    from .device import CSR, ptr, stream_handle, u32

    _nnz, rp, col_cdf, col_of_rank, val_cdf, scale = host_tables(spec)
    total = int(rp[-1])
    d_ptr = u32(rp)
    d_cdf = torch.from_numpy(col_cdf.view(np.int64).copy()).cuda()
    d_rank = u32(col_of_rank)
    d_vcdf = torch.from_numpy(val_cdf.view(np.int64).copy()).cuda()
    d_scale = torch.from_numpy(scale).cuda() if scale is not None else None
    idx = torch.empty(total, dtype=torch.int32, device="cuda")
    val = torch.empty(total, dtype=torch.float16, device="cuda")
    lib = _abi.load()
    _abi.check(lib.cs_b200_synth_csr(spec.rows, spec.cols, ptr(d_ptr), ptr(d_cdf), ptr(d_rank), ptr(d_vcdf),
                                     len(val_cdf), ptr(d_scale), spec.seed, ptr(idx), ptr(val),
                                     stream_handle(stream)), "synth_csr")
    return CSR(spec.rows, spec.cols, d_ptr, idx, val)


def masks_and_labels(rows: int, cols: int, groups: int, keep_frac: float = 0.7, kept_features: int = 20000,
                     seed: int = SEED_BASE + 20):
    """Row mask ~ Bernoulli(keep_frac), `kept_features` random kept columns, uniform labels (numpy)."""
    rng = np.random.default_rng(seed)
    row_keep = (rng.random(rows) < keep_frac).astype(np.uint8)
    feature_keep = np.zeros(cols, dtype=np.uint8)
    feature_keep[rng.choice(cols, size=min(kept_features, cols), replace=False)] = 1
    labels = rng.integers(0, groups, size=rows, dtype=np.uint32)
    return row_keep, feature_keep, labels
