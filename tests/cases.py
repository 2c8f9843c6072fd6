"""Seeded small sparse inputs for parity tests (numpy, host side)."""

from __future__ import annotations

import numpy as np


def random_csr(rows, cols, density=0.05, seed=0, empty_frac=0.1, integer=True, dup_rows=0, unsorted_rows=0,
               max_row=None):
    """CSR (ptr, idx, val_bits) with sorted unique columns unless dup/unsorted rows are requested."""
    rng = np.random.default_rng(seed)
    ptr = np.zeros(rows + 1, np.uint32)
    idx_parts, val_parts = [], []
    for r in range(rows):
        if cols == 0 or rng.random() < empty_frac:
            n = 0
        else:
            n = int(rng.binomial(cols, density))
            if max_row is not None:
                n = min(n, max_row)
        c = np.sort(rng.choice(cols, size=n, replace=False)).astype(np.uint32) if n else np.zeros(0, np.uint32)
        if integer:
            v = rng.integers(1, 40, size=n).astype(np.float16)
        else:
            v = (rng.standard_normal(n) * 3).astype(np.float16)
        idx_parts.append(c)
        val_parts.append(v.view(np.uint16))
        ptr[r + 1] = ptr[r] + n
    idx = np.concatenate(idx_parts) if idx_parts else np.zeros(0, np.uint32)
    val = np.concatenate(val_parts) if val_parts else np.zeros(0, np.uint16)
    # rows with repeated / out-of-order columns (the reference overwrites in CSR order)
    nz_rows = [r for r in range(rows) if ptr[r + 1] - ptr[r] >= 3]
    for r in nz_rows[:dup_rows]:
        a = ptr[r]
        idx[a + 2] = idx[a]  # repeat the first column later in the row
    for r in nz_rows[dup_rows:dup_rows + unsorted_rows]:
        a, b = ptr[r], ptr[r + 1]
        idx[a:b] = idx[a:b][::-1].copy()
    return ptr, idx.astype(np.uint32), val.astype(np.uint16)


def to_device_csr(rows, cols, ptr, idx, val):
    import torch

    from cellshard_b200.device import CSR

    def t32(a):
        return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32).copy()).cuda()

    v = torch.from_numpy(np.ascontiguousarray(val, np.uint16).view(np.float16).copy()).cuda()
    return CSR(rows, cols, t32(ptr), t32(idx) if len(idx) else torch.zeros(0, dtype=torch.int32, device="cuda"), v)


def np_u32(t):
    return t.cpu().numpy().view(np.uint32)


def np_u16(t):
    return t.cpu().numpy().view(np.uint16)
