"""Pins the restated COO -> Blocked-ELL (oracle/cs_oracle.c, after
src/convert/blocked_ell_from_compressed.cuh:105-257,349-437 of the reference)
against the reference's own host routines: golden/ref_coo.npz (shuffled COO,
repeated entries, a column map) and, with oracle/_ref built, live."""

from pathlib import Path

import numpy as np
import pytest

from cases import random_csr

GOLD = Path(__file__).resolve().parent / "golden"


def test_restatement_matches_reference_vectors(orc):
    conv, gold = np.load(GOLD / "ref_conversions.npz"), np.load(GOLD / "ref_coo.npz")
    checked = 0
    for n in sorted({k.split("/")[0] for k in gold.files}):
        rows, cols = (int(x) for x in conv[f"{n}/shape"])
        row, col, val = (gold[f"{n}/coo/{k}"] for k in ("row", "col", "val"))
        fmap = gold[f"{n}/coo/map"] if f"{n}/coo/map" in gold.files else None
        for B in (2, 3, 8, 16):
            mine = orc.blocked_ell_from_coo(rows, cols, row, col, val, B, fmap)
            ell_cols, nnz = (int(x) for x in gold[f"{n}/coo{B}/meta"])
            assert mine["ell_cols"] == ell_cols and mine["nnz_host"] == nnz, (n, B)
            assert np.array_equal(mine["bci"], gold[f"{n}/coo{B}/bci"]), (n, B)
            assert np.array_equal(mine["val"], gold[f"{n}/coo{B}/val"]), (n, B)
            checked += 1
        b, fill, padded = orc.choose_block_size_from_coo(rows, cols, row, col, [2, 4, 8, 16], fmap)
        assert (b, padded) == tuple(int(x) for x in gold[f"{n}/coo_choose"])
        assert fill == float(gold[f"{n}/coo_choose_fill"][0])
    assert checked >= 20


@pytest.mark.parametrize("rows,cols,density,B,dups,remap", [
    (300, 500, 0.03, 16, 6, False),
    (64, 64, 0.5, 8, 10, True),
    (33, 900, 0.01, 3, 2, True),
])
def test_restatement_matches_live_reference(orc, rows, cols, density, B, dups, remap):
    if not orc.ref_available():
        pytest.skip("reference bridge not built")
    ptr, idx, val = random_csr(rows, cols, density, rows + B, 0.2)
    rng = np.random.default_rng(rows)
    row = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(ptr.astype(np.int64)))
    col, v = idx.copy(), val.copy()
    if dups:
        k = rng.integers(0, len(row), dups)
        row, col, v = np.concatenate([row, row[k]]), np.concatenate([col, col[k]]), np.concatenate([v, v[k] ^ 0x400])
    p = rng.permutation(len(row))
    row, col, v = row[p].astype(np.uint32), col[p].astype(np.uint32), v[p].astype(np.uint16)
    fmap = rng.permutation(cols).astype(np.uint32) if remap else None
    mine = orc.blocked_ell_from_coo(rows, cols, row, col, v, B, fmap)
    ref = orc.ref_blocked_ell_from_coo(rows, cols, cols, row, col, v, B, fmap)
    assert mine["ell_cols"] == ref["ell_cols"] and mine["nnz_host"] == ref["nnz"]
    assert np.array_equal(mine["bci"], ref["bci"]) and np.array_equal(mine["val"], ref["val"])
    assert orc.choose_block_size_from_coo(rows, cols, row, col, [2, 4, 8, 16, 32], fmap) == \
        orc.ref_choose_block_size_from_coo(rows, cols, cols, row, col, v, [2, 4, 8, 16, 32], fmap)
