"""Pins the restated .cspack record layout (oracle/oracle.py cspack_*, after
src/io/pack/packfile.cu of the reference) byte for byte against records the
reference's own store_*_raw functions write (oracle/_ref, when built)."""

import numpy as np
import pytest

from cases import random_csr


@pytest.fixture
def ref_bucket(orc):
    if not orc.ref_bucket_available():
        pytest.skip("reference codec bridge not built")
    return orc


def test_records_match_reference_store(ref_bucket, tmp_path):
    orc = ref_bucket
    rows, cols = 37, 90
    ptr, idx, val = random_csr(rows, cols, 0.1, 4, 0.2)
    nnz = len(idx)
    cases = []
    b = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, 4)
    cases.append((orc.CSPACK_BLOCKED_ELL, (4, b["ell_cols"], b["bci"], b["val"]),
                  orc.cspack_blocked_ell(rows, cols, b["nnz"], 4, b["ell_cols"], b["bci"], b["val"]), b["nnz"]))
    s = orc.sliced_ell_from_csr(rows, ptr, idx, val, 8)
    cases.append((orc.CSPACK_SLICED_ELL, (s["offsets"], s["widths"], s["col_idx"], s["val"]),
                  orc.cspack_sliced_ell(rows, cols, nnz, s["offsets"], s["widths"], s["col_idx"], s["val"]), nnz))
    cases.append((orc.CSPACK_COMPRESSED, (0, ptr, idx, val), orc.cspack_compressed(rows, cols, nnz, 0, ptr, idx, val),
                  nnz))
    row = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(ptr.astype(np.int64)))
    cases.append((orc.CSPACK_COO, (row, idx, val), orc.cspack_coo(rows, cols, row, idx, val), nnz))
    for fmt, arrays, mine, n in cases:
        path = tmp_path / f"f{fmt}.cspack"
        assert orc.ref_cspack_store(fmt, path, rows, cols, n, *arrays) == 1
        assert path.read_bytes() == mine, fmt
