""".cspack raw records between files and device memory: records this build
writes are byte for byte the restated layout (pinned against the reference's
own store_*_raw), and records the reference writes load back into device
memory unchanged; a record larger than one staging chunk round-trips."""

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu


def test_store_matches_record_layout_and_reference(cuda, orc, tmp_path):
    import torch

    from cellshard_b200.device import blocked_ell_from_csr, cspack_store, cspack_store_coo, sliced_ell_from_csr

    rows, cols = 333, 500
    ptr, idx, val = random_csr(rows, cols, 0.05, 9, 0.2)
    csr = to_device_csr(rows, cols, ptr, idx, val)
    bell = blocked_ell_from_csr(csr, 8)
    sell = sliced_ell_from_csr(csr, 32)
    row = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(ptr.astype(np.int64)))
    rt = torch.from_numpy(row.view(np.int32).copy()).cuda()
    files = {k: tmp_path / f"{k}.cspack" for k in ("csr", "bell", "sell", "coo")}
    cspack_store(files["csr"], csr)
    cspack_store(files["bell"], bell)
    cspack_store(files["sell"], sell)
    cspack_store_coo(files["coo"], rows, cols, rt, csr.idx, csr.val)
    b = (np_u32(bell.bci), np_u16(bell.val))
    s = (np_u32(sell.slice_row_offsets), np_u32(sell.slice_widths), np_u32(sell.col_idx), np_u16(sell.val))
    want = {
        "csr": orc.cspack_compressed(rows, cols, len(idx), 0, ptr, idx, val),
        "bell": orc.cspack_blocked_ell(rows, cols, bell.nnz, 8, bell.ell_cols, *b),
        "sell": orc.cspack_sliced_ell(rows, cols, sell.nnz, *s),
        "coo": orc.cspack_coo(rows, cols, row, idx, val),
    }
    for k, path in files.items():
        assert path.read_bytes() == want[k], k
    if orc.ref_bucket_available():
        ref = tmp_path / "ref.cspack"
        orc.ref_cspack_store(orc.CSPACK_BLOCKED_ELL, ref, rows, cols, bell.nnz, 8, bell.ell_cols, *b)
        assert ref.read_bytes() == files["bell"].read_bytes()
        orc.ref_cspack_store(orc.CSPACK_SLICED_ELL, ref, rows, cols, sell.nnz, *s)
        assert ref.read_bytes() == files["sell"].read_bytes()


def test_load_reference_records(cuda, orc, tmp_path):
    from cellshard_b200.device import cspack_load

    rows, cols = 257, 300
    ptr, idx, val = random_csr(rows, cols, 0.08, 3, 0.1)
    b = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, 16)
    s = orc.sliced_ell_from_csr(rows, ptr, idx, val, 7)
    row = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(ptr.astype(np.int64)))
    recs = {
        "bell": orc.cspack_blocked_ell(rows, cols, b["nnz"], 16, b["ell_cols"], b["bci"], b["val"]),
        "sell": orc.cspack_sliced_ell(rows, cols, len(idx), s["offsets"], s["widths"], s["col_idx"], s["val"]),
        "csr": orc.cspack_compressed(rows, cols, len(idx), 0, ptr, idx, val),
        "coo": orc.cspack_coo(rows, cols, row, idx, val),
    }
    for k, data in recs.items():
        path = tmp_path / f"{k}.cspack"
        if orc.ref_bucket_available():  # written by the reference's codec itself
            args = {"bell": (orc.CSPACK_BLOCKED_ELL, b["nnz"], 16, b["ell_cols"], b["bci"], b["val"]),
                    "sell": (orc.CSPACK_SLICED_ELL, len(idx), s["offsets"], s["widths"], s["col_idx"], s["val"]),
                    "csr": (orc.CSPACK_COMPRESSED, len(idx), 0, ptr, idx, val),
                    "coo": (orc.CSPACK_COO, len(idx), row, idx, val)}[k]
            assert orc.ref_cspack_store(args[0], path, rows, cols, args[1], *args[2:]) == 1
            assert path.read_bytes() == data
        else:
            path.write_bytes(data)
        m = cspack_load(path)
        if k == "bell":
            assert m.ell_cols == b["ell_cols"] and np.array_equal(np_u32(m.bci), b["bci"])
            assert np.array_equal(np_u16(m.val), b["val"])
        elif k == "sell":
            assert np.array_equal(np_u32(m.slice_row_offsets), s["offsets"])
            assert np.array_equal(np_u32(m.slice_widths), s["widths"])
            assert np.array_equal(np_u32(m.slice_slot_offsets), s["slot_offsets"])
            assert np.array_equal(np_u32(m.col_idx), s["col_idx"]) and np.array_equal(np_u16(m.val), s["val"])
        elif k == "csr":
            assert np.array_equal(np_u32(m.ptr), ptr) and np.array_equal(np_u32(m.idx), idx)
            assert np.array_equal(np_u16(m.val), val)
        else:
            _r, _c, rr, cc, vv = m
            assert np.array_equal(np_u32(rr), row) and np.array_equal(np_u32(cc), idx)
            assert np.array_equal(np_u16(vv), val)


def test_multi_chunk_round_trip(cuda, tmp_path):
    """A 20,000 x 1,024 Blocked-ELL-16 (40 MB of values: two staging chunks)."""
    import torch

    from cellshard_b200.device import BlockedELL, cspack_load, cspack_store

    rows, ell_cols, B = 20_000, 1_024, 16
    g = torch.Generator(device="cuda").manual_seed(1)
    bci = torch.randint(0, 4096, ((rows // B) * (ell_cols // B),), device="cuda", generator=g, dtype=torch.int32)
    val = torch.randint(-30000, 30000, (rows * ell_cols,), device="cuda", generator=g,
                        dtype=torch.int32).to(torch.int16).view(torch.float16)
    m = BlockedELL(rows, 65536, B, ell_cols, bci, val, 123)
    path = tmp_path / "big.cspack"
    cspack_store(path, m)
    assert path.stat().st_size == 13 + 8 + bci.numel() * 4 + val.numel() * 2
    back = cspack_load(path)
    assert back.nnz == 123 and torch.equal(back.bci, bci) and torch.equal(back.val.view(torch.int16),
                                                                          val.view(torch.int16))
