"""Pins the restated execution bucketing (oracle/cs_oracle.c, after
src/io/csh5/execution_builders_part.hh:1011-1596 of the reference) against
the reference's own builders: the committed outputs in golden/ref_bucketing.npz
and, when oracle/_ref is built, the compiled builders live on fresh inputs."""

from pathlib import Path

import numpy as np
import pytest

from cases import random_csr

GOLD = Path(__file__).resolve().parent / "golden"


def _cases(gold):
    return sorted({k.split("/")[0] for k in gold.files})


def test_blocked_restatement_matches_reference_vectors(orc):
    conv, gold = np.load(GOLD / "ref_conversions.npz"), np.load(GOLD / "ref_bucketing.npz")
    checked = 0
    for n in _cases(gold):
        rows, cols = (int(x) for x in conv[f"{n}/shape"])
        for B in (4, 16):
            key = f"{n}/bell{B}"
            ell_cols, _nnz = (int(x) for x in conv[f"{key}/meta"])
            bci, bval = conv[f"{key}/bci"], conv[f"{key}/val"]
            for req in (1, 2, 3, 8):
                g = f"{key}/bucket{req}"
                mine = orc.bell_bucketed(rows, B, ell_cols, bci, bval, req)
                S, nbytes = (int(x) for x in gold[f"{g}/meta"])
                assert mine["segment_count"] == S and mine["bytes"] == nbytes, g
                seg = gold[f"{g}/seg"].reshape(-1, 3)
                assert np.array_equal(mine["seg_rows"], seg[:, 0]) and np.array_equal(mine["seg_w"] * B, seg[:, 1])
                assert np.array_equal(mine["seg_bci"], gold[f"{g}/bci"]) and np.array_equal(mine["seg_val"],
                                                                                           gold[f"{g}/val"])
                assert np.array_equal(mine["e2c"], gold[f"{g}/e2c"]), g
                checked += 1
            assert orc.bell_choose_bucket_count(rows, B, ell_cols, bci) == tuple(int(x) for x in gold[f"{key}/choose"])
    assert checked >= 40


def test_sliced_restatement_matches_reference_vectors(orc):
    conv, gold = np.load(GOLD / "ref_conversions.npz"), np.load(GOLD / "ref_bucketing.npz")
    checked = 0
    for n in _cases(gold):
        rows = int(conv[f"{n}/shape"][0])
        for h in (3, 32):
            key = f"{n}/sell{h}"
            if f"{key}/choose" not in gold.files:
                continue
            offs, widths, col, val = (conv[f"{key}/{f}"] for f in ("offsets", "widths", "col_idx", "val"))
            for req in (1, 2, 3, 8):
                g = f"{key}/bucket{req}"
                mine = orc.sell_bucketed(rows, offs, widths, col, val, req)
                S, nbytes = (int(x) for x in gold[f"{g}/meta"])
                assert mine["segment_count"] == S and mine["bytes"] == nbytes, g
                seg = gold[f"{g}/seg"].reshape(-1, 3)
                assert np.array_equal(np.diff(mine["seg_row"]), seg[:, 0]) and np.array_equal(mine["seg_w"], seg[:, 1])
                assert np.array_equal(mine["seg_col"], gold[f"{g}/col_idx"]) and np.array_equal(mine["seg_val"],
                                                                                               gold[f"{g}/val"])
                assert np.array_equal(mine["e2c"], gold[f"{g}/e2c"]), g
                checked += 1
            assert orc.sell_choose_bucket_count(rows, offs, widths, col) == tuple(int(x) for x in gold[f"{key}/choose"])
    assert checked >= 20


@pytest.mark.parametrize("rows,cols,B,density,seed", [
    (1000, 2000, 16, 0.01, 7),   # heavy-tailed rows: several segments survive the byte rule
    (257, 500, 8, 0.03, 2),      # partial last row block
    (64, 64, 4, 0.5, 3),         # dense: widths equal, buckets merge
    (1, 10, 4, 0.5, 4),          # a single partial row block
])
def test_restatement_matches_live_reference(orc, rows, cols, B, density, seed):
    if not orc.ref_bucket_available():
        pytest.skip("reference bucketing bridge not built")
    ptr, idx, val = random_csr(rows, cols, density, seed, 0.3)
    b = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
    for req in (1, 2, 4, 5, 8, 100):
        mine = orc.bell_bucketed(rows, B, b["ell_cols"], b["bci"], b["val"], req)
        ref = orc.ref_build_bucketed_bell(rows, cols, b["nnz"], B, b["ell_cols"], b["bci"], b["val"], req)
        assert mine["segment_count"] == ref["segment_count"] and mine["bytes"] == ref["bytes"]
        assert np.array_equal(mine["e2c"], ref["e2c"]) and np.array_equal(mine["c2e"], ref["c2e"])
        assert np.array_equal(mine["seg_bci"], np.concatenate([g["bci"] for g in ref["segments"]]))
        assert np.array_equal(mine["seg_val"], np.concatenate([g["val"] for g in ref["segments"]]))
        assert [g["nnz"] for g in ref["segments"]] == [
            int(sum(min(B, rows - int(rb) * B) * int(mine["widths"][rb]) * B
                    for rb in mine["order"][mine["seg_rb"][s]:mine["seg_rb"][s + 1]])) for s in range(len(ref["segments"]))]
    assert orc.bell_choose_bucket_count(rows, B, b["ell_cols"], b["bci"]) == orc.ref_choose_bucket_count_for_part(
        rows, cols, b["nnz"], B, b["ell_cols"], b["bci"], b["val"])
    s = orc.sliced_ell_from_csr(rows, ptr, idx, val, 32)
    for req in (1, 2, 4, 8, 50):
        mine = orc.sell_bucketed(rows, s["offsets"], s["widths"], s["col_idx"], s["val"], req)
        ref = orc.ref_build_bucketed_sell(rows, cols, len(idx), s["offsets"], s["widths"], s["col_idx"], s["val"], req)
        assert mine["segment_count"] == ref["segment_count"] and mine["bytes"] == ref["bytes"]
        assert np.array_equal(mine["e2c"], ref["e2c"])
        assert np.array_equal(mine["seg_col"], np.concatenate([g["col_idx"] for g in ref["segments"]]))
        assert np.array_equal(mine["seg_val"], np.concatenate([g["val"] for g in ref["segments"]]))
    assert orc.sell_choose_bucket_count(rows, s["offsets"], s["widths"], s["col_idx"]) == \
        orc.ref_choose_bucket_count_for_sliced_part(rows, cols, len(idx), s["offsets"], s["widths"], s["col_idx"],
                                                    s["val"])
