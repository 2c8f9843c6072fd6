"""Pins the CPU restatement (oracle/cs_oracle.c) before anything trusts it:

* against the reference's own known-answer test (tests/mask_groups_runtime_test.cu
  of the reference, restated in golden/mask_groups_known_answers.json);
* against outputs of the reference's own conversion code on seeded inputs
  (golden/ref_conversions.npz, written by golden/make_golden.py);
* against the reference code itself, live, when oracle/_ref is built.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from cases import random_csr

GOLD = Path(__file__).resolve().parent / "golden"
KA = json.loads((GOLD / "mask_groups_known_answers.json").read_text())


def h(vals):
    return np.asarray(vals, np.float32).astype(np.float16).view(np.uint16)


def u(vals):
    return np.asarray(vals, np.uint64).astype(np.uint32)


def _filt():
    f = KA["filter"]
    return (float(f[0]), int(f[1]), float(f[2]), int(f[3]))


def test_known_answers_blocked(orc):
    b = KA["blocked"]
    res = orc.group_reduce_bell(KA["rows"], KA["cols"], b["block_size"], b["ell_cols"], u(b["block_cols"]),
                                h(b["values"]), u(KA["group_masks"]), KA["group_count"], u8(KA["row_keep"]),
                                u8(KA["feature_keep"]), _filt())
    e = KA["expect_blocked"]
    assert np.allclose(res["row_totals"], e["row_totals"], atol=1e-3)
    assert list(res["detected_features"]) == e["detected"]
    assert list(res["row_keep"]) == e["keep"]
    for k, v in e["group_counts"].items():
        assert abs(res["group_counts"][int(k)] - v) <= 1e-3
    for k, v in e["group_percentages"].items():
        assert abs(res["group_percentages"][int(k)] - v) <= 1e-3


def u8(vals):
    return np.asarray(vals, np.uint8)


def test_known_answers_no_groups(orc):
    b = KA["blocked"]
    res = orc.group_reduce_bell(KA["rows"], KA["cols"], b["block_size"], b["ell_cols"], u(b["block_cols"]),
                                h(b["values"]), None, 0, None, None, _filt())
    e = KA["expect_no_groups"]
    assert res["group_counts"] is None
    assert abs(res["row_totals"][0] - e["row_totals0"]) <= 1e-3
    assert res["detected_features"][0] == e["detected0"]


def test_known_answers_compressed(orc):
    c = KA["compressed"]
    res = orc.group_reduce_csr(KA["rows"], KA["cols"], u(c["ptr"]), u(c["idx"]), h(c["values"]),
                               u(KA["group_masks"]), KA["group_count"], u8(KA["row_keep"]), u8(KA["feature_keep"]),
                               _filt())
    e = KA["expect_compressed"]
    assert abs(res["row_totals"][2] - e["row_totals2"]) <= 1e-3
    assert abs(res["group_counts"][8] - e["group_counts8"]) <= 1e-3


def test_known_answers_sliced(orc):
    s = KA["sliced"]
    res = orc.group_reduce_sell(KA["rows"], KA["cols"], s["slice_rows"], u(s["offsets"]), u(s["widths"]),
                                u(s["slot_offsets"]), u(s["col_idx"]), h(s["values"]), u(KA["group_masks"]),
                                KA["group_count"], u8(KA["row_keep"]), u8(KA["feature_keep"]), _filt())
    e = KA["expect_sliced"]
    assert abs(res["row_totals"][0] - e["row_totals0"]) <= 1e-3
    assert abs(res["row_totals"][3] - e["row_totals3"]) <= 1e-3


def test_known_answers_reoptimize(orc):
    b, r = KA["blocked"], KA["reoptimize"]
    major, idx, val = orc.reoptimize_bell(KA["rows"], KA["cols"], b["block_size"], b["ell_cols"], u(b["block_cols"]),
                                          h(b["values"]), u8(KA["row_keep"]), u8(KA["feature_keep"]),
                                          u(r["row_remap"]), u(r["feature_remap"]), r["output_rows"],
                                          r["output_cols"])
    assert int(major[-1]) == KA["expect_reoptimize"]["live_nnz"]
    assert len(major) == KA["expect_reoptimize"]["kept_rows"] + 1
    assert idx.max() < KA["expect_reoptimize"]["kept_features"]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD / "ref_conversions.npz")


def _cases(gold):
    names = sorted({k.split("/")[0] for k in gold.files})
    for n in names:
        rows, cols = (int(x) for x in gold[f"{n}/shape"])
        yield n, rows, cols, gold[f"{n}/ptr"], gold[f"{n}/idx"], gold[f"{n}/val"]


def test_restated_blocked_ell_matches_reference_vectors(orc, gold):
    checked = 0
    for n, rows, cols, ptr, idx, val in _cases(gold):
        for B in (1, 2, 3, 4, 8, 16):
            r = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
            ell_cols, nnz = (int(x) for x in gold[f"{n}/bell{B}/meta"])
            assert r["ell_cols"] == ell_cols, (n, B)
            assert r["nnz"] == nnz, (n, B)
            assert np.array_equal(r["bci"], gold[f"{n}/bell{B}/bci"]), (n, B)
            assert np.array_equal(r["val"], gold[f"{n}/bell{B}/val"]), (n, B)
            checked += 1
    assert checked >= 30


def test_restated_sliced_ell_matches_reference_vectors(orc, gold):
    checked = 0
    for n, rows, cols, ptr, idx, val in _cases(gold):
        for hgt in (1, 3, 16, 32, 64):
            key = f"{n}/sell{hgt}/meta"
            if key not in gold.files:
                continue
            r = orc.sliced_ell_from_csr(rows, ptr, idx, val, hgt)
            S, _nnz, total = (int(x) for x in gold[key])
            assert r["slice_count"] == S and r["total_slots"] == total, (n, hgt)
            assert np.array_equal(r["offsets"], gold[f"{n}/sell{hgt}/offsets"])
            assert np.array_equal(r["widths"], gold[f"{n}/sell{hgt}/widths"])
            assert np.array_equal(r["col_idx"], gold[f"{n}/sell{hgt}/col_idx"])
            assert np.array_equal(r["val"], gold[f"{n}/sell{hgt}/val"])
            checked += 1
    assert checked >= 20


def _bell_cases(gold):
    for n, rows, cols, ptr, idx, val in _cases(gold):
        for B in (3, 4, 16):
            key = f"{n}/bell{B}"
            if f"{key}/sell3/meta" not in gold.files:
                continue
            ell_cols, nnz = (int(x) for x in gold[f"{key}/meta"])
            bval = gold[f"{key}/val_special"] if f"{key}/val_special" in gold.files else gold[f"{key}/val"]
            yield n, key, rows, cols, nnz, B, ell_cols, gold[f"{key}/bci"], bval


def test_restated_bell_to_sliced_matches_reference_vectors(orc, gold):
    """convert::sliced_ell_from_blocked_ell of the reference on its own
    Blocked-ELL outputs (with a -0.0 and a NaN planted in the B = 4 matrices)."""
    checked = 0
    for n, key, rows, cols, nnz, B, ell_cols, bci, bval in _bell_cases(gold):
        for hgt in (3, 32):
            S, rnnz, total = (int(x) for x in gold[f"{key}/sell{hgt}/meta"])
            r = orc.sliced_ell_from_bell(rows, cols, B, ell_cols, bci, bval, hgt)
            assert rnnz == nnz, key  # the reference carries the source's nnz field
            assert r["slice_count"] == S and r["total_slots"] == total, (key, hgt)
            assert np.array_equal(r["widths"], gold[f"{key}/sell{hgt}/widths"]), (key, hgt)
            assert np.array_equal(r["col_idx"], gold[f"{key}/sell{hgt}/col_idx"]), (key, hgt)
            assert np.array_equal(r["val"], gold[f"{key}/sell{hgt}/val"]), (key, hgt)
            checked += 1
        hr, S, padded, pbytes = (int(x) for x in gold[f"{key}/choose_sell"])
        live_ptr, _, _ = orc.bell_live_csr(rows, cols, B, ell_cols, bci, bval)
        assert orc.choose_sliced_slice_rows(rows, nnz, live_ptr, (8, 16, 32, 64))[0] == hr, key
    assert checked >= 30


def test_restated_sliced_chooser_matches_reference_vectors(orc, gold):
    for n, rows, cols, ptr, idx, val in _cases(gold):
        hr, S, padded, pbytes = (int(x) for x in gold[f"{n}/choose_sell"])
        # restated evaluate_sliced_candidate_ + choose_sliced_ell_slice_rows in Python doubles
        best = None
        nnz = len(idx)
        for c in (8, 16, 32, 64):
            hh = max(1, min(c, rows)) if rows else 0
            slots = orc.sliced_padded_slots(rows, ptr, c)
            cnt = (rows + hh - 1) // hh if rows else 0
            pb = slots * 6 + (cnt * 2 + 1) * 4
            ratio = 1.0 if nnz == 0 else slots / nnz
            pen = 0.0 if rows == 0 else 0.25 * (cnt / rows)
            score = ratio + pen
            cand = (hh, cnt, slots, pb, score)
            if (best is None or score + 1e-12 < best[4] or (score <= best[4] + 1e-12 and pb < best[3])
                    or (score <= best[4] + 1e-12 and pb == best[3] and hh > best[0])):
                best = cand
        assert best[:4] == (hr, S, padded, pbytes), n
        assert best[4] == gold[f"{n}/choose_sell_f"][2]


def test_restated_blocked_shape_matches_reference_chooser(orc, gold):
    for n, rows, cols, ptr, idx, val in _cases(gold):
        bsz, pbytes = (int(x) for x in gold[f"{n}/choose_bell"])
        fill = float(gold[f"{n}/choose_bell_fill"][0])
        best = None
        for B in (4, 8, 16, 32):
            w, tot = orc.blocked_ell_shape(rows, cols, ptr, idx, B)
            rb = (rows + B - 1) // B
            if rows == 0 or cols == 0:
                f = 0.0
            else:
                f = 1.0 if (rb == 0 or w == 0) else tot / (rb * w)
            pb = rows * w * B * 2
            if (best is None or pb + 1 < best[1] or (pb == best[1] and f > best[2] + 1e-9)
                    or (pb == best[1] and f + 1e-9 >= best[2] and B > best[0])):
                best = (B, pb, f)
        assert (best[0], best[1]) == (bsz, pbytes), n
        assert best[2] == fill


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).ref_available(),
                    reason="reference bridge not built")
def test_restatement_matches_live_reference_random(orc):
    for seed in range(6):
        rows, cols = 50 + 13 * seed, 40 + 29 * seed
        ptr, idx, val = random_csr(rows, cols, 0.1, 100 + seed, 0.15)
        for B in (2, 5, 16):
            a = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, B)
            b = orc.ref_blocked_ell_from_compressed(rows, cols, ptr, idx, val, B)
            assert a["ell_cols"] == b["ell_cols"] and a["nnz"] == b["nnz"]
            assert np.array_equal(a["bci"], b["bci"]) and np.array_equal(a["val"], b["val"])
        for hh in (7, 32):
            a = orc.sliced_ell_from_csr(rows, ptr, idx, val, hh)
            b = orc.ref_sliced_ell_from_compressed(rows, cols, ptr, idx, val, hh)
            assert np.array_equal(a["col_idx"], b["col_idx"]) and np.array_equal(a["val"], b["val"])
            assert np.array_equal(a["widths"], b["widths"])


def test_transpose_and_bucketing_restatement_properties(orc):
    ptr, idx, val = random_csr(120, 70, 0.08, 9, 0.2)
    tptr, tidx, tval = orc.csr_transpose(120, 70, ptr, idx, val)
    # transposing twice is the identity on sorted CSR
    bptr, bidx, bval = orc.csr_transpose(70, 120, tptr, tidx, tval)
    assert np.array_equal(bptr, ptr) and np.array_equal(bidx, idx) and np.array_equal(bval, val)
    nnz, srt, order, offs = orc.major_nnz_plan(ptr, 120, 7)
    assert np.array_equal(nnz, np.diff(ptr))
    assert np.array_equal(srt, np.sort(nnz, kind="stable"))
    assert np.array_equal(order, np.argsort(nnz, kind="stable"))
    sizes = np.diff(offs.astype(np.int64))
    assert sizes.sum() == 120 and sizes.max() - sizes.min() <= 1 and list(sizes) == sorted(sizes, reverse=True)
    bins = orc.pow2_bins(srt)
    for k in range(33):
        seg = srt[bins[k]:bins[k + 1]]
        lo = 0 if k == 0 else 2 ** k
        assert np.all(seg >= lo) and np.all(seg < 2 ** (k + 1))
    dptr, didx, dval, inv = orc.rebuild(ptr, idx, val, 120, order)
    assert np.array_equal(inv[order], np.arange(120))
    for i in range(120):
        s = order[i]
        assert np.array_equal(didx[dptr[i]:dptr[i + 1]], idx[ptr[s]:ptr[s + 1]])


def test_moments_oracle_small_exact(orc):
    ptr, idx, val = random_csr(90, 33, 0.3, 11, 0.1)
    rng = np.random.default_rng(3)
    keep = (rng.random(90) < 0.7).astype(np.uint8)
    fk = (rng.random(33) < 0.8).astype(np.uint8)
    lab = rng.integers(0, 5, 90).astype(np.uint32)
    r = orc.group_moments_csr(90, 33, ptr, idx, val, keep, fk, lab, 5, ddof=1, nthreads=3)
    x = np.zeros((90, 33))
    for i in range(90):
        x[i, idx[ptr[i]:ptr[i + 1]]] = orc.h2f(val[ptr[i]:ptr[i + 1]])
    for g in range(5):
        rows = (keep == 1) & (lab == g)
        s = x[rows].sum(0) * fk
        assert np.allclose(r["sum"][g], s)
        assert r["group_rows"][g] == rows.sum()
        if rows.sum() > 1:
            v = x[rows].var(0, ddof=1) * fk
            assert np.allclose(r["var"][g], v)
