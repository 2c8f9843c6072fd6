"""Regenerates the committed golden fixtures in this directory.

  python tests/golden/make_golden.py

1. mask_groups_known_answers.json -- the inputs and expected values of the
   reference's own known-answer test, tests/mask_groups_runtime_test.cu:56-198
   (4 x 5 matrix, 3 feature groups, row/feature masks, filter, remaps) restated
   as data.
2. ref_conversions.npz -- outputs of the reference's own conversion code
   (convert::blocked_ell_from_compressed, choose_blocked_ell_block_size,
   sliced_ell_from_compressed, choose_sliced_ell_slice_rows_from_compressed,
   sliced_ell_from_blocked_ell, choose_sliced_ell_slice_rows_from_blocked_ell),
   compiled from the reference sources into oracle/_ref/libcs_ref.so by
   oracle/Makefile, on seeded small CSR inputs.  Needs the reference tree
   (only here, not on the GPU machine).
3. ref_bucketing.npz -- outputs of the reference's execution-bucketing
   builders (build_bucketed_execution_partition, choose_bucket_count_for_part,
   build_bucketed_sliced_execution_partition,
   choose_bucket_count_for_sliced_part, src/io/csh5/execution_builders_part.hh)
   compiled into oracle/_ref/libcs_ref_bucket.so, on the Blocked-ELL and
   Sliced-ELL matrices of the conversion cases.
4. ref_coo.npz -- outputs of the reference's COO -> Blocked-ELL host routines
   (convert::blocked_ell_from_coo, choose_blocked_ell_block_size_from_coo,
   src/convert/blocked_ell_from_compressed.cuh) on the conversion cases as
   shuffled COO, some with repeated (row, column) entries and a column map.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

INVALID = 0xFFFFFFFF


def known_answers() -> dict:
    # tests/mask_groups_runtime_test.cu:57-66 group masks / row / feature masks
    return {
        "source": "tests/mask_groups_runtime_test.cu:56-198 of the reference",
        "rows": 4,
        "cols": 5,
        "group_masks": [1, 2, 3, 0, 4],  # bit0, bit1, bit0|bit1, 0, bit2 (:58-64)
        "row_keep": [1, 0, 1, 1],  # :65
        "feature_keep": [1, 1, 0, 1, 1],  # :66
        "filter": [1.0, 1, 0.80, 0],  # min_total, min_detected, max_fraction, fraction group (:82)
        "group_count": 3,
        "blocked": {  # :88-111, block 2, ell_cols 4, nnz 10
            "block_size": 2,
            "ell_cols": 4,
            "block_cols": [0, 1, 0, 1, 0, 1, 1, 2],
            "values": [5, 3, 7, 0, 9, 0, 0, 0, 1, 4, 6, 2, 0, 8, 0, 10],
        },
        "expect_blocked": {  # :114-119, two entries corrected, see below
            "row_totals": [8, 0, 7, 18],
            "detected": [2, 0, 3, 2],
            "keep": [1, 0, 1, 1],
            "group_counts": {"0": 5, "1": 3, "2": 0, "6": 1, "7": 4, "8": 0},
            "group_percentages": {"0": 62.5, "4": 0.0},
        },
        # The reference test asserts keep[3] == 0 (:116) and group_counts[8] == 2
        # (:118).  Its own kernel (mask_groups.cu:131-194) gives keep[3] = 1
        # (row 3: total 18, detected 2, group-0 fraction 0/18 <= 0.8) and, for
        # the Blocked-ELL matrix it builds (row block 1 holds block columns
        # {0, 1}, so row 2's value 2 sits at gene 3, which has no group),
        # group_counts[8] = 0.  The GPU tests run the reference's own test
        # binary and kernels to confirm (the binary stops at `return 14`).
        "reference_test_asserts": {"keep3": 0, "blocked_group_counts8": 2, "expected_exit_code": 14},
        "expect_no_groups": {"group_count": 0, "row_totals0": 15, "detected0": 3},  # :121-124
        "compressed": {  # :126-128
            "ptr": [0, 3, 4, 8, 10],
            "idx": [0, 1, 2, 0, 0, 1, 2, 4, 1, 4],
            "values": [5, 3, 7, 9, 1, 4, 6, 2, 8, 10],
        },
        "expect_compressed": {"row_totals2": 7, "group_counts8": 2},  # :143
        "sliced": {  # :145-174, one slice of 4 rows, width 3
            "offsets": [0, 4],
            "widths": [3],
            "slot_offsets": [0],
            "slice_rows": 4,
            "nnz": 9,
            "col_idx": [0, 1, 2, 0, INVALID, INVALID, 0, 1, 4, 1, 4, INVALID],
            "values": [5, 3, 7, 9, 0, 0, 1, 4, 2, 8, 10, 0],
        },
        "expect_sliced": {"row_totals0": 8, "row_totals3": 18},  # :177
        "reoptimize": {  # :182-191
            "row_remap": [0, INVALID, 1, 2],
            "feature_remap": [0, 1, INVALID, 2, 3],
            "output_rows": 3,
            "output_cols": 4,
        },
        "expect_reoptimize": {"kept_rows": 3, "kept_features": 4, "live_nnz": 7},  # :195-197
    }


CONVERSION_CASES = [
    # name, rows, cols, density, seed, empty_frac, dup_rows, unsorted_rows
    ("small", 67, 45, 0.12, 1, 0.1, 0, 0),
    ("wide", 40, 300, 0.05, 2, 0.2, 0, 0),
    ("dense", 33, 20, 0.7, 3, 0.0, 0, 0),
    ("empty_rows", 20, 30, 0.1, 4, 0.6, 0, 0),
    ("all_empty", 9, 12, 0.0, 5, 1.0, 0, 0),
    ("dups", 30, 25, 0.3, 6, 0.0, 4, 3),
]
BLOCK_SIZES = [1, 2, 3, 4, 8, 16]
SLICE_ROWS = [1, 3, 16, 32, 64]
BLOCK_CANDIDATES = [4, 8, 16, 32]
SLICE_CANDIDATES = [8, 16, 32, 64]
BELL_TO_SELL_BLOCKS = [3, 4, 16]
BELL_TO_SELL_ROWS = [3, 32]


def ref_conversions() -> dict:
    from cases import random_csr

    from oracle import oracle

    out = {}
    for name, rows, cols, dens, seed, empty, dups, unsorted in CONVERSION_CASES:
        ptr, idx, val = random_csr(rows, cols, dens, seed, empty, True, dups, unsorted)
        out[f"{name}/ptr"], out[f"{name}/idx"], out[f"{name}/val"] = ptr, idx, val
        out[f"{name}/shape"] = np.array([rows, cols], np.uint32)
        for B in BLOCK_SIZES:
            r = oracle.ref_blocked_ell_from_compressed(rows, cols, ptr, idx, val, B)
            out[f"{name}/bell{B}/bci"] = r["bci"]
            out[f"{name}/bell{B}/val"] = r["val"]
            out[f"{name}/bell{B}/meta"] = np.array([r["ell_cols"], r["nnz"]], np.uint64)
        if dups == 0 and unsorted == 0:
            for h in SLICE_ROWS:
                r = oracle.ref_sliced_ell_from_compressed(rows, cols, ptr, idx, val, h)
                out[f"{name}/sell{h}/offsets"] = r["offsets"]
                out[f"{name}/sell{h}/widths"] = r["widths"]
                out[f"{name}/sell{h}/col_idx"] = r["col_idx"]
                out[f"{name}/sell{h}/val"] = r["val"]
                out[f"{name}/sell{h}/meta"] = np.array([r["slice_count"], r["nnz"], r["total_slots"]], np.uint64)
        t = oracle.ref_choose_blocked_ell_block_size(rows, cols, ptr, idx, val, BLOCK_CANDIDATES)
        out[f"{name}/choose_bell"] = np.array([t[0], t[2]], np.uint64)
        out[f"{name}/choose_bell_fill"] = np.array([t[1]], np.float64)
        s = oracle.ref_choose_sliced_ell_slice_rows(rows, cols, ptr, idx, val, SLICE_CANDIDATES)
        out[f"{name}/choose_sell"] = np.array([s["slice_rows"], s["slice_count"], s["padded_slots"],
                                               s["padded_bytes"]], np.uint64)
        out[f"{name}/choose_sell_f"] = np.array([s["storage_ratio"], s["slice_penalty"], s["score"]], np.float64)
        # Blocked-ELL -> Sliced-ELL on the reference's own Blocked-ELL of this case; the
        # B = 4 matrix also gets a -0.0 and a NaN value (zero and live as floats)
        for B in BELL_TO_SELL_BLOCKS:
            key = f"{name}/bell{B}"
            bci, bval = out[f"{key}/bci"], out[f"{key}/val"].copy()
            ell_cols, bnnz = (int(x) for x in out[f"{key}/meta"])
            if B == 4 and bval.size >= 2:
                bval[0], bval[bval.size // 2] = 0x8000, 0x7E00
                out[f"{key}/val_special"] = bval
            for h in BELL_TO_SELL_ROWS:
                r = oracle.ref_sliced_ell_from_blocked_ell(rows, cols, bnnz, B, ell_cols, bci, bval, h)
                k2 = f"{key}/sell{h}"
                out[f"{k2}/widths"] = r["widths"]
                out[f"{k2}/col_idx"] = r["col_idx"]
                out[f"{k2}/val"] = r["val"]
                out[f"{k2}/meta"] = np.array([r["slice_count"], r["nnz"], r["total_slots"]], np.uint64)
            t = oracle.ref_choose_sliced_ell_slice_rows_from_blocked_ell(rows, cols, bnnz, B, ell_cols, bci, bval,
                                                                         SLICE_CANDIDATES)
            out[f"{key}/choose_sell"] = np.array([t["slice_rows"], t["slice_count"], t["padded_slots"],
                                                  t["padded_bytes"]], np.uint64)
    return out


BUCKET_BLOCKS = [4, 16]
BUCKET_SLICES = [3, 32]
BUCKET_REQUESTS = [1, 2, 3, 8]


def ref_bucketing(conv: dict) -> dict:
    """The reference's bucketed partitions of the conversion cases' own Blocked-ELL
    and Sliced-ELL matrices (taken from `conv`)."""
    from oracle import oracle

    out = {}
    names = sorted({k.split("/")[0] for k in conv})
    for name in names:
        rows, cols = (int(x) for x in conv[f"{name}/shape"])
        for B in BUCKET_BLOCKS:
            key = f"{name}/bell{B}"
            bci, bval = conv[f"{key}/bci"], conv[f"{key}/val"]
            ell_cols, bnnz = (int(x) for x in conv[f"{key}/meta"])
            for req in BUCKET_REQUESTS:
                r = oracle.ref_build_bucketed_bell(rows, cols, bnnz, B, ell_cols, bci, bval, req)
                k2 = f"{key}/bucket{req}"
                segs = r["segments"]
                out[f"{k2}/meta"] = np.array([r["segment_count"], r["bytes"]], np.uint64)
                out[f"{k2}/seg"] = np.array([[g["rows"], g["ell_cols"], g["nnz"]] for g in segs], np.uint32)
                out[f"{k2}/bci"] = np.concatenate([g["bci"] for g in segs] + [np.zeros(0, np.uint32)])
                out[f"{k2}/val"] = np.concatenate([g["val"] for g in segs] + [np.zeros(0, np.uint16)])
                out[f"{k2}/e2c"] = r["e2c"]
            out[f"{key}/choose"] = np.array(oracle.ref_choose_bucket_count_for_part(rows, cols, bnnz, B, ell_cols,
                                                                                   bci, bval), np.uint64)
        for h in BUCKET_SLICES:
            key = f"{name}/sell{h}"
            if f"{key}/widths" not in conv:
                continue
            offs, widths, col, val = (conv[f"{key}/{f}"] for f in ("offsets", "widths", "col_idx", "val"))
            nnz = int(conv[f"{key}/meta"][1])
            for req in BUCKET_REQUESTS:
                r = oracle.ref_build_bucketed_sell(rows, cols, nnz, offs, widths, col, val, req)
                k2 = f"{key}/bucket{req}"
                segs = r["segments"]
                out[f"{k2}/meta"] = np.array([r["segment_count"], r["bytes"]], np.uint64)
                out[f"{k2}/seg"] = np.array([[g["rows"], int(g["widths"][0]) if g["slice_count"] else 0, g["nnz"]]
                                             for g in segs], np.uint32)
                out[f"{k2}/col_idx"] = np.concatenate([g["col_idx"] for g in segs] + [np.zeros(0, np.uint32)])
                out[f"{k2}/val"] = np.concatenate([g["val"] for g in segs] + [np.zeros(0, np.uint16)])
                out[f"{k2}/e2c"] = r["e2c"]
            out[f"{key}/choose"] = np.array(oracle.ref_choose_bucket_count_for_sliced_part(rows, cols, nnz, offs,
                                                                                          widths, col, val), np.uint64)
    return out


COO_BLOCKS = [2, 3, 8, 16]
COO_CANDIDATES = [2, 4, 8, 16]


def coo_case(name, rows, cols, ptr, idx, val, seed):
    """The CSR case as COO: entries shuffled; every third case repeats a few
    (row, column) pairs with other values, every second gets a column map."""
    rng = np.random.default_rng(seed)
    row = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(ptr.astype(np.int64)))
    col, v = idx.astype(np.uint32), val.astype(np.uint16)
    if seed % 3 == 0 and len(row) > 4:
        k = rng.integers(0, len(row), 4)
        row, col = np.concatenate([row, row[k]]), np.concatenate([col, col[k]])
        v = np.concatenate([v, (v[k] ^ 0x0400).astype(np.uint16)])
    p = rng.permutation(len(row))
    fmap = rng.permutation(cols).astype(np.uint32) if seed % 2 == 0 else None
    return row[p].astype(np.uint32), col[p].astype(np.uint32), v[p].astype(np.uint16), fmap


def ref_coo(conv: dict) -> dict:
    from oracle import oracle

    out = {}
    names = sorted({k.split("/")[0] for k in conv})
    for seed, name in enumerate(names):
        rows, cols = (int(x) for x in conv[f"{name}/shape"])
        row, col, val, fmap = coo_case(name, rows, cols, conv[f"{name}/ptr"], conv[f"{name}/idx"],
                                       conv[f"{name}/val"], seed)
        out[f"{name}/coo/row"], out[f"{name}/coo/col"], out[f"{name}/coo/val"] = row, col, val
        if fmap is not None:
            out[f"{name}/coo/map"] = fmap
        for B in COO_BLOCKS:
            r = oracle.ref_blocked_ell_from_coo(rows, cols, cols, row, col, val, B, fmap)
            out[f"{name}/coo{B}/bci"], out[f"{name}/coo{B}/val"] = r["bci"], r["val"]
            out[f"{name}/coo{B}/meta"] = np.array([r["ell_cols"], r["nnz"]], np.uint64)
        t = oracle.ref_choose_block_size_from_coo(rows, cols, cols, row, col, val, COO_CANDIDATES, fmap)
        out[f"{name}/coo_choose"] = np.array([t[0], t[2]], np.uint64)
        out[f"{name}/coo_choose_fill"] = np.array([t[1]], np.float64)
    return out


def main() -> None:
    (HERE / "mask_groups_known_answers.json").write_text(json.dumps(known_answers(), indent=1) + "\n")
    from oracle import oracle

    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libcs_ref.so missing: run `make -C oracle ref` with the reference tree present")
    conv = ref_conversions()
    np.savez_compressed(HERE / "ref_conversions.npz", **conv)
    if not oracle.ref_bucket_available():
        raise SystemExit("oracle/_ref/libcs_ref_bucket.so missing: run `make -C oracle ref`")
    np.savez_compressed(HERE / "ref_bucketing.npz", **ref_bucketing(conv))
    np.savez_compressed(HERE / "ref_coo.npz", **ref_coo(conv))
    print("wrote", HERE / "mask_groups_known_answers.json", HERE / "ref_conversions.npz",
          HERE / "ref_bucketing.npz", HERE / "ref_coo.npz")


if __name__ == "__main__":
    main()
