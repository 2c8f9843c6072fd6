"""The C++ drop-in shim (include/cellshard_b200.hpp): a C++ program written
the way reference host code is written (cellshard::runtime / device /
convert / bucket calls, workspaces, device::upload staging) is compiled
against the shim and the library, run on the GPU, and its results checked:
the mask_groups known answers of the reference's runtime test, and the
restatement for the conversion, chooser, bucketing, reoptimize and transpose
calls on the same inputs."""

import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
KA = json.loads((ROOT / "tests" / "golden" / "mask_groups_known_answers.json").read_text())


def _inputs_text():
    lines = [f"rows {KA['rows']}", f"cols {KA['cols']}", "group_masks " + " ".join(map(str, KA["group_masks"])),
             "row_keep " + " ".join(map(str, KA["row_keep"])), "feature_keep " + " ".join(map(str, KA["feature_keep"])),
             f"group_count {KA['group_count']}", "filter " + " ".join(map(str, KA["filter"]))]
    for sec in ("blocked", "compressed", "sliced", "reoptimize"):
        for k, v in KA[sec].items():
            lines.append(f"{sec}.{k} " + (" ".join(map(str, v)) if isinstance(v, list) else str(v)))
    return "\n".join(lines) + "\n"


@pytest.fixture(scope="module")
def shim_out(cuda, tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    d = tmp_path_factory.mktemp("shim")
    exe = d / "shim_runtime_test"
    lib = ROOT / "cellshard_b200"
    subprocess.run([nvcc, "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", str(ROOT / "include"), "-o", str(exe),
                    str(ROOT / "tests" / "cpp" / "shim_runtime_test.cpp"), "-L", str(lib), "-lcellshard_b200",
                    "-Xlinker", f"-rpath,{lib}"], check=True)
    inp = d / "inputs.txt"
    inp.write_text(_inputs_text())
    p = subprocess.run([str(exe), str(inp)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    out = {}
    for line in p.stdout.splitlines():
        parts = line.split()
        out[parts[0]] = np.array([float(x) for x in parts[1:]])
    return out


def close(a, b, tol=1e-3):
    return abs(float(a) - float(b)) <= tol


def test_shim_mask_groups_known_answers(shim_out):
    o = shim_out
    e = KA["expect_blocked"]
    assert all(close(a, b) for a, b in zip(o["blocked.row_totals"], e["row_totals"]))
    assert list(o["blocked.detected"]) == e["detected"] and list(o["blocked.keep"]) == e["keep"]
    for k, v in e["group_counts"].items():
        assert close(o["blocked.group_counts"][int(k)], v)
    for k, v in e["group_percentages"].items():
        assert close(o["blocked.group_percentages"][int(k)], v)
    assert close(o["no_groups.row_totals"][0], 15) and o["no_groups.detected"][0] == 3
    assert "no_groups.group_counts" not in o
    assert o["null_filter"][0] == 0
    assert close(o["compressed.row_totals"][2], 7) and close(o["compressed.group_counts"][8], 2)
    assert close(o["sliced.row_totals"][0], 8) and close(o["sliced.row_totals"][3], 18)
    assert list(o["sliced.view"]) == [KA["sliced"]["slice_rows"], len(KA["sliced"]["widths"])]
    assert list(o["sliced.slot_offsets"]) == KA["sliced"]["slot_offsets"]
    er = KA["expect_reoptimize"]
    assert list(o["reoptimize.meta"]) == [er["kept_rows"], er["kept_features"], er["live_nnz"]]
    assert o["done"][0] == 0


def test_shim_matches_c_abi_path(shim_out, cuda):
    """The shim adds no arithmetic: its reduce outputs equal the C-ABI path's."""
    import torch

    from cellshard_b200 import runtime
    from cellshard_b200.device import BlockedELL

    b = KA["blocked"]
    bell = BlockedELL(KA["rows"], KA["cols"], b["block_size"], b["ell_cols"],
                      torch.tensor(b["block_cols"], dtype=torch.int32, device="cuda"),
                      torch.tensor(b["values"], dtype=torch.float16, device="cuda"))
    f = KA["filter"]
    r = runtime.compute_sparse_group_reduce(
        bell, torch.tensor(np.array(KA["group_masks"], np.uint32).view(np.int32), device="cuda"), 3,
        torch.tensor(KA["row_keep"], dtype=torch.uint8, device="cuda"),
        torch.tensor(KA["feature_keep"], dtype=torch.uint8, device="cuda"), runtime.FilterParams(*f))
    torch.cuda.synchronize()
    assert np.array_equal(r["row_totals"].cpu().numpy(), shim_out["blocked.row_totals"].astype(np.float32))
    assert np.array_equal(r["group_counts"].cpu().numpy().ravel(),
                          shim_out["blocked.group_counts"].astype(np.float32))
    assert np.array_equal(r["group_percentages"].cpu().numpy().ravel(),
                          shim_out["blocked.group_percentages"].astype(np.float32))


def test_shim_convert_bucket_transpose_reoptimize(shim_out, orc):
    o = shim_out
    c = KA["compressed"]
    rows, cols = KA["rows"], KA["cols"]
    ptr = np.array(c["ptr"], np.uint32)
    idx = np.array(c["idx"], np.uint32)
    val = np.array(c["values"], np.float16).view(np.uint16)
    ref = orc.blocked_ell_from_csr(rows, cols, ptr, idx, val, 2)
    assert list(o["convert.blocked"][:2]) == [2, ref["ell_cols"]] and o["convert.blocked"][2] == ref["nnz"]
    assert np.array_equal(o["convert.block_cols"].astype(np.uint32), ref["bci"])
    assert np.array_equal(o["convert.values"].astype(np.float16).view(np.uint16), ref["val"])
    # Blocked-ELL (B = 2) -> Sliced-ELL at the height the chooser picks from 2 / 4 / 8
    lp, _, _ = orc.bell_live_csr(rows, cols, 2, ref["ell_cols"], ref["bci"], ref["val"])
    hb = orc.choose_sliced_slice_rows(rows, ref["nnz"], lp, (2, 4, 8))[0]
    sb = orc.sliced_ell_from_bell(rows, cols, 2, ref["ell_cols"], ref["bci"], ref["val"], hb)
    assert list(o["convert.sell_from_bell"]) == [hb, sb["slice_count"], ref["nnz"]]
    assert np.array_equal(o["convert.sell_from_bell.col"].astype(np.uint32), sb["col_idx"])
    assert np.array_equal(o["convert.sell_from_bell.val"].astype(np.float16).view(np.uint16), sb["val"])
    # execution bucketing of that Sliced-ELL and of the Blocked-ELL-2, both choosers, the ingest plan
    eb = orc.sell_bucketed(rows, sb["offsets"], sb["widths"], sb["col_idx"], sb["val"], 2)
    seg_nnz = [int(sum(eb["row_widths"][eb["order"][eb["seg_row"][k]:eb["seg_row"][k + 1]]]))
               for k in range(eb["segment_count"])]
    want = [eb["segment_count"], eb["bytes"]]
    for k in range(eb["segment_count"]):
        want += [int(eb["seg_row"][k + 1] - eb["seg_row"][k]), int(eb["seg_w"][k]), seg_nnz[k]]
    assert list(o["exec.sell"]) == want
    assert np.array_equal(o["exec.sell.e2c"].astype(np.uint32), eb["e2c"])
    assert tuple(o["exec.sell.choose"]) == orc.sell_choose_bucket_count(rows, sb["offsets"], sb["widths"],
                                                                         sb["col_idx"])
    bb = orc.bell_bucketed(rows, 2, ref["ell_cols"], ref["bci"], ref["val"], 2)
    want = [bb["segment_count"], bb["bytes"]]
    for k in range(bb["segment_count"]):
        rbs = bb["order"][bb["seg_rb"][k]:bb["seg_rb"][k + 1]]
        nnz_k = int(sum(min(2, rows - 2 * int(r)) * int(bb["widths"][r]) * 2 for r in rbs))
        want += [int(bb["seg_rows"][k]), int(bb["seg_w"][k]) * 2, nnz_k]
    assert list(o["exec.bell"]) == want
    assert np.array_equal(o["exec.bell.block_cols"].astype(np.uint32), bb["seg_bci"])
    assert np.array_equal(o["exec.bell.e2c"].astype(np.uint32), bb["e2c"])
    assert list(o["exec.bell.choose"]) == [*orc.bell_choose_bucket_count(rows, 2, ref["ell_cols"], ref["bci"]),
                                          orc.bell_choose_ingest_bucket_count(rows, 2, ref["ell_cols"], ref["bci"])]
    po, pw = orc.bell_bucket_plan(rows, 2, ref["ell_cols"], ref["bci"])
    assert np.array_equal(o["exec.plan.order"].astype(np.uint32), po)
    assert np.array_equal(o["exec.plan.width"].astype(np.uint32), pw)
    # the same matrix as reversed COO through the COO chooser (2 / 4) and builder
    crow = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(ptr.astype(np.int64)))[::-1].copy()
    ccol, cval = idx[::-1].copy(), val[::-1].copy()
    cb, _fill, _pad = orc.choose_block_size_from_coo(rows, cols, crow, ccol, (2, 4))
    cref = orc.blocked_ell_from_coo(rows, cols, crow, ccol, cval, cb)
    assert list(o["coo.blocked"]) == [cb, cref["ell_cols"], cref["nnz_gpu"]]
    assert np.array_equal(o["coo.block_cols"].astype(np.uint32), cref["bci"])
    assert np.array_equal(o["coo.values"].astype(np.float16).view(np.uint16), cref["val"])
    h, score, _ = orc.choose_sliced_slice_rows(rows, int(ptr[-1]), ptr, (16, 32, 64))
    assert o["convert.slice_choice"][0] == h and o["convert.slice_choice"][3] == score
    _nnz, _srt, order, offs = orc.major_nnz_plan(ptr, rows, 2)
    assert np.array_equal(o["bucket.order"].astype(np.uint32), order)
    assert np.array_equal(o["bucket.offsets"].astype(np.uint32), offs)
    rptr, _ridx, _rval, rinv = orc.rebuild(ptr, idx, val, rows, order)
    assert np.array_equal(o["bucket.rebuilt_ptr"].astype(np.uint32), rptr)
    assert np.array_equal(o["bucket.inverse"].astype(np.uint32), rinv)
    tptr, tidx, tval = orc.csr_transpose(rows, cols, ptr, idx, val)
    assert np.array_equal(o["transpose.ptr"].astype(np.uint32), tptr)
    assert np.array_equal(o["transpose.idx"].astype(np.uint32), tidx)
    assert np.array_equal(o["transpose.val"].astype(np.float16).view(np.uint16), tval)
    rr = KA["reoptimize"]
    b = KA["blocked"]
    major, ridx, rval = orc.reoptimize_bell(rows, cols, b["block_size"], b["ell_cols"],
                                            np.array(b["block_cols"], np.uint32),
                                            np.array(b["values"], np.float16).view(np.uint16),
                                            np.array(KA["row_keep"], np.uint8), np.array(KA["feature_keep"], np.uint8),
                                            np.array(rr["row_remap"], np.uint32),
                                            np.array(rr["feature_remap"], np.uint32), rr["output_rows"],
                                            rr["output_cols"])
    # filter (= the masked reoptimize's entries) -> bucket plan -> rebuild -> Blocked-ELL-2
    assert list(o["filter.meta"]) == [len(ridx), rr["output_rows"], 1]
    assert np.array_equal(o["filter.ptr"].astype(np.uint32), major)
    assert np.array_equal(o["filter.idx"].astype(np.uint32), ridx)
    _n, _s, order2, _o = orc.major_nnz_plan(major, rr["output_rows"], 2)
    assert np.array_equal(o["filter.bucket_order"].astype(np.uint32), order2)
    bp, bi, bv, _inv = orc.rebuild(major, ridx, rval, rr["output_rows"], order2)
    rep = orc.blocked_ell_from_csr(rr["output_rows"], rr["output_cols"], bp, bi, bv, 2)
    kept_src = int(np.count_nonzero(np.array(KA["row_keep"])))
    assert list(o["repack.meta"]) == [kept_src, len(ridx), rep["ell_width"], rep["ell_cols"]]
    assert np.array_equal(o["repack.block_cols"].astype(np.uint32), rep["bci"])
    assert np.array_equal(o["repack.values"].astype(np.float16).view(np.uint16), rep["val"])
    assert np.array_equal(o["reoptimize.ptr"].astype(np.uint32), major)
    assert np.array_equal(o["reoptimize.idx"].astype(np.uint32), ridx)
    assert np.array_equal(o["reoptimize.val"].astype(np.float16).view(np.uint16), rval)


SHARD_FILTER = (1.0, 1, 0.9, 0)
BELL_VIEW_BYTES = 48  # sizeof(device::blocked_ell_view)


def _r256(x):
    return (int(x) + 255) // 256 * 256


def _shard_parts(o):
    parts = []
    for p in range(5):
        rows, ell_cols, nnz, B = (int(x) for x in o[f"shard.part{p}.meta"])
        bci = o[f"shard.part{p}.bci"].astype(np.uint32)
        val = o[f"shard.part{p}.val"].astype(np.float16).view(np.uint16)
        parts.append((rows, ell_cols, nnz, B, bci, val))
    return parts


def test_shim_shard_staging_records_and_swap(shim_out):
    """sharded<blocked_ell> of five partitions (37/64/21/50/9 rows) cut into two shards
    by set_equal_shards; stage_shard packs a shard's partitions into one block (views
    48 bytes apart, the first partition owning the block); swap_shard stages shard 1
    and hands shard 0's block to the cache; restaging shard 0 takes that same block."""
    o = shim_out
    assert list(o["shard.offsets"]) == [0, 101, 181] and list(o["shard.parts"]) == [0, 2, 5]
    empty = [0, 0, 0, -1, -1]
    s0 = [0, 2, 1, 0, 0, 0, 2, 0, 0, BELL_VIEW_BYTES]
    s1 = [2, 5, 1, 0, 0, 2, 5, 0, 0, BELL_VIEW_BYTES, 2, 5, 0, 0, 2 * BELL_VIEW_BYTES]
    assert list(o["shard.records.s0"][:25]) == s0 + empty * 3
    assert list(o["shard.records.swapped"][:25]) == empty * 2 + s1
    assert list(o["shard.records.restaged"][:25]) == s0 + s1
    assert [o[f"shard.records.{k}.cache"][0] for k in ("s0", "swapped", "restaged")] == [0, 1, 0]
    assert o["shard.records.s0"].size == 25 and o["shard.reuse"].tolist() == [1, 1]


def test_shim_shard_staged_reduces_match_oracle(shim_out, orc):
    """Every partition staged as part of a shard (first staging, after the swap, after
    restaging from the cache) reduces to the restatement's per-row results."""
    o = shim_out
    masks = o["shard.group_masks"].astype(np.uint32)
    parts = _shard_parts(o)
    seen = 0
    for tag in ("shard.s0", "shard.s1", "shard.both"):
        for p, (rows, ell_cols, _nnz, B, bci, val) in enumerate(parts):
            key = f"{tag}.p{p}"
            if key + ".row_totals" not in o:
                continue
            ref = orc.group_reduce_bell(rows, 48, B, ell_cols, bci, val, masks, 4, None, None, SHARD_FILTER)
            assert np.array_equal(o[key + ".row_totals"].astype(np.float32), ref["row_totals"]), key
            assert np.array_equal(o[key + ".detected"].astype(np.uint32), ref["detected_features"]), key
            assert np.array_equal(o[key + ".max"].astype(np.float32), ref["max_values"]), key
            assert np.array_equal(o[key + ".keep"].astype(np.uint8), ref["row_keep"]), key
            assert np.array_equal(o[key + ".group_counts"].astype(np.float32), ref["group_counts"]), key
            seen += 1
    assert seen == 2 + 3 + 5


def test_shim_shard_bytes_and_cuts(shim_out):
    """Metadata-only device bytes equal the C ABI's for the materialised part; a packed
    shard takes one 256-byte view block plus each partition's arrays; the byte, nnz and
    explicit cuts follow the reference's rules; a host part dropped after upload stays
    staged, and once released cannot be staged again without a file backend."""
    o = shim_out
    parts = _shard_parts(o)
    b = o["shard.bytes"].astype(np.int64)
    per = b[:10].reshape(5, 2)
    assert np.array_equal(per[:, 0], per[:, 1])
    arrays = [_r256(((r + B - 1) // B) * (e // B) * 4) + _r256(r * e * 2) for (r, e, _n, B, _b, _v) in parts]
    assert list(per[:, 0]) == [256 + a for a in arrays]
    assert b[10] == per[0, 0] + per[1, 0] and b[11] == per[2:, 0].sum()
    assert b[12] == _r256(2 * BELL_VIEW_BYTES) + arrays[0] + arrays[1]

    def cut(weights, limit):
        offs, used, row, rows = [0], 0, 0, [p[0] for p in parts]
        for w, r in zip(weights, rows):
            if w and used and used + w > limit:
                offs.append(row)
                used = 0
            used += w
            row += r
        return offs + [sum(rows)]

    assert list(o["shard.by_device_bytes"]) == cut(list(per[:, 0]), per[0, 0] + per[1, 0])
    assert list(o["shard.by_nnz"]) == cut([p[2] for p in parts], 400)
    assert o["shard.reshard"].tolist() == [1, 0]
    assert o["shard.dropped"].tolist() == [1, 4, 5]
    assert o["shard.stage_codes"].tolist() == [0, 1]


def test_shim_compressed_and_sliced_shards(shim_out, orc):
    """A compressed and a Sliced-ELL shard of three partitions each, staged as one
    packed block apiece (the Sliced-ELL slot offsets computed on the device per
    partition); every staged partition reduces to the restatement's results."""
    o = shim_out
    masks = o["cshard.group_masks"].astype(np.uint32)
    for p in range(3):
        ptr = o[f"cshard.part{p}.ptr"].astype(np.uint32)
        idx = o[f"cshard.part{p}.idx"].astype(np.uint32)
        val = o[f"cshard.part{p}.val"].astype(np.float16).view(np.uint16)
        rows = len(ptr) - 1
        rc = orc.group_reduce_csr(rows, 48, ptr, idx, val, masks, 4, None, None, SHARD_FILTER)
        assert np.array_equal(o[f"cshard.c{p}.row_totals"].astype(np.float32), rc["row_totals"])
        assert np.array_equal(o[f"cshard.c{p}.detected"].astype(np.uint32), rc["detected_features"])
        assert np.array_equal(o[f"cshard.c{p}.group_counts"].astype(np.float32), rc["group_counts"])
        sl = orc.sliced_ell_from_csr(rows, ptr, idx, val, 8)
        assert np.array_equal(o[f"cshard.s{p}.slot_offsets"].astype(np.uint32), sl["slot_offsets"])
        rs = orc.group_reduce_sell(rows, 48, 8, sl["offsets"], sl["widths"], sl["slot_offsets"], sl["col_idx"],
                                   sl["val"], masks, 4, None, None, SHARD_FILTER)
        assert np.array_equal(o[f"cshard.s{p}.row_totals"].astype(np.float32), rs["row_totals"])
        assert np.array_equal(o[f"cshard.s{p}.group_counts"].astype(np.float32), rs["group_counts"])
        assert o[f"cshard.group"].tolist() == [0, 3, 0, 3]
