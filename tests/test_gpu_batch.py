"""Batched CSR -> Sliced-ELL + nnz plans over uneven partitions (one
persistent launch per wave from a device queue, CUDA-graph replay).

Per partition: the chosen slice height equals the chooser's (restated in
Python doubles, and the reference's own chooser when oracle/_ref is built);
the Sliced-ELL arrays equal the restatement (and the reference conversion)
at that height bit for bit; the plan equals the restatement of
build_major_nnz_bucket_plan_raw, and the power-of-two bins the restated
lower bounds.  Waves, tile shapes, autotuning and graph replay must not
change any output.
"""

import numpy as np
import pytest

from cases import np_u16, np_u32, random_csr, to_device_csr

pytestmark = pytest.mark.gpu

CANDS = (16, 32, 64)
ROWS = [0, 1, 5, 15, 16, 17, 63, 64, 65, 100, 1000, 2999, 4096, 4097, 7777]


def _host_parts(rows_list, seed, cols=300):
    out = []
    rng = np.random.default_rng(seed)
    for i, r in enumerate(rows_list):
        dens = float(rng.choice([0.005, 0.03, 0.2]))
        out.append((r, cols) + random_csr(r, cols, dens, seed * 1000 + i, 0.15, integer=bool(i % 2)))
    return out


def _device(parts):
    return [to_device_csr(r, c, p, i, v) for (r, c, p, i, v) in parts]


def _choose(orc, rows, nnz, ptr, cands):
    return orc.choose_sliced_slice_rows(rows, nnz, ptr, cands)


def _check_part(orc, hp, res, bucket_count=16):
    rows, cols, ptr, idx, val = hp
    assert res.status == 0, hex(res.status)
    nnz = int(ptr[-1]) if rows else 0
    if rows == 0:
        assert res.slice_rows == 0 and res.slice_count == 0
    else:
        h, score, _ = _choose(orc, rows, nnz, ptr, CANDS)
        assert res.slice_rows == h
        assert res.score == score
        ref = orc.sliced_ell_from_csr(rows, ptr, idx, val, h)
        s = res.sliced
        assert res.slice_count == ref["slice_count"] and res.total_slots == ref["total_slots"]
        assert np.array_equal(np_u32(s.slice_row_offsets), ref["offsets"])
        assert np.array_equal(np_u32(s.slice_widths), ref["widths"])
        assert np.array_equal(np_u32(s.slice_slot_offsets), ref["slot_offsets"])
        assert np.array_equal(np_u32(s.col_idx), ref["col_idx"])
        assert np.array_equal(np_u16(s.val), ref["val"])
    pl = res.plan
    if pl is not None:
        rnnz, srt, order, offs = orc.major_nnz_plan(ptr, rows, bucket_count)
        if rows == 0:
            assert int(np_u32(pl["bucket_offsets"])[0]) == 0
        else:
            assert np.array_equal(np_u32(pl["bucket_offsets"]), offs)
            assert np.array_equal(np_u32(pl["nnz"])[:rows], rnnz)
            assert np.array_equal(np_u32(pl["sorted"])[:rows], srt)
            assert np.array_equal(np_u32(pl["order"])[:rows], order)
            assert np.array_equal(np_u32(pl["pow2_bins"]), orc.pow2_bins(srt))


def test_batch_matches_restatement(cuda, orc):
    from cellshard_b200.batch import BatchSlicedConverter

    hp = _host_parts(ROWS, 1)
    conv = BatchSlicedConverter(_device(hp), CANDS, bucket_count=16)
    conv.run()
    results, deferred, err = conv.results()
    assert deferred == 0 and err == 0
    for h, r in zip(hp, results):
        _check_part(orc, h, r)


def test_batch_vs_reference_chooser_and_conversion(cuda, orc):
    if not orc.ref_available():
        pytest.skip("reference library not built")
    from cellshard_b200.batch import BatchSlicedConverter

    hp = _host_parts([37, 500, 2048, 3001], 2, cols=700)
    conv = BatchSlicedConverter(_device(hp), CANDS, with_plan=False)
    conv.run()
    results, deferred, err = conv.results()
    assert deferred == 0 and err == 0
    for (rows, cols, ptr, idx, val), r in zip(hp, results):
        ch = orc.ref_choose_sliced_ell_slice_rows(rows, cols, ptr, idx, val, list(CANDS))
        assert ch is not None and ch["slice_rows"] == r.slice_rows and ch["score"] == r.score
        ref = orc.ref_sliced_ell_from_compressed(rows, cols, ptr, idx, val, r.slice_rows)
        assert ref["total_slots"] == r.total_slots
        assert np.array_equal(np_u32(r.sliced.slice_row_offsets), ref["offsets"])
        assert np.array_equal(np_u32(r.sliced.slice_widths), ref["widths"])
        assert np.array_equal(np_u32(r.sliced.col_idx), ref["col_idx"])
        assert np.array_equal(np_u16(r.sliced.val), ref["val"])


def test_batch_waves_defer_and_finish(cuda, orc):
    import torch

    from cellshard_b200.batch import BatchSlicedConverter, part_bounds

    hp = _host_parts([900, 3000, 40, 2500, 1200, 700, 3100], 3)
    dev = _device(hp)
    b = part_bounds(dev, CANDS)
    small = max(sum(b) // 3, max(b))
    conv = BatchSlicedConverter(dev, CANDS, arena_bytes=small)
    done = {}
    waves = 0
    while True:
        conv.run()
        waves += 1
        results, deferred, err = conv.results()
        assert err == 0
        for i, r in enumerate(results):
            if i not in done and r.status == 0:
                # keep the converted partition: copy out of the arena before it is reused
                sl = r.sliced
                done[i] = (r, [np_u32(sl.slice_row_offsets), np_u32(sl.slice_widths), np_u32(sl.slice_slot_offsets),
                               np_u32(sl.col_idx), np_u16(sl.val)])
        if deferred == 0:
            break
        assert waves < len(hp) + 1
        conv.next_wave(torch.empty_like(conv.arena))
    assert waves > 1 and len(done) == len(hp)
    # reset: every partition forms one wave again in an arena that holds them all
    conv.reset(torch.empty(sum(b) + 4096, dtype=torch.uint8, device="cuda"))
    conv.run()
    results, deferred, err = conv.results()
    assert deferred == 0 and err == 0
    for h, r in zip(hp, results):
        _check_part(orc, h, r)
    # a partition larger than the whole arena is refused, not deferred forever
    tiny = BatchSlicedConverter(dev[:2], CANDS, arena_bytes=4096)
    tiny.run()
    res, deferred, err = tiny.results()
    assert err & 0x1000 and all(r.status & 0x1000 for r in res)
    for i, h in enumerate(hp):
        r, arrs = done[i]
        rows, cols, ptr, idx, val = h
        hh = _choose(orc, rows, int(ptr[-1]), ptr, CANDS)[0]
        ref = orc.sliced_ell_from_csr(rows, ptr, idx, val, hh)
        assert r.slice_rows == hh
        for got, key in zip(arrs, ("offsets", "widths", "slot_offsets", "col_idx", "val")):
            assert np.array_equal(got, ref[key]), (i, key)


@pytest.mark.parametrize("tiles", [
    {"layout_rows": 32, "emit_rows": 1, "emit_lanes": 4},
    {"layout_rows": 96, "emit_rows": 7, "emit_lanes": 8, "ctas_per_sm": 1},
    {"layout_rows": 8192, "emit_rows": 4096, "emit_lanes": 32},
])
def test_batch_tiles_do_not_change_results(cuda, orc, tiles):
    from cellshard_b200.batch import BatchSlicedConverter

    hp = _host_parts([3, 64, 1000, 4097, 150], 4)
    conv = BatchSlicedConverter(_device(hp), CANDS, tiles=tiles)
    assert conv.tiles()["emit_lanes"] == tiles["emit_lanes"]
    for _ in range(2):  # graph replay
        conv.run()
        results, deferred, err = conv.results()
        assert deferred == 0 and err == 0
        for h, r in zip(hp, results):
            _check_part(orc, h, r)


def test_batch_autotune_and_generated_partitions(cuda, orc):
    from cellshard_b200 import synth
    from cellshard_b200.batch import BatchSlicedConverter

    specs, parts, hp = [], [], []
    for k, rows in enumerate([2000, 5300, 3100, 9000]):
        spec = synth.MatrixSpec(rows, 32768, 0.025 * 32768, 1, 16384, seed=synth.SEED_BASE + 300 + k)
        csr = synth.make_csr(spec)
        parts.append(csr)
        hp.append((rows, 32768, np_u32(csr.ptr), np_u32(csr.idx), np_u16(csr.val)))
    conv = BatchSlicedConverter(parts, CANDS, bucket_count=8)
    t = conv.autotune()
    assert t["emit_lanes"] in (8, 16, 32) and t["items"] > 0
    conv.run()
    results, deferred, err = conv.results()
    assert deferred == 0 and err == 0
    for h, r in zip(hp, results):
        _check_part(orc, h, r, bucket_count=8)
