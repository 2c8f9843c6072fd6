"""Precision study of grouped moments: the three accumulation schemes against
the FP64 oracle on NB counts with 1 % of rows scaled x100.

The matrix is the precision workload (32,768 columns, ~3 % density, 1 % x100
outlier rows, stored as Blocked-ELL with 16 x 16 blocks), 256 uniform row
labels, all rows and features kept.  Two value sets: the integer counts
themselves, and the counts scaled by 0.731 and rounded to fp16 (non-integer,
like size-factor-normalised expression), where fp32 sums stop being exact.
The row count defaults to 20,000 so the test stays short;
CS_PRECISION_ROWS=1000000 runs the full-size study.  The per-scheme max and
median relative errors of mean and variance (fp32 outputs; the FP64-combine
scheme also through its fp64 outputs) are printed as one JSON line.

Tolerance: the two compensated schemes stay within 1e-6 relative of FP64
for the mean; the FP64-combine scheme also for the variance.  Plain FP32 is
reported, and only required to be finite.
"""

import json
import os

import numpy as np
import pytest

from cases import np_u16, np_u32

pytestmark = pytest.mark.gpu

G = 256
RTOL = 1e-6


def _rel(got, exp, mask):
    e = np.abs(got[mask] - exp[mask]) / np.abs(exp[mask])
    return (float(e.max()), float(np.median(e))) if e.size else (0.0, 0.0)


@pytest.mark.parametrize("values", ["counts", "scaled"])
def test_precision_three_schemes(cuda, orc, values):
    import torch

    from cellshard_b200 import runtime, synth
    from cellshard_b200.device import CSR, blocked_ell_from_csr

    rows = int(os.environ.get("CS_PRECISION_ROWS", "20000"))
    spec = synth.precision_spec(rows)
    csr = synth.make_csr(spec)
    if values == "scaled":
        csr = CSR(csr.rows, csr.cols, csr.ptr, csr.idx, (csr.val.float() * 0.731).half())
    bell = blocked_ell_from_csr(csr, 16)
    labels = np.random.default_rng(spec.seed + 7).integers(0, G, rows).astype(np.uint32)
    d_lab = torch.from_numpy(labels.view(np.int32).copy()).cuda()
    ptr, idx, val = np_u32(csr.ptr), np_u32(csr.idx), np_u16(csr.val)
    del csr
    ref = orc.group_moments_csr(rows, spec.cols, ptr, idx, val, None, None, labels, G, ddof=1,
                                nthreads=os.cpu_count() or 1)
    m_mask = ref["mean"] != 0
    v_mask = ref["var"] > 0
    report = {"values": values, "rows": rows, "cols": spec.cols, "groups": G, "nnz": int(ptr[-1]),
              "outlier_rows_frac": 0.01, "ell_cols": bell.ell_cols, "schemes": {}}
    names = {runtime.PLAIN_F32: "plain_f32", runtime.TWOSUM_F32: "twosum_f32",
             runtime.TWOSUM_F64_COMBINE: "twosum_f32_f64_combine"}
    errs = {}
    for scheme, name in names.items():
        f64 = scheme == runtime.TWOSUM_F64_COMBINE
        res = runtime.compute_sparse_group_moments(bell, G, None, None, d_lab, scheme=scheme, ddof=1, want_f64=f64)
        torch.cuda.synchronize()
        assert int(res["status"].item()) == 0
        assert np.array_equal(res["group_rows"].cpu().numpy().astype(np.int64),
                              ref["group_rows"].astype(np.int64))
        mean = res["mean"].cpu().numpy().astype(np.float64)
        var = res["var"].cpu().numpy().astype(np.float64)
        assert np.all(np.isfinite(mean)) and np.all(np.isfinite(var))
        errs[name] = {"mean": _rel(mean, ref["mean"], m_mask), "var": _rel(var, ref["var"], v_mask)}
        report["schemes"][name] = {"mean_max_rel": errs[name]["mean"][0], "mean_median_rel": errs[name]["mean"][1],
                                   "var_max_rel": errs[name]["var"][0], "var_median_rel": errs[name]["var"][1]}
        if f64:
            m64 = res["mean64"].cpu().numpy()
            v64 = res["var64"].cpu().numpy()
            e_m, e_v = _rel(m64, ref["mean"], m_mask), _rel(v64, ref["var"], v_mask)
            errs[name + "_fp64_out"] = {"mean": e_m, "var": e_v}
            report["schemes"][name]["fp64_outputs"] = {"mean_max_rel": e_m[0], "mean_median_rel": e_m[1],
                                                       "var_max_rel": e_v[0], "var_median_rel": e_v[1]}
    print(json.dumps({"precision_study": report}))
    assert errs["twosum_f32"]["mean"][0] <= RTOL
    assert errs["twosum_f32_f64_combine"]["mean"][0] <= RTOL
    assert errs["twosum_f32_f64_combine"]["var"][0] <= RTOL
    assert errs["twosum_f32_f64_combine_fp64_out"]["mean"][0] <= RTOL
    assert errs["twosum_f32_f64_combine_fp64_out"]["var"][0] <= RTOL
