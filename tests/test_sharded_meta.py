"""The C++ shim's sharded<T> host helpers (include/cellshard_b200.hpp) against
the reference's own (runtime/layout/sharded.cuh, runtime/host/sharded_host.cuh,
compiled into oracle/_ref/libcs_ref_sharded.so) on the CPU: the stitched
matrix's layout, the shard cut rules (equal rows, nnz limit, host-byte limit,
row targets, explicit offsets) and the row -> partition / shard -> partition
lookups, on random metadata-only partition tables, must agree exactly."""

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
UL = C.c_ulong


@pytest.fixture(scope="module")
def libs(cs_lib, tmp_path_factory):
    from oracle import oracle

    ref_path = oracle.HERE / "_ref" / "libcs_ref_sharded.so"
    if not ref_path.exists():
        pytest.skip("reference sharded bridge not built")
    d = tmp_path_factory.mktemp("sharded")
    so = d / "libshim_sharded.so"
    cuda_inc = Path(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc").resolve().parents[1] / "include"
    subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-I", str(ROOT / "include"), "-I", str(cuda_inc),
                    "-o", str(so), str(ROOT / "tests" / "cpp" / "sharded_meta.cpp"), "-L", str(ROOT / "cellshard_b200"),
                    "-lcellshard_b200", f"-Wl,-rpath,{ROOT / 'cellshard_b200'}"], check=True)
    return C.CDLL(str(ref_path)), C.CDLL(str(so))


def _arr(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _table(rng, n):
    rows = rng.integers(0, 300, n).astype(np.uint64)
    nnz = (rows * rng.integers(0, 40, n)).astype(np.uint64)
    B = rng.choice([2, 4, 8, 16], n).astype(np.uint64)
    W = rng.integers(0, 50, n).astype(np.uint64)
    aux = (W << np.uint64(16)) | B
    return rows, nnz, aux


def _cuts(lib, fn, mode, rows, nnz, aux, param, offsets_in=None):
    n = len(rows)
    offs = np.zeros(n + 2, np.uint64) if offsets_in is None else _arr(np.concatenate([offsets_in, [0]]))
    parts = np.zeros(n + 2, np.uint64)
    f = getattr(lib, fn)
    f.restype = C.c_long
    c = f(C.c_int(mode), UL(n), _p(rows), _p(nnz), _p(aux), UL(1000), UL(param), _p(offs), _p(parts))
    if c < 0:
        return (c,)
    return c, offs[:c + 1].tolist(), parts[:c + 1].tolist() if mode != 3 else None


def test_sharded_layout_matches_reference(libs):
    ref, shim = libs
    a = np.zeros(7, np.uint64)
    b = np.zeros(7, np.uint64)
    ref.csref_sharded_layout(_p(a))
    shim.cs_shim_sharded_layout(_p(b))
    assert a.tolist() == b.tolist()


@pytest.mark.parametrize("seed", range(12))
def test_shard_cut_rules_match_reference(libs, seed):
    ref, shim = libs
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 40))
    rows, nnz, aux = (_arr(x) for x in _table(rng, n))
    total_rows = int(rows.sum())
    for mode, params in ((0, [0, 1, 2, 3, n // 2 + 1, n, n + 5]),
                         (1, [0, 1, int(nnz.max(initial=0)), int(nnz.sum()) // 3 + 1, 10 ** 9]),
                         (2, [0, 1, 4096, 200_000, 10 ** 12]),
                         (3, [0, 1, 150, total_rows // 4 + 1, 10 ** 9])):
        for prm in params:
            assert _cuts(ref, "csref_shard_cuts", mode, rows, nnz, aux, prm) == \
                _cuts(shim, "cs_shim_shard_cuts", mode, rows, nnz, aux, prm), (mode, prm)
    # explicit offsets: partition boundaries, a non-boundary, a wrong end
    bounds = np.concatenate([[0], np.cumsum(rows)]).astype(np.uint64)
    pick = np.unique(rng.choice(bounds, size=min(len(bounds), 4)))
    good = np.unique(np.concatenate([[0], pick, [total_rows]])).astype(np.uint64)
    tries = [good, np.array([0, total_rows + 1], np.uint64)]
    if total_rows > 2 and (total_rows // 2) not in set(bounds.tolist()):
        tries.append(np.array([0, total_rows // 2, total_rows], np.uint64))
    for offs in tries:
        k = len(offs) - 1
        assert _cuts(ref, "csref_shard_cuts", 4, rows, nnz, aux, k, offs) == \
            _cuts(shim, "cs_shim_shard_cuts", 4, rows, nnz, aux, k, offs), offs.tolist()


@pytest.mark.parametrize("seed", range(6))
def test_shard_lookups_match_reference(libs, seed):
    ref, shim = libs
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 30))
    rows, nnz, aux = (_arr(x) for x in _table(rng, n))
    shards = int(rng.integers(1, n + 2))
    out = []
    for lib, fn in ((ref, "csref_shard_queries"), (shim, "cs_shim_shard_queries")):
        por = np.zeros(int(rows.sum()) + 1, np.uint64)
        info = np.zeros(4 * (n + 1), np.uint64)
        pb = np.zeros(n, np.uint64)
        getattr(lib, fn)(UL(n), _p(rows), _p(nnz), _p(aux), UL(1000), UL(shards), _p(por), _p(info), _p(pb))
        out.append((por.tolist(), info.tolist(), pb.tolist()))
    assert out[0] == out[1]
