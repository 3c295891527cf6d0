"""The C-ABI library loads and exports every entry point its headers declare
(no GPU needed), and its host-only reader matches the reference."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def header_c_symbols():
    text = open(os.path.join(ROOT, "include", "taichi_b200.h")).read()
    return sorted(set(re.findall(r"TC_API\s+[\w\s\*]*?\b(tc_\w+)\s*\(", text)))


def header_cpp_symbols():
    text = open(os.path.join(ROOT, "include", "TaiChi.h")).read()
    text += open(os.path.join(ROOT, "include", "morphutils.h")).read()
    return sorted(set(re.findall(r"TAICHI(?:_MORPH)?_API\s+\w+\s+(\w+)\s*\(", text)))


def test_c_symbols_exported(tc):
    syms = header_c_symbols()
    assert len(syms) >= 20
    L = tc.lib()
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(tc.EXPORTS) <= set(syms)


def test_flag_values_match_header(tc):
    """Every TC_FLAG_* of the C header has the same value in the Python view,
    and no two flags share a bit."""
    text = open(os.path.join(ROOT, "include", "taichi_b200.h")).read()
    flags = {k: int(v, 16) for k, v in re.findall(r"#define\s+(TC_FLAG_\w+)\s+(0x[0-9a-fA-F]+)", text)}
    assert "TC_FLAG_HOST_Y_MAPPED" in flags and len(flags) >= 15
    for k, v in flags.items():
        assert getattr(tc, k) == v, k
        assert v & (v - 1) == 0, k
    assert len(set(flags.values())) == len(flags)


def test_cpp_compat_symbols_exported(tc):
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", tc.LIB_PATH],
                         stdout=subprocess.PIPE, text=True, check=True).stdout
    names = set(re.findall(r" T (\w+)\(", out))
    missing = [s for s in header_cpp_symbols() if s not in names]
    assert not missing, missing
    # exact reference signatures (TaiChi.h:79-107)
    for sig in ("readMtx(char*, int&, int&, unsigned long&, int*&, int*&, float*&)",
                "partition_shapes(char*, int, int, int, int*&, int*&, float*&, TaiChi_new*)",
                "taichi_SpMV(int, int, TaiChi_new*, float*, float*)",
                "free_taichi_new(TaiChi_new*)",
                "getSdf(std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> >, "
                "int, int, int, int*&, int*&, float*&, std::__cxx11::basic_string<char, "
                "std::char_traits<char>, std::allocator<char> >&, Point_t&, int&, "
                "std::vector<Point_t, std::allocator<Point_t> >&, std::vector<double, "
                "std::allocator<double> >&)"):
        assert sig in out, sig


def test_struct_layout():
    """TaiChi_new / TaiChi / shape keep the reference's byte layout."""
    src = r'''
#include <cstddef>
#include <cstdio>
#include "TaiChi.h"
int main() {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(TaiChi_new), offsetof(TaiChi_new, xStart),
         offsetof(TaiChi_new, csrCol), sizeof(TaiChi), offsetof(TaiChi, nnz), sizeof(shape));
}'''
    import tempfile
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "l.cpp"), "w") as f:
        f.write(src)
    exe = os.path.join(d, "l")
    subprocess.run(["g++", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(d, "l.cpp"), "-o", exe], check=True)
    got = subprocess.run([exe], stdout=subprocess.PIPE, text=True, check=True).stdout.split()
    # 7 ints + pad, 7 pointers | char + 5 ints .. | 1 + 1024 + 10 ints
    assert [int(v) for v in got] == [88, 32, 80, 104, 80, 1068]


def test_status_strings(tc):
    L = tc.lib()
    assert L.tc_status_string(0) == b"ok"
    assert L.tc_status_string(7) == b"device wait timed out"


def test_read_mtx_matches_reference(tc, golden):
    for name, rec in golden["mtx"].items():
        path = os.path.join(GOLD, "mtx", name)
        if rec["rc"] != 0:
            with pytest.raises(tc.TcError) as e:
                tc.read_mtx(path)
            assert "reference code %d" % rec["rc"] in str(e.value)
            continue
        M, N, rp, col, val = tc.read_mtx(path)
        assert (M, N) == (rec["M"], rec["N"])
        assert rp.tolist() == rec["rowptr"] and col.tolist() == rec["col"], name
        np.testing.assert_array_equal(val, np.array(rec["val"], np.float32))


def test_read_mtx_large_parallel_parse(tc, tmp_path):
    """A file big enough for the multi-threaded parser gives the oracle's CSR."""
    import oracle
    from taichi_b200 import matgen
    M, N, rp, col = matgen.segments(40000, [(0, 40000, 0, 3, 0.9)], noise=20000, seed=3)
    path = str(tmp_path / "m.mtx")
    matgen.to_mtx(path, M, N, rp, col, field="integer", symmetric=False)
    got = tc.read_mtx(path)
    rc, want = oracle.read_mtx(path)
    assert rc == 0
    for a, b in zip(got[2:], want[2:]):
        np.testing.assert_array_equal(a, b)
    # symmetric storage: lower triangle written, both halves come back
    lo = col <= np.repeat(np.arange(M), np.diff(rp))
    rows = np.repeat(np.arange(M), np.diff(rp))[lo]
    keys = rows.astype(np.int64) * N + col[lo]
    from taichi_b200.matgen import _csr_from_keys
    lrp, lcol = _csr_from_keys(M, N, keys)
    matgen.to_mtx(path, M, N, lrp, lcol, field="pattern", symmetric=True)
    got = tc.read_mtx(path)
    rc, want = oracle.read_mtx(path)
    for a, b in zip(got[2:], want[2:]):
        np.testing.assert_array_equal(a, b)
