"""getSdf through the reference's own C++ signature (morphutils.h:40-41), as
the reference's partition_shapes calls it (TaiChi.cu:327): a small C++
program compiled against include/morphutils.h and linked to the library.
The shape corners must equal the golden ones (cv2 restatement of the
reference's getSdf, pinned by make_golden.py), and the widths cv2's
contourArea / corner distance (tests/golden/sdf_widths.json)."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests.golden import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu

SRC = r'''
#include <cstdio>
#include <string>
#include <vector>
#include "morphutils.h"
int main(int argc, char **argv)
{
    FILE *f = std::fopen(argv[1], "rb");
    int hdr[3];
    if (!f || std::fread(hdr, sizeof(int), 3, f) != 3) return 2;
    const int M = hdr[0], N = hdr[1], nnz = hdr[2];
    int *rp = new int[M + 1];
    int *col = new int[nnz > 0 ? nnz : 1];
    if (std::fread(rp, sizeof(int), M + 1, f) != (size_t)M + 1) return 2;
    if (nnz && std::fread(col, sizeof(int), nnz, f) != (size_t)nnz) return 2;
    std::fclose(f);
    float *val = nullptr;
    std::string category;
    Point_t size{-1, -1};
    int shapes = -1;
    std::vector<Point_t> pts;
    std::vector<double> widths;
    getSdf(std::string(argv[1]), M, N, nnz, rp, col, val, category, size, shapes, pts, widths);
    std::printf("RESULT %s %d %d %d %zu %zu\n", category.c_str(), size.x, size.y, shapes, pts.size(), widths.size());
    for (const Point_t &p : pts) std::printf("P %d %d\n", p.x, p.y);
    for (double w : widths) std::printf("W %.17g\n", w);
    delete[] rp;
    delete[] col;
    return 0;
}
'''


@pytest.fixture(scope="module")
def exe(tc, tmp_path_factory):
    d = tmp_path_factory.mktemp("getsdf")
    src, out = str(d / "sdf.cpp"), str(d / "sdf")
    with open(src, "w") as f:
        f.write(SRC)
    libdir = os.path.dirname(tc.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), src, "-o", out,
                    "-L", libdir, "-ltaichi_b200", "-Wl,-rpath," + libdir], check=True)
    return out


def run_getsdf(exe, tmp_path, M, N, rp, col):
    path = str(tmp_path / "m.bin")
    with open(path, "wb") as f:
        np.array([M, N, rp[M]], np.int32).tofile(f)
        np.ascontiguousarray(rp, np.int32).tofile(f)
        np.ascontiguousarray(col, np.int32).tofile(f)
    r = subprocess.run([exe, path], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    res = next(l for l in lines if l.startswith("RESULT")).split()
    pts = [tuple(map(int, l.split()[1:])) for l in lines if l.startswith("P ")]
    ws = [float(l.split()[1]) for l in lines if l.startswith("W ")]
    return res[1], (int(res[2]), int(res[3])), int(res[4]), pts, ws, r.stdout


NAMES = ["band_holes", "two_segments", "offdiag_blocks", "multi_shape", "many_shapes", "rmat16_selfloops",
         "mesh2048"]


@pytest.mark.parametrize("name", NAMES)
def test_getsdf_matches_golden(exe, tmp_path, golden, name):
    case = next(c for c in cases.MATRIX_CASES if c["name"] == name)
    rec = next(r for r in golden["partitions"] if r["name"] == name)
    with open(os.path.join(ROOT, "tests", "golden", "sdf_widths.json")) as f:
        want_w = json.load(f)["widths"][name]
    M, N, rp, col = cases.matrix(case)
    cat, size, n, pts, ws, _ = run_getsdf(exe, tmp_path, M, N, rp, col)
    assert cat == "diagonal" and size == (rec["mF"], rec["W"])
    corners = [list(pts[2 * i]) + list(pts[2 * i + 1]) for i in range(n)]
    assert corners == rec["corners"]
    assert len(ws) == len(want_w) == n
    np.testing.assert_allclose(ws, want_w, rtol=1e-12, atol=0)


def test_getsdf_too_small(exe, tmp_path):
    """At most 512 rows: the reference's message, category set, the other
    outputs untouched (morohutils.cu:186-196)."""
    M = N = 300
    rp = np.arange(M + 1, dtype=np.int32)
    col = np.arange(M, dtype=np.int32)
    cat, size, n, pts, ws, out = run_getsdf(exe, tmp_path, M, N, rp, col)
    assert "the matrix is too small! exit" in out
    assert cat == "diagonal" and size == (-1, -1) and n == -1 and not pts and not ws
