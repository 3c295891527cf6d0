/*
 * ref_bridge.cpp -- links against the reference's own TaiChi.cu / mmio.cpp
 * (compiled unmodified from their sources by oracle/build.py into
 * oracle/_ref/libtaichi_ref.so) and exposes them to the tests through plain
 * extern "C" entry points.  Test infrastructure only.
 *
 * The reference's getSdf (morohutils.cu:182-291) needs the OpenCV C++
 * library, which is not installed.  This file supplies getSdf with the same
 * signature (morphutils.h:40-41): it returns the shape corners that the
 * caller injected with ref_set_shapes() -- computed by cv2 (the stand-in for
 * OpenCV) in tests/golden/make_golden.py -- or, when none were injected, the
 * oracle's C restatement of the morphology.
 */
#include <cstring>
#include <string>
#include <vector>

#include "morphutils.h"
#include "TaiChi.h"

extern "C" {
#include "taichi_oracle.h"
}

char matrixName[1024] = "ref";   /* defined by the caller (main.cu:17) */

static bool g_inject = false;
static int g_mF = 0, g_W = 0;
static std::vector<int> g_corners;

void getSdf(string path, int M, int N, int nnz, int *&rowptr, int *&col,
            float *&val, string &category, Point_t &size, int &shapeNum,
            vector<Point_t> &shapePoints, vector<double> &widths)
{
    (void)path; (void)nnz; (void)val; (void)widths;
    category = "diagonal";
    int mF = 0, W = 0, n = 0;
    int *cs = nullptr;
    if (g_inject) {
        mF = g_mF; W = g_W; n = (int)g_corners.size() / 4; cs = g_corners.data();
    } else {
        or_params p;
        or_params_default(&p);
        n = or_getsdf(M, N, rowptr, col, &p, &mF, &W, &cs, nullptr);
        if (n < 0) n = 0;
    }
    if (mF == 0) return;   /* matrix too small: getSdf returns early */
    size.x = mF;
    size.y = W;
    shapeNum = n;
    for (int i = 0; i < n; ++i) {
        shapePoints.push_back(Point_t{cs[4 * i], cs[4 * i + 1]});
        shapePoints.push_back(Point_t{cs[4 * i + 2], cs[4 * i + 3]});
    }
    if (!g_inject) or_free(cs);
}

extern "C" {

void ref_set_shapes(int mF, int W, int n, const int *corners)
{
    g_inject = true; g_mF = mF; g_W = W;
    g_corners.assign(corners, corners + 4 * (size_t)n);
}

void ref_clear_shapes(void) { g_inject = false; g_corners.clear(); }

int ref_read_mtx(const char *path, int *m, int *n, unsigned long *nnz,
                 int **rowptr, int **col, float **val)
{
    int M = 0, N = 0;
    unsigned long z = 0;
    int *rp = nullptr, *ci = nullptr;
    float *va = nullptr;
    int rc = readMtx(const_cast<char *>(path), M, N, z, rp, ci, va);
    *m = M; *n = N; *nnz = z; *rowptr = rp; *col = ci; *val = va;
    return rc;
}

/* Runs partition_shapes on caller-owned CSR arrays (val is mutated) and
 * returns a malloc'd TaiChi_new.  When the format aliases the input CSR
 * (dense_nnz == 0) its csrRow/csrCol point into rowptr/col. */
TaiChi_new *ref_partition(int M, int N, int nnz, int *rowptr, int *col, float *val)
{
    TaiChi_new *t = (TaiChi_new *)malloc(sizeof(TaiChi_new));
    memset(t, 0, sizeof(TaiChi_new));
    int *rp = rowptr, *ci = col;
    float *va = val;
    partition_shapes(const_cast<char *>("ref.mtx"), M, N, nnz, rp, ci, va, t);
    return t;
}

void ref_free_taichi_new(TaiChi_new *t) { free_taichi_new(t); }

/* The reference's GPU multiply (needs a GPU; ends with cudaDeviceReset). */
void ref_taichi_spmv(int M, int N, TaiChi_new *t, float *x, float *y)
{
    taichi_SpMV(M, N, t, x, y);
}

void ref_free(void *p) { free(p); }

} /* extern "C" */
