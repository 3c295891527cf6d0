/*
 * taichi_oracle.c -- CPU restatement of TaiChi's binary-SpMV path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  See taichi_oracle.h.
 * Written for clarity, sequentially, in the reference's own loop orders so
 * that every output (including FP32 sums of the serial CPU loop) matches.
 */
#define _GNU_SOURCE
#include "taichi_oracle.h"

#include <ctype.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

void or_params_default(or_params *p)
{
    p->thumb_height = 512;   /* morohutils.cu:191 */
    p->open_len = 30;        /* morohutils.cu:239,242 */
    p->eye_size = 5;         /* morohutils.cu:250 */
    p->min_contour = 80;     /* morohutils.cu:140 */
    p->min_shape_side = 1000;/* TaiChi.cu:379 */
    p->density = 0.6;        /* TaiChi.cu:757 */
}

void or_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Matrix Market -> CSR (TaiChi.cu:120-278, mmio.cpp:96-218)                 */
/* ------------------------------------------------------------------------ */

static void lower(char *s) { for (; *s; ++s) *s = (char)tolower((unsigned char)*s); }

int or_read_mtx(const char *path, int *m, int *n, unsigned long *nnz,
                int **rowptr, int **col, float **val)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[1025];
    char t0[64], t1[64], t2[64], t3[64], t4[64];
    /* banner: 5 tokens, "%%MatrixMarket matrix coordinate|array <type> <sym>" */
    if (!fgets(line, sizeof line, f) ||
        sscanf(line, "%63s %63s %63s %63s %63s", t0, t1, t2, t3, t4) != 5) {
        fclose(f); return -2;
    }
    lower(t1); lower(t2); lower(t3); lower(t4);
    int is_real = 0, is_int = 0, is_pat = 0, is_cplx = 0, is_sym = 0;
    if (strncmp(t0, "%%MatrixMarket", 14) != 0 || strcmp(t1, "matrix") != 0 ||
        (strcmp(t2, "coordinate") != 0 && strcmp(t2, "array") != 0)) {
        fclose(f); return -2;
    }
    if (!strcmp(t3, "real")) is_real = 1;
    else if (!strcmp(t3, "complex")) is_cplx = 1;
    else if (!strcmp(t3, "pattern")) is_pat = 1;
    else if (!strcmp(t3, "integer")) is_int = 1;
    else { fclose(f); return -2; }
    if (!strcmp(t4, "symmetric") || !strcmp(t4, "hermitian")) is_sym = 1;
    else if (strcmp(t4, "general") != 0 && strcmp(t4, "skew-symmetric") != 0) {
        fclose(f); return -2;
    }
    if (is_cplx) { fclose(f); return -3; }

    /* size line: skip '%' comment lines; "M N nnz" */
    int M = 0, N = 0;
    unsigned long nz = 0;
    do {
        if (!fgets(line, sizeof line, f)) { fclose(f); return -4; }
    } while (line[0] == '%');
    if (sscanf(line, "%d %d %lu", &M, &N, &nz) != 3) {
        int got;
        do {
            got = fscanf(f, "%d %d %lu", &M, &N, &nz);
            if (got == EOF) { fclose(f); return -4; }
        } while (got != 3);
    }
    if (M < 0 || N < 0) { fclose(f); return -4; }

    int *ri = (int *)malloc((nz ? nz : 1) * sizeof(int));
    int *ci = (int *)malloc((nz ? nz : 1) * sizeof(int));
    float *vi = (float *)malloc((nz ? nz : 1) * sizeof(float));
    int *cnt = (int *)calloc((size_t)M + 1, sizeof(int));
    for (unsigned long k = 0; k < nz; ++k) {
        int i = 0, j = 0, iv = 0, got = 0;
        double fv = 0.0;
        if (is_real) { got = fscanf(f, "%d %d %lg\n", &i, &j, &fv); got = got == 3; }
        else if (is_int) { got = fscanf(f, "%d %d %d\n", &i, &j, &iv); fv = iv; got = got == 3; }
        else if (is_pat) { got = fscanf(f, "%d %d\n", &i, &j); fv = 1.0; got = got == 2; }
        /* The reference does not check these; a short or out-of-range entry
         * makes it index out of bounds.  The oracle reports -5 instead. */
        if (!got || i < 1 || i > M || j < 1 || j > N) {
            free(ri); free(ci); free(vi); free(cnt); fclose(f); return -5;
        }
        ri[k] = i - 1; ci[k] = j - 1; vi[k] = (float)fv;
        cnt[i - 1]++;
    }
    fclose(f);
    if (is_sym) {
        for (unsigned long k = 0; k < nz; ++k)
            if (ri[k] != ci[k]) {
                if (ci[k] >= M) { free(ri); free(ci); free(vi); free(cnt); return -5; }
                cnt[ci[k]]++;
            }
    }
    int *rp = (int *)malloc(((size_t)M + 1) * sizeof(int));
    long run = 0;
    for (int r = 0; r < M; ++r) { rp[r] = (int)run; run += cnt[r]; }
    rp[M] = (int)run;
    int *co = (int *)malloc((run ? run : 1) * sizeof(int));
    float *va = (float *)malloc((run ? run : 1) * sizeof(float));
    memset(cnt, 0, ((size_t)M + 1) * sizeof(int));
    for (unsigned long k = 0; k < nz; ++k) {
        int i = ri[k], j = ci[k];
        int at = rp[i] + cnt[i]++;
        co[at] = j; va[at] = vi[k];
        if (is_sym && i != j) {
            at = rp[j] + cnt[j]++;
            co[at] = i; va[at] = vi[k];
        }
    }
    free(ri); free(ci); free(vi); free(cnt);
    *m = M; *n = N; *nnz = (unsigned long)run;
    *rowptr = rp; *col = co; *val = va;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Thumbnail + morphology (morohutils.cu:73-83, 153-261)                     */
/* ------------------------------------------------------------------------ */

int or_thumb_dims(int M, int N, int height, int *W, int *pM, int *pN)
{
    if (M <= height) return 0;
    *pM = M / height;
    double scale = (double)height / (double)M;
    *W = (int)(scale * N);
    if (*W <= 0) return -1;     /* the reference divides by zero here */
    *pN = N / *W;
    return 1;
}

void or_raster(int M, const int *rowptr, const int *col, int H, int W, int pM,
               int pN, unsigned char *img)
{
    memset(img, 255, (size_t)H * W);
    for (int i = 0; i < M; ++i) {
        int px = i / pM;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int py = col[k] / pN;
            if (px < H && py < W) img[(size_t)px * W + py] = 0;
        }
    }
}

void or_imfill(const unsigned char *src, int H, int W, unsigned char *dst)
{
    /* Flood the zero pixels 4-connected to a one-pixel zero frame around the
     * image; everything the flood cannot reach that is zero is a hole. */
    int PH = H + 2, PW = W + 2;
    unsigned char *reach = (unsigned char *)calloc((size_t)PH * PW, 1);
    int *stack = (int *)malloc((size_t)PH * PW * sizeof(int));
    long sp = 0;
#define ZERO_AT(py, px) ((py) == 0 || (px) == 0 || (py) == PH - 1 || (px) == PW - 1 || \
                         src[(size_t)((py) - 1) * W + ((px) - 1)] == 0)
    reach[0] = 1; stack[sp++] = 0;
    while (sp) {
        int v = stack[--sp];
        int py = v / PW, px = v % PW;
        const int dy[4] = {-1, 1, 0, 0}, dx[4] = {0, 0, -1, 1};
        for (int d = 0; d < 4; ++d) {
            int qy = py + dy[d], qx = px + dx[d];
            if (qy < 0 || qx < 0 || qy >= PH || qx >= PW) continue;
            size_t q = (size_t)qy * PW + qx;
            if (reach[q] || !ZERO_AT(qy, qx)) continue;
            reach[q] = 1; stack[sp++] = (int)q;
        }
    }
#undef ZERO_AT
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            unsigned char s = src[(size_t)y * W + x];
            int hole = (s == 0) && !reach[(size_t)(y + 1) * PW + (x + 1)];
            dst[(size_t)y * W + x] = (unsigned char)(s | (hole ? 255 : 0));
        }
    free(reach); free(stack);
}

/* Erosion then dilation over the same list of (dy,dx) offsets; outside the
 * image the erosion sees 255 and the dilation sees 0 (OpenCV's default
 * morphology border), and neither reflects the structuring element. */
static void open_offsets(const unsigned char *src, int H, int W, const int *dy,
                         const int *dx, int n, unsigned char *dst)
{
    unsigned char *er = (unsigned char *)malloc((size_t)H * W);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            unsigned char m = 255;
            for (int k = 0; k < n; ++k) {
                int yy = y + dy[k], xx = x + dx[k];
                if (yy < 0 || xx < 0 || yy >= H || xx >= W) continue;
                unsigned char v = src[(size_t)yy * W + xx];
                if (v < m) m = v;
            }
            er[(size_t)y * W + x] = m;
        }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            unsigned char m = 0;
            for (int k = 0; k < n; ++k) {
                int yy = y + dy[k], xx = x + dx[k];
                if (yy < 0 || xx < 0 || yy >= H || xx >= W) continue;
                unsigned char v = er[(size_t)yy * W + xx];
                if (v > m) m = v;
            }
            dst[(size_t)y * W + x] = m;
        }
    free(er);
}

void or_open_rect(const unsigned char *src, int H, int W, int kw, int kh,
                  unsigned char *dst)
{
    int n = kw * kh, ax = kw / 2, ay = kh / 2, k = 0;
    int *dy = (int *)malloc(n * sizeof(int)), *dx = (int *)malloc(n * sizeof(int));
    for (int j = 0; j < kh; ++j)
        for (int i = 0; i < kw; ++i) { dy[k] = j - ay; dx[k] = i - ax; ++k; }
    open_offsets(src, H, W, dy, dx, n, dst);
    free(dy); free(dx);
}

void or_open_eye(const unsigned char *src, int H, int W, int ksz,
                 unsigned char *dst)
{
    int a = ksz / 2;
    int *dy = (int *)malloc(ksz * sizeof(int)), *dx = (int *)malloc(ksz * sizeof(int));
    for (int t = 0; t < ksz; ++t) { dy[t] = t - a; dx[t] = t - a; }
    open_offsets(src, H, W, dy, dx, ksz, dst);
    free(dy); free(dx);
}

/* ------------------------------------------------------------------------ */
/* Border following (Suzuki & Abe 1985), OpenCV's RETR_CCOMP output order    */
/* ------------------------------------------------------------------------ */

/* Neighbour directions: 0 = +x, then counter-clockwise on screen (y down). */
static const int DX8[8] = {1, 1, 0, -1, -1, -1, 0, 1};
static const int DY8[8] = {0, -1, -1, -1, 0, 1, 1, 1};

typedef struct { int nbd, hole, parent; long first, count; } border_t;

int or_find_contours(const unsigned char *img, int H, int W, int **pts_out,
                     int **lens_out, long *total_out)
{
    int PW = W + 2, PH = H + 2;
    int *f = (int *)calloc((size_t)PW * PH, sizeof(int));
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            f[(size_t)(y + 1) * PW + x + 1] = img[(size_t)y * W + x] != 0;

    long cap_b = 64, nb = 0, cap_p = 1024, np = 0;
    border_t *bs = (border_t *)malloc(cap_b * sizeof(border_t));
    int *pts = (int *)malloc(cap_p * 2 * sizeof(int));
    /* hole flag and parent per label; label 1 is the frame (a hole) */
    long cap_l = 64;
    int *lhole = (int *)malloc(cap_l * sizeof(int));
    int *lpar = (int *)malloc(cap_l * sizeof(int));
    lhole[1] = 1; lpar[1] = 0;
    int nbd = 1;

    for (int y = 1; y <= H; ++y) {
        int lnbd = 1;
        for (int x = 1; x <= W; ++x) {
            size_t at = (size_t)y * PW + x;
            int v = f[at];
            if (v == 0) continue;
            int start = 0, hole = 0;
            if (v == 1 && f[at - 1] == 0) { start = 1; hole = 0; }
            else if (v >= 1 && f[at + 1] == 0) {
                start = 1; hole = 1;
                if (v > 1) lnbd = v;
            }
            if (start) {
                ++nbd;
                if (nbd >= cap_l) {
                    cap_l *= 2;
                    lhole = (int *)realloc(lhole, cap_l * sizeof(int));
                    lpar = (int *)realloc(lpar, cap_l * sizeof(int));
                }
                lhole[nbd] = hole;
                lpar[nbd] = (lhole[lnbd] == hole) ? lpar[lnbd] : lnbd;
                if (nb == cap_b) { cap_b *= 2; bs = (border_t *)realloc(bs, cap_b * sizeof(border_t)); }
                border_t *b = &bs[nb++];
                b->nbd = nbd; b->hole = hole; b->parent = lpar[nbd]; b->first = np;

                /* 3.1: clockwise from the zero neighbour that started us */
                int s = hole ? 0 : 4, s0 = s, found = 0;
                do {
                    s = (s - 1) & 7;
                    if (f[(size_t)(y + DY8[s]) * PW + x + DX8[s]] != 0) { found = 1; break; }
                } while (s != s0);
                if (!found) {
                    f[at] = -nbd;
                    if (np == cap_p) { cap_p *= 2; pts = (int *)realloc(pts, cap_p * 2 * sizeof(int)); }
                    pts[2 * np] = x - 1; pts[2 * np + 1] = y - 1; ++np;
                } else {
                    int ly = y + DY8[s], lx = x + DX8[s];   /* last border pixel */
                    int cy = y, cx = x;
                    for (;;) {
                        /* 3.3: counter-clockwise from the previous pixel */
                        int k = s, east_zero = 0, ny, nx;
                        for (;;) {
                            ++k;
                            int d = k & 7;
                            ny = cy + DY8[d]; nx = cx + DX8[d];
                            if (f[(size_t)ny * PW + nx] != 0) break;
                            if (d == 0) east_zero = 1;
                        }
                        s = k & 7;
                        size_t c = (size_t)cy * PW + cx;
                        if (east_zero) f[c] = -nbd;
                        else if (f[c] == 1) f[c] = nbd;
                        if (np == cap_p) { cap_p *= 2; pts = (int *)realloc(pts, cap_p * 2 * sizeof(int)); }
                        pts[2 * np] = cx - 1; pts[2 * np + 1] = cy - 1; ++np;
                        if (ny == y && nx == x && cy == ly && cx == lx) break;
                        cy = ny; cx = nx;
                        s = (s + 4) & 7;
                    }
                }
                b->count = np - b->first;
            }
            if (f[at] != 1) lnbd = abs(f[at]);
        }
    }

    /* Output order: outer borders newest first; after each, its holes
     * newest first. */
    int *lens = (int *)malloc((nb ? nb : 1) * sizeof(int));
    int *opts = (int *)malloc((np ? np : 1) * 2 * sizeof(int));
    long *bynbd = (long *)malloc((size_t)(nbd + 1) * sizeof(long));
    long *head = (long *)malloc((nb ? nb : 1) * sizeof(long));  /* newest hole of an outer */
    long *next = (long *)malloc((nb ? nb : 1) * sizeof(long));  /* next older sibling hole */
    for (long i = 0; i < nb; ++i) { bynbd[bs[i].nbd] = i; head[i] = -1; next[i] = -1; }
    for (long i = 0; i < nb; ++i)
        if (bs[i].hole && bs[i].parent >= 2) {   /* a hole's parent is an outer border */
            long par = bynbd[bs[i].parent];
            next[i] = head[par]; head[par] = i;
        }
    int nout = 0; long op = 0;
    for (long i = nb - 1; i >= 0; --i) {
        if (bs[i].hole) continue;
        lens[nout++] = (int)bs[i].count;
        memcpy(opts + 2 * op, pts + 2 * bs[i].first, bs[i].count * 2 * sizeof(int));
        op += bs[i].count;
        for (long j = head[i]; j >= 0; j = next[j]) {
            lens[nout++] = (int)bs[j].count;
            memcpy(opts + 2 * op, pts + 2 * bs[j].first, bs[j].count * 2 * sizeof(int));
            op += bs[j].count;
        }
    }
    free(head); free(next);
    free(bynbd); free(bs); free(pts); free(lhole); free(lpar); free(f);
    *pts_out = opts; *lens_out = lens; *total_out = op;
    return nout;
}

/* ------------------------------------------------------------------------ */
/* getSdf (morohutils.cu:182-291)                                            */
/* ------------------------------------------------------------------------ */

int or_getsdf(int M, int N, const int *rowptr, const int *col,
              const or_params *p, int *mF, int *Wout, int **corners,
              unsigned char *stages)
{
    int H = p->thumb_height, W = 0, pM = 0, pN = 0;
    *mF = 0; *Wout = 0; *corners = NULL;
    int ok = or_thumb_dims(M, N, H, &W, &pM, &pN);
    if (ok <= 0) return ok;   /* 0: too small, no shapes; -1: W == 0 */
    size_t n = (size_t)H * W;
    unsigned char *img = (unsigned char *)malloc(n), *rev = (unsigned char *)malloc(n);
    unsigned char *fil = (unsigned char *)malloc(n), *o1 = (unsigned char *)malloc(n);
    unsigned char *o2 = (unsigned char *)malloc(n), *del = (unsigned char *)malloc(n);
    unsigned char *eo = (unsigned char *)malloc(n);
    or_raster(M, rowptr, col, H, W, pM, pN, img);
    for (size_t i = 0; i < n; ++i) rev[i] = (unsigned char)(255 - img[i]);
    or_imfill(rev, H, W, fil);
    or_open_rect(fil, H, W, p->open_len, 1, o1);
    or_open_rect(o1, H, W, 1, p->open_len, o2);
    for (size_t i = 0; i < n; ++i) del[i] = rev[i] > o2[i] ? (unsigned char)(rev[i] - o2[i]) : 0;
    or_open_eye(del, H, W, p->eye_size, eo);
    if (stages) {
        memcpy(stages + 0 * n, rev, n);
        memcpy(stages + 1 * n, fil, n);
        memcpy(stages + 2 * n, o2, n);
        memcpy(stages + 3 * n, del, n);
        memcpy(stages + 4 * n, eo, n);
    }
    int *pts, *lens; long tot;
    int nc = or_find_contours(eo, H, W, &pts, &lens, &tot);
    int *cs = (int *)malloc((nc ? nc : 1) * 4 * sizeof(int));
    int kept = 0; long off = 0;
    for (int i = 0; i < nc; ++i) {
        if (lens[i] >= p->min_contour) {
            cs[4 * kept + 0] = pts[2 * off];
            cs[4 * kept + 1] = pts[2 * off + 1];
            cs[4 * kept + 2] = pts[2 * (off + lens[i] / 2)];
            cs[4 * kept + 3] = pts[2 * (off + lens[i] / 2) + 1];
            ++kept;
        }
        off += lens[i];
    }
    free(pts); free(lens);
    free(img); free(rev); free(fil); free(o1); free(o2); free(del); free(eo);
    *mF = H; *Wout = W; *corners = cs;
    return kept;
}

/* ------------------------------------------------------------------------ */
/* Shape geometry (TaiChi.cu:280-311, 689-699, 881-916)                      */
/* ------------------------------------------------------------------------ */

void or_cal_shape_size(int M, int N, int mF, int x1, int y1, int a1, int b1,
                       int *x, int *y, int *a, int *b, float *gain)
{
    float g;
    if (M > mF) {
        g = (float)M / (float)mF;
        *x = (int)((float)x1 * g); *y = (int)((float)y1 * g);
        *a = (int)((float)a1 * g); *b = (int)((float)b1 * g);
    } else if (M < mF) {
        g = (float)mF / (float)M;
        *x = (int)((float)x1 / g); *y = (int)((float)y1 / g);
        *a = (int)((float)a1 / g); *b = (int)((float)b1 / g);
    } else {
        g = 1.0f; *x = x1; *y = y1; *a = a1; *b = b1;
    }
    if (*x < 0) *x = 0;
    if (*x > M - 1) *x = M - 1;
    if (*y < 0) *y = 0;
    if (*y > N - 1) *y = N - 1;
    if (*y + *a > N) *a = N - *y;
    if (*x + *b > M) *b = M - *x;
    if (*a > *b) *a = *b; else *b = *a;
    *gain = g;
}

int or_band_width(int s)
{
    double w;
    if (s >= 10000000) w = s * 0.000001;
    else if (s >= 1000000) w = s * 0.00001;
    else if (s >= 100000) w = s * 0.001;
    else if (s >= 10000) w = s * 0.01;
    else w = s * 0.1;
    return (int)w;
}

void or_cal_start_end(int M_sub, int N_sub, int width, int off, int n,
                      int *start, int *end)
{
    int ao = abs(off);
    if (M_sub >= N_sub) {
        if (n >= width - 1) { *start = 0; *end = N_sub - off; }
        else if (ao > M_sub - N_sub) { *start = ao; *end = M_sub; }
        else { *start = ao; *end = N_sub + ao; }
    } else {
        if (n <= width - 1) { *start = ao; *end = M_sub; }
        else if (ao > N_sub - M_sub) { *start = 0; *end = N_sub - ao; }
        else { *start = 0; *end = M_sub; }
    }
}

/* ------------------------------------------------------------------------ */
/* Partition (TaiChi.cu:313-638, 677-879)                                    */
/* ------------------------------------------------------------------------ */

static int unclaimed(float v)
{
    float d = v - FLT_MAX;          /* TaiChi.cu:730: fabs(csrVal[j]-FLT_MAX)>ZERO */
    return fabs((double)d) > 1e-8;
}

typedef struct {
    int xStart, yStart, M_sub, N_sub, width, neg, nnz;
    int *offs, *nzero, **holes;
} dshape_t;

static void dia_shape(int M, const int *rowptr, const int *col, float *val,
                      int hx, int hy, int ha, int hb, double thr, dshape_t *S)
{
    memset(S, 0, sizeof *S);
    S->M_sub = hb; S->N_sub = ha; S->xStart = hx; S->yStart = hy;
    int small = hb < ha ? hb : ha;
    int w = or_band_width(small);
    S->width = w;
    int nd = 2 * w - 1;
    if (nd <= 0) return;
    int dof = hy - hx;
    long *cnt = (long *)calloc(nd, sizeof(long));
    /* pass 1: per-diagonal counts of unclaimed in-band entries */
#define IN_BAND(r, c, j) ((r) >= hx && (r) < hx + hb && (c) >= hy && (c) < hy + ha && \
                          (c) >= (r) + dof - w + 1 && (c) <= (r) + dof + w - 1 && unclaimed(val[j]))
    for (int r = 0; r < M; ++r)
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) {
            int c = col[j];
            if (IN_BAND(r, c, j)) cnt[c - r - dof + w - 1]++;
        }
    long *fillp = (long *)calloc(nd, sizeof(long));
    int **rows = (int **)calloc(nd, sizeof(int *));
    for (int d = 0; d < nd; ++d) rows[d] = (int *)malloc((cnt[d] ? cnt[d] : 1) * sizeof(int));
    for (int r = 0; r < M; ++r)
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) {
            int c = col[j];
            if (IN_BAND(r, c, j)) { int d = c - r - dof + w - 1; rows[d][fillp[d]++] = r - hx; }
        }
    /* dense diagonals */
    int *offs = (int *)malloc(nd * sizeof(int)), *st = (int *)malloc(nd * sizeof(int));
    int *en = (int *)malloc(nd * sizeof(int)), *idx = (int *)malloc(nd * sizeof(int));
    int neg = 0;
    for (int d = 0; d < nd; ++d) {
        int off = d - w + 1, s, e;
        or_cal_start_end(hb, ha, w, off, d, &s, &e);
        float dens = (float)cnt[d] / (float)(e - s);
        if ((double)dens >= thr) { offs[neg] = off; st[neg] = s; en[neg] = e; idx[neg] = d; ++neg; }
    }
    S->neg = neg;
    if (neg > 0) {
        S->offs = (int *)malloc(neg * sizeof(int));
        S->nzero = (int *)malloc(neg * sizeof(int));
        S->holes = (int **)calloc(neg, sizeof(int *));
        long tot = 0;
        for (int k = 0; k < neg; ++k) {
            int d = idx[k];
            S->offs[k] = offs[k];
            tot += cnt[d];
            int nz = en[k] - st[k] - (int)cnt[d];
            S->nzero[k] = nz;
            S->holes[k] = (int *)malloc((nz > 0 ? nz : 1) * sizeof(int));
            /* TaiChi.cu:809-827: walk the rows of the diagonal against the
             * list of rows that hold an entry; keep the first nz holes. */
            long p = 0; int got = 0;
            for (int r = st[k]; r < en[k]; ++r) {
                int hole;
                if (p >= cnt[d]) hole = 1;
                else if (r < rows[d][p]) hole = 1;
                else { ++p; hole = 0; }
                if (hole && got < nz) S->holes[k][got++] = r;
            }
        }
        S->nnz = (int)tot;
        /* claim the entries on dense diagonals (TaiChi.cu:848-874) */
        for (int r = 0; r < M; ++r)
            for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) {
                int c = col[j];
                if (IN_BAND(r, c, j)) {
                    int o = (c - hy) - (r - hx);
                    for (int k = 0; k < neg; ++k)
                        if (o == offs[k]) val[j] = FLT_MAX;
                }
            }
    }
#undef IN_BAND
    for (int d = 0; d < nd; ++d) free(rows[d]);
    free(rows); free(cnt); free(fillp); free(offs); free(st); free(en); free(idx);
}

static void dshape_free(dshape_t *S)
{
    for (int k = 0; k < S->neg; ++k) free(S->holes ? S->holes[k] : NULL);
    free(S->holes); free(S->offs); free(S->nzero);
}

int or_partition(int M, int N, int nnz, int *rowptr, int *col, float *val,
                 const or_params *p, const int *corners_in, int nshapes_in,
                 int mF_in, or_format *out)
{
    memset(out, 0, sizeof *out);
    int mF = 0, ns = 0, W = 0;
    int *corners = NULL;
    if (corners_in) { mF = mF_in; ns = nshapes_in; corners = (int *)corners_in; }
    else {
        ns = or_getsdf(M, N, rowptr, col, p, &mF, &W, &corners, NULL);
        if (ns < 0) return ns;
    }
    dshape_t *S = (dshape_t *)calloc(ns ? ns : 1, sizeof(dshape_t));
    int dia_shapes = 0, num_negs = 0;
    long dense = 0;
    for (int i = 0; i < ns; ++i) {
        int x1 = corners[4 * i], y1 = corners[4 * i + 1];
        int a1 = corners[4 * i + 2] - x1, b1 = corners[4 * i + 3] - y1;
        int x, y, a, b; float g;
        or_cal_shape_size(M, N, mF, x1, y1, a1, b1, &x, &y, &a, &b, &g);
        if (a < p->min_shape_side || b < p->min_shape_side) continue;
        dia_shape(M, rowptr, col, val, x, y, a, b, p->density, &S[i]);
        if (S[i].nnz > 0) { dia_shapes++; num_negs += S[i].neg; dense += S[i].nnz; }
    }
    if (!corners_in) free(corners);

    out->dia_shapes = dia_shapes; out->num_negs = num_negs;
    out->dense_nnz = (int)dense;
    out->sparse_nnz = nnz - (int)dense;
    long zeros = 0;
    if (dia_shapes > 0) {
        out->xStart = (int *)malloc(dia_shapes * sizeof(int));
        out->yStart = (int *)malloc(dia_shapes * sizeof(int));
        out->xStop = (int *)malloc(dia_shapes * sizeof(int));
        out->nDiasPtr = (int *)malloc((dia_shapes + 1) * sizeof(int));
        out->neg_offsets = (int *)malloc(num_negs * sizeof(int));
        out->nDiasPtr[0] = 0;
        int d = 0, t = 0;
        for (int i = 0; i < ns; ++i) {
            if (S[i].nnz <= 0) continue;
            out->xStart[d] = S[i].xStart; out->yStart[d] = S[i].yStart;
            out->xStop[d] = S[i].xStart + S[i].M_sub;
            out->nDiasPtr[d + 1] = out->nDiasPtr[d] + S[i].neg;
            memcpy(out->neg_offsets + t, S[i].offs, S[i].neg * sizeof(int));
            t += S[i].neg; ++d;
            for (int k = 0; k < S[i].neg; ++k) zeros += S[i].nzero[k];
        }
        int mn = out->xStart[0], mx = out->xStop[0];
        for (int k = 1; k < dia_shapes; ++k) {
            if (out->xStart[k] < mn) mn = out->xStart[k];
            if (out->xStop[k] > mx) mx = out->xStop[k];
        }
        out->row_start = mn; out->row_stop = mx;
    }
    out->zero_elements = (int)zeros;

    if (dense == 0) {
        /* the reference aliases the caller's CSR here; the oracle copies it */
        out->csr_aliases_input = 1;
        out->csrRow = (int *)malloc(((size_t)M + 1) * sizeof(int));
        memcpy(out->csrRow, rowptr, ((size_t)M + 1) * sizeof(int));
        out->csrCol = (int *)malloc((rowptr[M] ? rowptr[M] : 1) * sizeof(int));
        memcpy(out->csrCol, col, (size_t)rowptr[M] * sizeof(int));
    } else {
        /* per row: holes (shape order, diagonal order, ascending row), then
         * the unclaimed entries in CSR order (TaiChi.cu:495-612) */
        long *zc = (long *)calloc((size_t)M + 1, sizeof(long));
        for (int i = 0; i < ns; ++i) {
            if (S[i].nnz <= 0) continue;
            for (int k = 0; k < S[i].neg; ++k)
                for (int h = 0; h < S[i].nzero[k]; ++h) zc[S[i].xStart + S[i].holes[k][h]]++;
        }
        long *rp = (long *)malloc(((size_t)M + 1) * sizeof(long));
        rp[0] = 0;
        for (int r = 0; r < M; ++r) {
            long sp = 0;
            for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) sp += unclaimed(val[j]);
            rp[r + 1] = rp[r] + zc[r] + sp;
        }
        out->csrRow = (int *)malloc(((size_t)M + 1) * sizeof(int));
        for (int r = 0; r <= M; ++r) out->csrRow[r] = (int)rp[r];
        out->csrCol = (int *)malloc((rp[M] ? rp[M] : 1) * sizeof(int));
        long *fill = (long *)calloc((size_t)M, sizeof(long));
        for (int i = 0; i < ns; ++i) {
            if (S[i].nnz <= 0) continue;
            for (int k = 0; k < S[i].neg; ++k)
                for (int h = 0; h < S[i].nzero[k]; ++h) {
                    int rs = S[i].holes[k][h];
                    int r = S[i].xStart + rs;
                    int c = S[i].yStart + rs + S[i].offs[k];
                    out->csrCol[rp[r] + fill[r]++] = c << 1;
                }
        }
        for (int r = 0; r < M; ++r)
            for (int j = rowptr[r]; j < rowptr[r + 1]; ++j)
                if (unclaimed(val[j])) out->csrCol[rp[r] + fill[r]++] = (col[j] << 1) + 1;
        free(zc); free(rp); free(fill);
    }
    for (int i = 0; i < ns; ++i) dshape_free(&S[i]);
    free(S);
    return 0;
}

void or_format_free(or_format *f)
{
    free(f->xStart); free(f->yStart); free(f->xStop); free(f->nDiasPtr);
    free(f->neg_offsets); free(f->csrRow); free(f->csrCol);
    memset(f, 0, sizeof *f);
}

/* ------------------------------------------------------------------------ */
/* SpMV references                                                           */
/* ------------------------------------------------------------------------ */

void or_spmv_csr_f64(int M, const int *rowptr, const int *col,
                     const double *x, double *y)
{
    for (int r = 0; r < M; ++r) {
        double s = 0.0;
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) s += x[col[j]];
        y[r] = s;
    }
}

void or_spmv_csr_f32_serial(int M, const int *rowptr, const int *col,
                            const float *x, float *y)
{
    for (int i = 0; i < M; ++i) {          /* main.cu:61-69 */
        y[i] = 0.0f;
        for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) y[i] += x[col[j]];
    }
}

void or_spmv_csr_f32_omp(int M, const int *rowptr, const int *col,
                         const float *x, float *y, int threads)
{
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static, 4096)
#endif
    for (int i = 0; i < M; ++i) {
        float s = 0.0f;
        for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) s += x[col[j]];
        y[i] = s;
    }
    (void)threads;
}

void or_spmm_csr_f64(int M, const int *rowptr, const int *col, int k,
                     const double *X, double *Y)
{
    for (int r = 0; r < M; ++r) {
        double *yr = Y + (size_t)r * k;
        for (int t = 0; t < k; ++t) yr[t] = 0.0;
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) {
            const double *xr = X + (size_t)col[j] * k;
            for (int t = 0; t < k; ++t) yr[t] += xr[t];
        }
    }
}

void or_spmv_format_f64(const or_format *f, int M, int N, const double *x,
                        double *y)
{
    (void)N;
    for (int r = 0; r < M; ++r) {
        double s = 0.0;
        if (f->dense_nnz == 0) {
            for (int j = f->csrRow[r]; j < f->csrRow[r + 1]; ++j) s += x[f->csrCol[j]];
        } else {
            for (int j = f->csrRow[r]; j < f->csrRow[r + 1]; ++j) {
                int v = f->csrCol[j];
                s += (v & 1) ? x[v >> 1] : -x[v >> 1];
            }
            if (r >= f->row_start && r < f->row_stop)
                for (int d = 0; d < f->dia_shapes; ++d) {
                    int xs = f->xStart[d], xe = f->xStop[d], ys = f->yStart[d];
                    if (r < xs || r >= xe) continue;
                    for (int n = f->nDiasPtr[d]; n < f->nDiasPtr[d + 1]; ++n) {
                        int c = r - xs + ys + f->neg_offsets[n];
                        if (c >= ys && c < ys + (xe - xs)) s += x[c];
                    }
                }
        }
        y[r] = s;
    }
}
