/*
 * taichi_oracle.h -- CPU restatement of TaiChi's binary-SpMV path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in taichi_b200/: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.  Nothing in the product links it.
 *
 * Every function restates one piece of the reference (double-flower/TaiChi)
 * and cites the file:line it follows.  The morphology and contour steps
 * restate the OpenCV calls made by morohutils.cu (floodFill, morphologyEx,
 * findContours with RETR_CCOMP / CHAIN_APPROX_NONE) from their published
 * definitions (Suzuki & Abe 1985 border following); they are pinned against
 * cv2 4.13.0 by tests/golden/make_golden.py.
 */
#ifndef TAICHI_ORACLE_H
#define TAICHI_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same fields, same meaning as TaiChi_new (TaiChi.h:45-60). */
typedef struct or_format {
    int dia_shapes, num_negs, dense_nnz, zero_elements, sparse_nnz;
    int row_start, row_stop;
    int *xStart, *yStart, *xStop, *nDiasPtr, *neg_offsets;
    int *csrRow, *csrCol;   /* csrRow has M+1 entries; csrCol csrRow[M]     */
    int csr_aliases_input;  /* 1 when dense_nnz == 0 (TaiChi.cu:575-578)    */
} or_format;

/* Tunables of the partition.  or_params_default() returns the reference's
 * hard-coded values (morohutils.cu:140,191,239,242,250; TaiChi.cu:379,757). */
typedef struct or_params {
    int thumb_height;       /* 512  */
    int open_len;           /* 30   */
    int eye_size;           /* 5    */
    int min_contour;        /* 80   */
    int min_shape_side;     /* 1000 */
    double density;         /* 0.6  */
} or_params;

void or_params_default(or_params *p);

/* readMtx (TaiChi.cu:120-278) with the banner / size parsing of mmio.cpp:96-218.
 * Returns 0, -1 (open), -2 (banner), -3 (complex), -4 (size line). */
int or_read_mtx(const char *path, int *m, int *n, unsigned long *nnz,
                int **rowptr, int **col, float **val);
void or_free(void *p);

/* Thumbnail geometry of getSdf (morohutils.cu:191-200).  Returns 0 when the
 * matrix is too small for a thumbnail (M <= height), 1 otherwise. */
int or_thumb_dims(int M, int N, int height, int *W, int *pM, int *pN);

/* getSdf_GPU1 (morohutils.cu:153-180): img is H x W, 255 everywhere except 0
 * at pixels hit by a non-zero. */
void or_raster(int M, const int *rowptr, const int *col, int H, int W, int pM,
               int pN, unsigned char *img);

/* imfill (morohutils.cu:73-83): dst = src | ~(border flood of src's zeros). */
void or_imfill(const unsigned char *src, int H, int W, unsigned char *dst);

/* morphologyEx(MORPH_OPEN) with a kw x kh rectangle (anchor = centre). */
void or_open_rect(const unsigned char *src, int H, int W, int kw, int kh,
                  unsigned char *dst);
/* morphologyEx(MORPH_OPEN) with Mat::eye(k, k) (anchor = centre). */
void or_open_eye(const unsigned char *src, int H, int W, int k,
                 unsigned char *dst);

/* findContours(RETR_CCOMP, CHAIN_APPROX_NONE) in OpenCV's output order.
 * Points are (x=col, y=row) pairs.  Returns the number of contours; *pts
 * (2 ints per point) and *lens are malloc'd. */
int or_find_contours(const unsigned char *img, int H, int W, int **pts,
                     int **lens, long *total_pts);

/* The whole of getSdf (morohutils.cu:182-291).  Writes 4 ints per kept
 * contour into *corners: contour[0].x, contour[0].y, contour[n/2].x,
 * contour[n/2].y.  If stages != NULL it receives the 5 intermediate images
 * (raster, filled, open-open, subtracted, eye-opened) of H*W bytes each. */
int or_getsdf(int M, int N, const int *rowptr, const int *col,
              const or_params *p, int *mF, int *W, int **corners,
              unsigned char *stages);

/* cal_shape_size (TaiChi.cu:280-311) */
void or_cal_shape_size(int M, int N, int mF, int x1, int y1, int a1, int b1,
                       int *x, int *y, int *a, int *b, float *gain);
/* cal_start_end (TaiChi.cu:881-916) */
void or_cal_start_end(int M_sub, int N_sub, int width, int off, int n,
                      int *start, int *end);
/* width rule of partition_dia_shape (TaiChi.cu:689-699) */
int or_band_width(int smaller_dim);

/* partition_shapes (TaiChi.cu:313-638) run sequentially, with getSdf above.
 * Mutates val (FLT_MAX marks) exactly like the reference.  When
 * corners_in != NULL those shape corners (4 ints each) replace getSdf's
 * output and mF_in is used as the thumbnail height. */
int or_partition(int M, int N, int nnz, int *rowptr, int *col, float *val,
                 const or_params *p, const int *corners_in, int nshapes_in,
                 int mF_in, or_format *out);
void or_format_free(or_format *f);

/* y = A x over a plain CSR pattern, in double. */
void or_spmv_csr_f64(int M, const int *rowptr, const int *col,
                     const double *x, double *y);
/* main.cu:61-69: float accumulation in CSR order, one thread. */
void or_spmv_csr_f32_serial(int M, const int *rowptr, const int *col,
                            const float *x, float *y);
/* The same loop, rows split over `threads` OpenMP threads (same per-row
 * order, so bit-identical to the serial loop). */
void or_spmv_csr_f32_omp(int M, const int *rowptr, const int *col,
                         const float *x, float *y, int threads);
/* SpMM X (N x k, row-major) -> Y (M x k) in double. */
void or_spmm_csr_f64(int M, const int *rowptr, const int *col, int k,
                     const double *X, double *Y);
/* Applies a TaiChi format (diagonals + signed CSR) in double: the value the
 * reference kernels compute (TaiChi.cu:965-1265) in exact arithmetic. */
void or_spmv_format_f64(const or_format *f, int M, int N, const double *x,
                        double *y);

#ifdef __cplusplus
}
#endif
#endif
