/*
 * TaiChi.h -- drop-in declarations of the reference's entry points, served
 * by libtaichi_b200.so.
 *
 * Replaces the reference's TaiChi.h (TaiChi.h:1-107).  The three structs keep
 * the reference's field order and types, so their byte layout is identical and
 * a program compiled against either header links against this library.  The
 * functions keep C++ linkage and the reference's signatures; each one notes the
 * reference definition it replaces.
 */
#ifndef TAICHI_B200_COMPAT_H
#define TAICHI_B200_COMPAT_H

#include <cuda_runtime.h>

#if defined(__GNUC__)
#define TAICHI_API __attribute__((visibility("default")))
#else
#define TAICHI_API
#endif

/* Per-shape record of the partitioner (TaiChi.h:5-18). */
typedef struct shape {
    int id;
    char category[1024];
    int x1, y1, a1, b1, area1;   /* corner and extents in the thumbnail       */
    int x, y, a, b;              /* corner and extents in the matrix          */
    int width;
} shape;

/* Per-shape diagonal extraction result (TaiChi.h:20-43). */
typedef struct TaiChi {
    char shape;
    int M_sub, N_sub, xStart, yStart, width;
    int neg, maxNumZero;
    int *neg_offsets, *numZeroNeg;
    int **rowZeroNeg;
    int *start, *end, *cStart;
    int nnz;
    int *csrRow, *csrCol;
} TaiChi;

/* The hybrid format handed to the multiply (TaiChi.h:45-60). */
typedef struct TaiChi_new {
    int dia_shapes, num_negs, dense_nnz, zero_elements, sparse_nnz;
    int row_start, row_stop;
    int *xStart, *yStart, *xStop, *nDiasPtr, *neg_offsets;
    int *csrRow, *csrCol;
} TaiChi_new;

#ifndef VALUE_TYPE
#define VALUE_TYPE float
#endif
#ifndef NUM_RUN
#define NUM_RUN 500        /* timed launches inside taichi_SpMV              */
#endif
#ifndef NUM_TRANSFER
#define NUM_TRANSFER 50    /* timed format uploads inside taichi_SpMV        */
#endif
#define ZERO 1e-8

/* TaiChi.cu:120 -- Matrix Market file -> malloc'd host CSR. */
TAICHI_API int readMtx(char *filename, int &m, int &n, unsigned long &nnzA,
            int *&csrRowPtrA, int *&csrColIdxA, float *&csrValA);

/* TaiChi.cu:313 -- GPU partition of a host CSR into the hybrid format.
 * Marks the claimed entries of csrVal with FLT_MAX, as the reference does. */
TAICHI_API void partition_shapes(char *sdf_name, int M, int N, int nnz,
                      int *&csRow, int *&csrCol, float *&csrVal, TaiChi_new *neg_format);

/* TaiChi.cu:280 -- thumbnail box -> matrix box. */
TAICHI_API void cal_shape_size(int M, int N, int mF, int x1, int y1, int a1, int b1,
                    int &x, int &y, int &a, int &b, float &gain);

/* TaiChi.cu:677 -- dense-diagonal extraction of one shape (host arrays). */
TAICHI_API void partition_dia_shape(int M, int N, int nnz, int *&csRow, int *&csrCol, float *&csrVal,
                         float gain, shape &hi, TaiChi &neg_format_i);

/* TaiChi.cu:1331 -- multiply with host x / y (uploads, times, downloads). */
TAICHI_API void taichi_SpMV(int M, int N, TaiChi_new *neg_format, float *xHostPtr, float *yHostPtr);

/* TaiChi.cu:918 */
TAICHI_API void queryDevice();
/* TaiChi.cu:947, 956 */
TAICHI_API int max(int *a, int len);
TAICHI_API int min(int *a, int len);
/* TaiChi.cu:881 */
TAICHI_API void cal_start_end(int M_sub, int N_sub, int width, int dia_offsets_temp, int n,
                   int &start_temp, int &end_temp);
/* TaiChi.cu:77, 640 */
TAICHI_API void free_taichi_new(TaiChi_new *taichi_new);
TAICHI_API void free_taichi(int num_shapes, TaiChi *taichi);

#endif
