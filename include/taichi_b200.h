/*
 * taichi_b200.h -- C ABI of the B200-native TaiChi binary-SpMV library
 * (libtaichi_b200.so).  Plain pointers, sizes and status codes only.
 *
 * The library also exports the reference's own C++ entry points with their
 * original signatures (readMtx, partition_shapes, taichi_SpMV,
 * free_taichi_new, ... -- see TaiChi.h in this directory), so a program
 * written against the reference links against this library unchanged.
 *
 * Streams are passed as `void *` (a cudaStream_t; NULL = legacy default
 * stream).  Device pointers are plain CUDA device addresses of the current
 * device.  Every call returns a tc_status; tc_last_error() describes the last
 * failure on the calling thread.
 */
#ifndef TAICHI_B200_H
#define TAICHI_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TC_API __attribute__((visibility("default")))
#else
#define TC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tc_status {
    TC_OK = 0,
    TC_ERR_INVALID = 1,     /* bad argument                                  */
    TC_ERR_CUDA = 2,        /* a CUDA runtime call failed                    */
    TC_ERR_ALLOC = 3,       /* device or host allocation failed              */
    TC_ERR_IO = 4,          /* file could not be opened / parsed             */
    TC_ERR_FORMAT = 5,      /* inconsistent sparse format                    */
    TC_ERR_CAPACITY = 6,    /* a fixed capacity (pool, scratch) is exceeded  */
    TC_ERR_TIMEOUT = 7,     /* a bounded device-side wait gave up            */
    TC_ERR_UNSUPPORTED = 8  /* size or mode outside what the library handles */
} tc_status;

/* Partition and multiply parameters.  tc_params_default() gives the
 * reference's hard-coded partition constants (morohutils.cu:140,191,239,242,
 * 250; TaiChi.cu:379,757) and the library's default tile shape. */
typedef struct tc_params {
    int thumb_height;     /* thumbnail rows (512)                              */
    int open_len;         /* length of the 30x1 / 1x30 opening lines (30)      */
    int eye_size;         /* size of the diagonal opening element (5)          */
    int min_contour;      /* contours with fewer points are dropped (80)       */
    int min_shape_side;   /* shapes with a smaller side are skipped (1000)     */
    double density;       /* a diagonal is dense if nnz/len >= density (0.6)   */
    int tile_rows;        /* max rows per multiply tile (1024)                 */
    int tile_nnz;         /* rows with more CSR entries get a CTA each (2048)  */
    int max_lanes;        /* most lanes the planner gives one row: 1..32 (32)  */
    int ctas_per_sm;      /* resident CTAs per SM of the multiply grid (4)     */
    int tile_mode;        /* 0: rows and entries split evenly over a CTA's
                             threads (merge path); 1: lanes per row chosen
                             from the tile's row lengths; 2: stream tiles
                             (entry-parallel gather into shared memory, then
                             row sums), one CTA per tile (2)                   */
    int flags;            /* TC_FLAG_*                                         */
    int rows_w;           /* rows kernel: words of a row loaded together, 4, 6
                             or 8 (0: the least that holds 90 % of the rows)   */
} tc_params;

#define TC_FLAG_NO_PARTITION 0x1  /* skip the morphology: plain CSR plan      */
#define TC_FLAG_KEEP_HOST    0x2  /* keep a host copy of the format (export)  */
#define TC_FLAG_NO_PDL       0x4  /* launch without programmatic dependent
                                     launch (the multiply then starts only
                                     when the previous kernel has finished)  */
#define TC_FLAG_ROWS_STRIDED 0x8  /* stream tiles (tile_mode 2) sum one row
                                     per thread, never 4 consecutive rows   */
#define TC_FLAG_NO_DIRECT    0x10 /* tile_mode 2: no direct tiles (4-row runs
                                     read straight from global memory) for
                                     rows averaging at most one entry       */
#define TC_FLAG_NO_WIDE      0x20 /* tile_mode 2: no wide direct tiles (a
                                     1024-thread CTA per 4096 rows) for a
                                     matrix whose rows all qualify          */
#define TC_FLAG_NO_WINDOW    0x40 /* tile_mode 2: never run the window kernel
                                     (x staged in shared memory per tile of
                                     rows), even for a banded matrix        */
#define TC_FLAG_WIDE_BOUNDS  0x100 /* wide plans of whole tiles: pass each
                                     tile's word range in the launch
                                     parameters and stage its words in
                                     shared memory (off by default: measured
                                     slower on R-MAT scale 20)              */
#define TC_FLAG_WIDE_FIXED   0x200 /* wide plans: tiles of 4096 rows
                                     instead of two equal tiles per SM     */
#define TC_FLAG_ROWS         0x400 /* plans of stream tiles only: run the
                                     rows kernel (one row per thread, words
                                     straight from global memory) whatever
                                     the rows' mean length                  */
#define TC_FLAG_NO_ROWS      0x800 /* plans of stream tiles only: never run
                                     the rows kernel                        */
#define TC_FLAG_NO_PREFETCH  0x2000 /* stream and rows kernels: no L2
                                     prefetch of the operands of the CTA a
                                     wave ahead; wide kernel: no L2 prefetch
                                     of a tile's CSR words                  */
#define TC_FLAG_NO_PARAM_STARTS 0x4000 /* wide plans: each tile's word
                                     range from its tile record, not from
                                     the launch parameters                  */
#define TC_FLAG_WINDOW       0x80 /* tile_mode 2: run the window kernel
                                     whenever the rows fit its tiles, even
                                     where the planner would not choose it   */
#define TC_FLAG_HOST_Y_MAPPED 0x8000 /* tc_spmv_host / tc_spmv_host_async:
                                     when h_y is page-locked host memory
                                     the GPU can address (cudaHostAlloc,
                                     cudaMallocHost, mapped registrations),
                                     the multiply stores y straight into it
                                     over the host link instead of into a
                                     device buffer that a copy then reads
                                     back; other h_y take the copy          */

TC_API void tc_params_default(tc_params *p);

TC_API const char *tc_last_error(void);
TC_API const char *tc_status_string(tc_status s);

/* ----------------------------------------------------------------------- */
/* Resident plans: a formatted matrix kept in device memory.                */
/* ----------------------------------------------------------------------- */
typedef struct tc_plan tc_plan;

/* Format view with the fields of the reference's TaiChi_new (TaiChi.h:45-60).
 * All arrays are host arrays.  csrCol entries carry the sign bit
 * ((col << 1) | add) when dia_shapes > 0 and are plain column indices when
 * dia_shapes == 0. */
typedef struct tc_format {
    int dia_shapes, num_negs, dense_nnz, zero_elements, sparse_nnz;
    int row_start, row_stop;
    const int *xStart, *yStart, *xStop, *nDiasPtr, *neg_offsets;
    const int *csrRow, *csrCol;
} tc_format;

/* Builds a plan from a binary CSR pattern (values are ignored except for the
 * reference's FLT_MAX "already claimed" marker).  rowptr/col/val are host
 * arrays unless on_device != 0.  The partition (thumbnail, morphology,
 * contours, dense-diagonal extraction) runs on the GPU.  Replaces
 * partition_shapes (TaiChi.cu:313-638) + the device upload of taichi_SpMV
 * (TaiChi.cu:1357-1385). */
TC_API tc_status tc_plan_create(int M, int N, int64_t nnz, const int *rowptr, const int *col,
                         const float *val, int on_device, const tc_params *params,
                         void *stream, tc_plan **out);

/* Builds a plan from an already formatted matrix (host arrays). */
TC_API tc_status tc_plan_from_format(int M, int N, const tc_format *fmt, const tc_params *params,
                              void *stream, tc_plan **out);

TC_API tc_status tc_plan_destroy(tc_plan *plan);

typedef struct tc_plan_info {
    int M, N;
    int dia_shapes, num_negs, dense_nnz, zero_elements, sparse_nnz;
    int row_start, row_stop;
    int64_t nnz_input;        /* non-zeros of the input pattern               */
    int64_t nnz_csr;          /* entries of the CSR remainder                 */
    int ntiles, ntiles_vector, ntiles_long;
    int64_t device_bytes;     /* HBM held by the plan                         */
    int64_t spmv_bytes;       /* algorithmic bytes of one SpMV                */
    double partition_ms;      /* GPU partition time at creation               */
    int num_contours;         /* thumbnail contours kept (>= min_contour)      */
    int nwtiles;              /* window tiles (0: the plan has no window plan) */
    int window_lo, window_hi; /* x window of rows [r0, r0+n):
                                 [r0 + window_lo, r0 + n + window_hi)          */
    int kernel;               /* the multiply's kernel: TC_KERNEL_*            */
} tc_plan_info;

/* tc_plan_info.kernel */
#define TC_KERNEL_TILES   0   /* persistent grid over staged tiles (tile_mode 0 / 1) */
#define TC_KERNEL_GRID    1   /* one CTA per tile, every tile kind              */
#define TC_KERNEL_LEAN    2   /* one CTA per tile: stream, direct and long tiles */
#define TC_KERNEL_WIDE    3   /* wide direct tiles, one 1024-thread CTA each     */
#define TC_KERNEL_STREAM  4   /* stream tiles only                              */
#define TC_KERNEL_ROWS    5   /* one row per thread, no tiles                   */
#define TC_KERNEL_WINDOW  6   /* window tiles (x staged per tile)               */

TC_API tc_status tc_plan_info_get(const tc_plan *plan, tc_plan_info *info);

/* Copies the plan's format to caller-provided host arrays.  Pass NULL arrays
 * to query sizes only (csrRow needs M+1 ints, csrCol nnz_csr ints, xStart/
 * yStart/xStop dia_shapes ints, nDiasPtr dia_shapes+1, neg_offsets num_negs). */
TC_API tc_status tc_plan_export(const tc_plan *plan, int *xStart, int *yStart, int *xStop,
                         int *nDiasPtr, int *neg_offsets, int *csrRow, int *csrCol);

/* The thumbnail-stage images of the last partition (5 x height x W bytes,
 * 0/255: raster, filled, open-open, subtracted, eye-opened) and the kept
 * shape corners (4 ints each).  Sizes are returned through *W / *ncorners. */
TC_API tc_status tc_plan_thumbnail(const tc_plan *plan, unsigned char *stages, int *W,
                            int *corners, int *ncorners);

/* TC_ERR_TIMEOUT if a multiply of this plan gave up a bounded device-side
 * wait since the last check (its y is then incomplete); TC_OK otherwise.
 * Reading the flag clears it, so each give-up is reported once.
 * Synchronous. */
TC_API tc_status tc_plan_check(const tc_plan *plan);

/* Plan files: the plan's TaiChi_new format and build parameters, so a matrix
 * is partitioned once and reloaded later (a served pool restarts without
 * repartitioning).  No counterpart in the reference, which repartitions on
 * every run (TaiChi.cu:313-638).  tc_plan_load checks the file (magic, sizes,
 * checksum: TC_ERR_FORMAT; unreadable: TC_ERR_IO) before it touches the GPU,
 * then builds the plan with `params` (NULL: the saved parameters). */
TC_API tc_status tc_plan_save(const tc_plan *plan, const char *path);
TC_API tc_status tc_plan_load(const char *path, const tc_params *params, void *stream, tc_plan **out);

/* y = A x.  d_x: N floats, d_y: M floats, device memory.  Stream-ordered. */
TC_API tc_status tc_spmv(const tc_plan *plan, const float *d_x, float *d_y, void *stream);

/* The same multiply in double precision: d_x N doubles, d_y M doubles, device
 * memory, stream-ordered, over the same plan.  Replaces the reference's
 * VALUE_TYPE=double build of taichi_SpMV (TaiChi.h:62-64, TaiChi.cu:1331). */
TC_API tc_status tc_spmv_f64(const tc_plan *plan, const double *d_x, double *d_y, void *stream);

/* Same multiply on host buffers: copies x in, multiplies, copies y out and
 * waits.  Pinned host buffers give the full link bandwidth. */
TC_API tc_status tc_spmv_host(const tc_plan *plan, const float *h_x, float *h_y, void *stream);

#define TC_HOST_SLOTS 4  /* staging slots of tc_spmv_host_async */

/* The same three steps enqueued on `stream` without waiting, through the
 * plan's staging slot `slot` (0 .. TC_HOST_SLOTS-1; slot 0 is the one
 * tc_spmv_host uses).  h_y holds y once the stream has reached this point.
 * Calls on one slot must be ordered on the device (same stream, or an event
 * between streams); slots on separate streams let one call's x copy-in
 * overlap another's y copy-out, and with three or more a copy-in no longer
 * waits for the copy-out two calls back.
 * With TC_FLAG_HOST_Y_MAPPED and a page-locked, device-addressable h_y the
 * multiply itself writes h_y (no copy-out and no device y buffer); h_y must
 * then stay allocated, and unread and unwritten by the host, until the
 * stream has passed this call, as for the copy.
 * No counterpart in the reference (its taichi_SpMV copies synchronously,
 * TaiChi.cu:1357-1420). */
TC_API tc_status tc_spmv_host_async(const tc_plan *plan, const float *h_x, float *h_y, int slot,
                                    void *stream);

/* Y = A X for k right-hand sides (1 <= k <= 64).  X is N x k row-major with
 * leading dimension ldx >= k, Y is M x k with ldy >= k; device memory. */
TC_API tc_status tc_spmm(const tc_plan *plan, const float *d_X, int ldx, int k, float *d_Y,
                  int ldy, void *stream);

/* ----------------------------------------------------------------------- */
/* Thumbnail-level entry points of the GPU partitioner (device arrays).     */
/* ----------------------------------------------------------------------- */

/* Runs the thumbnail raster + morphology + contour tracing of getSdf
 * (morohutils.cu:182-291) on a device CSR.  Writes up to max_corners shape
 * corners (4 ints each, in OpenCV's contour order) to host memory and their
 * count to *ncorners; *mF receives the thumbnail height (0 when the matrix
 * has no thumbnail).  stages (optional, host) receives the 5 stage images. */
TC_API tc_status tc_getsdf(int M, int N, const int *d_rowptr, const int *d_col, const tc_params *p,
                    int *mF, int *W, int *corners, int max_corners, int *ncorners,
                    unsigned char *stages, void *stream);

/* The thumbnail stages of tc_getsdf (raster, filled, open-open, subtracted,
 * eye-opened; 5 x height x W bytes, 0/255) written to caller-owned DEVICE
 * memory, without allocating anything.  No counterpart in the reference: it
 * is for callers that cannot call cudaMalloc at this point -- code running
 * while another framework owns the device allocator, or a latency-critical
 * path that must not add cudaMalloc/cudaFree (they synchronize the device).
 * The working images live in a fixed device array of the library (512 KB,
 * held on every GPU that loads the library until exit), so the thumbnail is
 * limited to height <= 512 and W <= 1024 (TC_ERR_CAPACITY beyond).  The first
 * call on a device (and the first after the device's context was destroyed,
 * e.g. by cudaDeviceReset) looks up that array's address in the current
 * context.  Every call reads a status word back into host memory and
 * synchronizes `stream`, so no call may be made on a stream that is being
 * captured.  Calls share the array: calls that overlap on the GPU race.  *W
 * receives the width (0 when the matrix is too small for a thumbnail, in
 * which case nothing is written).  Parameters are range-checked as in
 * tc_plan_create (TC_ERR_INVALID) before anything is launched. */
TC_API tc_status tc_thumbnail_noalloc(int M, int N, const int *d_rowptr, const int *d_col,
                                      const tc_params *p, unsigned char *d_stages, int *W,
                                      void *stream);

/* Border following (findContours RETR_CCOMP / CHAIN_APPROX_NONE order) of a
 * host H x W 0/nonzero image on the GPU.  Writes contour lengths (up to
 * max_contours) and, for each, its first point and middle point (4 ints) to
 * host memory.  Returns the number of contours in *ncontours. */
TC_API tc_status tc_trace_contours(const unsigned char *img, int H, int W, int *lens, int *ends,
                            int max_contours, int *ncontours);

/* ----------------------------------------------------------------------- */
/* Matrix Market reader (host).                                             */
/* ----------------------------------------------------------------------- */

/* Parses a Matrix Market coordinate file into a malloc'd CSR (free with
 * tc_free).  Same result as readMtx (TaiChi.cu:120-278).  Returns TC_OK or
 * TC_ERR_IO; *ref_code receives the reference's code (0, -1 open, -2 banner,
 * -3 complex, -4 size line, -5 bad entry). */
TC_API tc_status tc_read_mtx(const char *path, int *M, int *N, int64_t *nnz, int **rowptr,
                      int **col, float **val, int *ref_code);
TC_API void tc_free(void *p);

/* The same file with the CSR built on the GPU: the text is parsed on the
 * host (as tc_read_mtx), the entries are copied to the device once, and a
 * stable radix sort by row puts them in readMtx's order (file order within
 * each row, a symmetric file's mirror right after its entry's step) --
 * replacing the host counting sort of readMtx (TaiChi.cu:170-270).  The
 * arrays are device memory (free each with tc_device_free) and can go
 * straight to tc_plan_create with on_device = 1.  *parse_ms / *build_ms
 * (optional) receive the host parse and the device build times.
 * Synchronizes `stream`. */
TC_API tc_status tc_read_mtx_device(const char *path, int *M, int *N, int64_t *nnz, int **d_rowptr,
                                    int **d_col, float **d_val, int *ref_code, double *parse_ms,
                                    double *build_ms, void *stream);
TC_API void tc_device_free(void *p);

/* Synthetic benchmark matrices (no counterpart in the reference, whose
 * datasets are external files): R-MAT graphs (each of ef * 2^scale edges
 * picks a quadrant per level with probabilities a, b, c, 1-a-b-c) and
 * banded patterns (dense diagonals -k..+k plus per_row random columns).
 * Sorted, duplicate-free malloc'd CSR (free with tc_free); multi-threaded,
 * the result depends only on the arguments. */
TC_API tc_status tc_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                             uint64_t seed, int self_loops, int *M, int **rowptr, int **col);
TC_API tc_status tc_gen_banded(int n, int k, int per_row, uint64_t seed, int **rowptr, int **col);

/* ----------------------------------------------------------------------- */
/* Autotuner: density threshold and tile shape, timed per matrix.           */
/* ----------------------------------------------------------------------- */
typedef struct tc_tune_result {
    tc_params params;       /* fastest parameters found                         */
    double spmv_us;         /* their mean multiply time (back-to-back launches) */
    double default_us;      /* the base parameters' time                        */
    int trials;             /* candidates timed (0 when served from the cache)  */
    int cached;             /* 1 when the result came from the cache            */
    uint64_t fingerprint;   /* matrix fingerprint the result is cached under    */
} tc_tune_result;

/* Partitions the host CSR at several density thresholds and tries several
 * tile shapes on the best format (at most max_trials candidates; <= 0 means
 * 32), timing each on the GPU.  Results are cached per matrix fingerprint
 * for the life of the process.  No counterpart in the reference, which fixes
 * the threshold at 0.6 (TaiChi.cu:757). */
TC_API tc_status tc_tune(int M, int N, int64_t nnz, const int *rowptr, const int *col,
                         const tc_params *base, int max_trials, void *stream,
                         tc_tune_result *out);
TC_API void tc_tune_cache_clear(void);

/* ----------------------------------------------------------------------- */
/* Batched form: many resident plans in one persistent launch.              */
/* ----------------------------------------------------------------------- */
typedef struct tc_batch tc_batch;

/* Groups n plans; x[i] / y[i] are device vectors of plan i (fixed at creation
 * so the launch can be captured in a CUDA graph). */
TC_API tc_status tc_batch_create(int n, tc_plan *const *plans, const float *const *d_x,
                          float *const *d_y, tc_batch **out);
TC_API tc_status tc_batch_run(tc_batch *b, void *stream);              /* one launch  */
TC_API tc_status tc_batch_graph_launch(tc_batch *b, void *stream);     /* graph replay */
TC_API tc_status tc_batch_destroy(tc_batch *b);

/* ----------------------------------------------------------------------- */
/* Served form: resident matrices, admission by HBM footprint, continuous   */
/* batching of SpMV requests.  No counterpart in the reference.             */
/* ----------------------------------------------------------------------- */
typedef struct tc_server tc_server;

typedef struct tc_serve_config {
    int64_t hbm_budget;   /* bytes for admitted plans + request arenas (64 GiB)    */
    int64_t arena_bytes;  /* device x / y space of one launch context (256 MiB)   */
    int contexts;         /* launch contexts (streams) (4)                       */
    int max_batch;        /* most requests packed into one launch (64, <= 128)   */
    int max_plans;        /* size of the resident plan table (1024)              */
    int max_inflight;     /* batches on the GPU at once, <= contexts (2): a new
                             batch launches when fewer are in flight, with every
                             request waiting by then                            */
    int max_pending;      /* online requests outstanding at once (65536)         */
    int64_t solo_bytes;   /* a request whose matrix moves at least this many
                             bytes per SpMV runs its own multiply launch (the
                             kernel tc_spmv picks) on a second stream beside
                             its batch's shared launch (16 MiB; 0: never)       */
} tc_serve_config;

typedef struct tc_serve_stats {
    int64_t requests, batches;
    double seconds;       /* first arrival to last completion                    */
    double spmv_per_s;    /* requests / seconds                                  */
    double p50_ms, p99_ms, mean_ms, max_ms;   /* completion - arrival            */
    double mean_batch;    /* requests per launch                                 */
    double mean_service_ms;   /* batch launch to its completion seen (batching)  */
    double mean_launch_us;    /* host time to pack and launch one batch          */
} tc_serve_stats;

TC_API void tc_serve_config_default(tc_serve_config *c);
TC_API tc_status tc_server_create(const tc_serve_config *c, tc_server **out);
/* Makes `plan` resident in the server (not owned; keep it alive).  Returns
 * TC_ERR_CAPACITY when its HBM footprint does not fit the budget left, or its
 * x and y do not fit an arena.  While the server is started, admission reuses
 * the slots of evicted matrices only (TC_ERR_UNSUPPORTED otherwise). */
TC_API tc_status tc_server_admit(tc_server *s, tc_plan *plan, int *matrix_id);
/* TC_ERR_CAPACITY while requests for the matrix are queued or running. */
TC_API tc_status tc_server_evict(tc_server *s, int matrix_id);
TC_API int64_t tc_server_hbm_used(const tc_server *s);

/* Online serving.  tc_server_start launches the server's dispatcher thread:
 * it batches the submitted requests continuously (a batch launches whenever
 * fewer than max_inflight are on the GPU, with every request waiting by then,
 * up to max_batch).  device_vectors != 0: requests carry device x / y that
 * the caller owns (requests in flight together must not share a y); 0: host
 * x / y (pinned memory gives full copy bandwidth), copied through the
 * contexts' arenas.  tc_server_submit may be called from any thread; it
 * returns a ticket for tc_server_poll (non-blocking: *done = 1 once y is
 * complete) or tc_server_wait (blocking, timeout in seconds, < 0: none;
 * TC_ERR_TIMEOUT when it runs out).  A failed batch fails its requests with
 * the dispatcher's status.  tc_server_stats covers the requests completed
 * since the start (latency = completion - submission).  tc_server_stop
 * serves what was submitted, then stops the thread. */
TC_API tc_status tc_server_start(tc_server *s, int device_vectors);
TC_API tc_status tc_server_submit(tc_server *s, int matrix_id, const float *x, float *y,
                                  uint64_t *ticket);
TC_API tc_status tc_server_poll(tc_server *s, uint64_t ticket, int *done);
TC_API tc_status tc_server_wait(tc_server *s, uint64_t ticket, double timeout_s);
TC_API tc_status tc_server_stats(tc_server *s, tc_serve_stats *stats);
TC_API tc_status tc_server_stop(tc_server *s);

/* Serves a request trace in real time: request r arrives arrival_s[r]
 * seconds after the call starts (non-decreasing), multiplies matrix[r] by the
 * host vector h_x[r] and leaves y in h_y[r].  mode 0: continuous batching
 * (the online path above, each request submitted at its arrival time); mode
 * 1: one synchronous request at a time on the calling thread (the plain
 * form).  With TC_SERVE_DEVICE_VECTORS added to the mode, h_x[r] / h_y[r] are
 * device vectors owned by the caller: nothing is copied, and the plain form
 * is one synchronous tc_spmv per request.  latency_ms[r] (optional) receives
 * completion minus arrival.  Not while the server is started. */
#define TC_SERVE_DEVICE_VECTORS 2
TC_API tc_status tc_server_run(tc_server *s, int nreq, const double *arrival_s, const int *matrix,
                               const float *const *h_x, float *const *h_y, int mode,
                               double *latency_ms, tc_serve_stats *stats);
/* Stops the server if started, then frees it. */
TC_API tc_status tc_server_destroy(tc_server *s);

#ifdef __cplusplus
}
#endif
#endif /* TAICHI_B200_H */
