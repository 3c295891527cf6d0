// tc_partition.cu -- the TaiChi partitioner on the GPU.
//
// Replaces getSdf (morohutils.cu:153-291) and partition_shapes /
// partition_dia_shape (TaiChi.cu:313-879).  Output is bit-identical to the
// reference for the same parameters:
//
//  1. raster       512 x W thumbnail of the pattern (getSdf_GPU1), one CTA per
//                  thumbnail row, bits in shared memory.
//  2. morphology   hole fill (imfill), 30x1 and 1x30 openings, subtraction and
//                  the eye(5) opening, on bit-packed rows in one CTA, with
//                  OpenCV's conventions (non-reflected element, anchor at the
//                  centre, erosion sees 1 and dilation 0 outside the image).
//  3. contours     findContours(RETR_CCOMP, CHAIN_APPROX_NONE): union-find
//                  labelling of 8-connected ones and 4-connected zeros gives
//                  every border's start pixel (Suzuki & Abe: the first pixel of
//                  a component starts its outer border; the pixel left of the
//                  first pixel of a hole starts that hole's border), a scan
//                  gives their discovery order, and one thread per border
//                  follows it.  OpenCV lists outer borders newest first, each
//                  followed by its holes newest first.
//  4. shapes       per kept contour, in order: cal_shape_size, the band
//                  histogram of unclaimed entries, the density test, hole rows
//                  and the claim of dense-diagonal entries.
//  5. assembly     per row: holes (shape, diagonal, row order) then unclaimed
//                  entries in CSR order, with the sign bit.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "tc_ctxcache.h"
#include "tc_internal.h"
#include "tc_scan.cuh"

namespace tc {
namespace {

// ---------------------------------------------------------------- buffers
struct DevBuf {
    void *p = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    tc_status alloc(size_t bytes)
    {
        if (p) { cudaFree(p); p = nullptr; }
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 16));
        if (e != cudaSuccess) return fail(TC_ERR_ALLOC, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
        return TC_OK;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// ------------------------------------------------------------- bit images
// An H x W binary image is stored as H rows of WW = ceil(W/32) uint32 words;
// pixel x of a row is bit (x & 31) of word (x >> 5).  Bits at x >= W are 0.

struct Img {
    unsigned *w;
    int H, W, WW;
    __device__ __forceinline__ unsigned lastmask() const
    {
        const int r = W & 31;
        return r ? (1u << r) - 1u : 0xffffffffu;
    }
    // word k of row y, with `fill` outside the image (also for x >= W)
    __device__ __forceinline__ unsigned get(int y, int k, unsigned fill) const
    {
        if (y < 0 || y >= H || k < 0 || k >= WW) return fill;
        unsigned v = w[y * WW + k];
        if (k == WW - 1) v = (v & lastmask()) | (fill & ~lastmask());
        return v;
    }
    // bits x+d (x = 32k..32k+31) of row y
    __device__ __forceinline__ unsigned shifted(int y, int k, int d, unsigned fill) const
    {
        const int q = d >> 5, r = d & 31;
        const unsigned lo = get(y, k + q, fill);
        if (r == 0) return lo;
        return __funnelshift_r(lo, get(y, k + q + 1, fill), r);
    }
    __device__ __forceinline__ int pix(int y, int x) const
    {
        if (y < 0 || y >= H || x < 0 || x >= W) return 0;
        return (w[y * WW + (x >> 5)] >> (x & 31)) & 1;
    }
};

// Raster (morohutils.cu:153-180): bit (px, col/pN) for every entry of the
// rows of thumbnail row px = row / pM, for px < H and col/pN < W.
__global__ void raster_kernel(const int *__restrict__ rowptr, const int *__restrict__ col, int M,
                              int pM, int pN, Img img)
{
    extern __shared__ unsigned srow[];
    const int px = blockIdx.x;
    for (int k = threadIdx.x; k < img.WW; k += blockDim.x) srow[k] = 0;
    __syncthreads();
    const long r0 = (long)px * pM;
    const long r1 = r0 + pM < (long)M ? r0 + pM : (long)M;   // rows >= H*pM are never drawn
    if (r0 < M) {
        const int b = __ldg(rowptr + r0), e = __ldg(rowptr + r1);
        unsigned cur_w = 0xffffffffu, cur_bits = 0;
        for (int j = b + threadIdx.x; j < e; j += blockDim.x) {
            const int py = __ldg(col + j) / pN;
            if (py < img.W) {
                const unsigned wi = (unsigned)py >> 5, bit = 1u << (py & 31);
                if (wi != cur_w) {
                    if (cur_bits) atomicOr(&srow[cur_w], cur_bits);
                    cur_w = wi;
                    cur_bits = 0;
                }
                cur_bits |= bit;
            }
        }
        if (cur_bits) atomicOr(&srow[cur_w], cur_bits);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < img.WW; k += blockDim.x) img.w[px * img.WW + k] = srow[k];
}

// --------------------------------------------------------------- morphology
// All stages in one CTA; images live wherever the pointers say (shared memory
// for thumbnails up to 32 KB per image, else global memory).

__device__ void erode_dilate_h(const Img &src, Img &tmp, Img &dst, int L)
{
    const int a = L / 2;
    const int n = src.H * src.WW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = i / src.WW, k = i % src.WW;
        unsigned v = 0xffffffffu;
        for (int d = -a; d < L - a; ++d) v &= src.shifted(y, k, d, 0xffffffffu);
        if (k == src.WW - 1) v &= src.lastmask();
        tmp.w[i] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = i / src.WW, k = i % src.WW;
        unsigned v = 0;
        for (int d = -a; d < L - a; ++d) v |= tmp.shifted(y, k, d, 0u);
        if (k == src.WW - 1) v &= src.lastmask();
        dst.w[i] = v;
    }
    __syncthreads();
}

__device__ void erode_dilate_v(const Img &src, Img &tmp, Img &dst, int L)
{
    const int a = L / 2;
    const int n = src.H * src.WW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = i / src.WW, k = i % src.WW;
        unsigned v = 0xffffffffu;
        for (int d = -a; d < L - a; ++d) v &= src.get(y + d, k, 0xffffffffu);
        if (k == src.WW - 1) v &= src.lastmask();
        tmp.w[i] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = i / src.WW, k = i % src.WW;
        unsigned v = 0;
        for (int d = -a; d < L - a; ++d) v |= tmp.get(y + d, k, 0u);
        if (k == src.WW - 1) v &= src.lastmask();
        dst.w[i] = v;
    }
    __syncthreads();
}

__device__ void erode_dilate_eye(const Img &src, Img &tmp, Img &dst, int K)
{
    const int a = K / 2;
    const int n = src.H * src.WW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = i / src.WW, k = i % src.WW;
        unsigned v = 0xffffffffu;
        for (int t = 0; t < K; ++t) v &= src.shifted(y + t - a, k, t - a, 0xffffffffu);
        if (k == src.WW - 1) v &= src.lastmask();
        tmp.w[i] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = i / src.WW, k = i % src.WW;
        unsigned v = 0;
        for (int t = 0; t < K; ++t) v |= tmp.shifted(y + t - a, k, t - a, 0u);
        if (k == src.WW - 1) v &= src.lastmask();
        dst.w[i] = v;
    }
    __syncthreads();
}

// Kogge-Stone fill of `g` through the set bits of `z` toward the MSB / LSB.
__device__ __forceinline__ unsigned fill_up(unsigned g, unsigned z)
{
    g |= z & (g << 1); z &= z << 1;
    g |= z & (g << 2); z &= z << 2;
    g |= z & (g << 4); z &= z << 4;
    g |= z & (g << 8); z &= z << 8;
    g |= z & (g << 16);
    return g;
}
__device__ __forceinline__ unsigned fill_down(unsigned g, unsigned z)
{
    g |= z & (g >> 1); z &= z >> 1;
    g |= z & (g >> 2); z &= z >> 2;
    g |= z & (g >> 4); z &= z >> 4;
    g |= z & (g >> 8); z &= z >> 8;
    g |= z & (g >> 16);
    return g;
}

// imfill (morohutils.cu:73-83): F = B | (zeros of B that a 4-connected flood
// from a zero frame around the image cannot reach).  R grows monotonically;
// alternating full row and full column closures converge.
__device__ void hole_fill(const Img &B, Img &Z, Img &R, Img &F, int *flag)
{
    const int H = B.H, WW = B.WW, n = H * WW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = i / WW, k = i % WW;
        unsigned z = ~B.w[i];
        if (k == WW - 1) z &= B.lastmask();
        Z.w[i] = z;
        unsigned r = 0;
        if (y == 0 || y == H - 1) r = z;
        if (k == 0) r |= z & 1u;
        if (k == WW - 1) {
            const int lb = (B.W - 1) & 31;
            r |= z & (1u << lb);
        }
        R.w[i] = r;
    }
    __syncthreads();
    for (int iter = 0;; ++iter) {
        int changed = 0;
        // rows: left-to-right then right-to-left closure with carries
        for (int y = threadIdx.x; y < H; y += blockDim.x) {
            unsigned carry = 0;
            for (int k = 0; k < WW; ++k) {
                const unsigned z = Z.w[y * WW + k], r0 = R.w[y * WW + k];
                unsigned g = fill_up(r0 | (carry & z & 1u), z);
                carry = g >> 31;
                if (g != r0) { R.w[y * WW + k] = g; changed = 1; }
            }
            carry = 0;
            for (int k = WW - 1; k >= 0; --k) {
                const unsigned z = Z.w[y * WW + k], r0 = R.w[y * WW + k];
                unsigned g = fill_down(r0 | ((carry << 31) & z & 0x80000000u), z);
                carry = g & 1u;
                if (g != r0) { R.w[y * WW + k] = g; changed = 1; }
            }
        }
        __syncthreads();
        // columns: top-down then bottom-up closure, 32 columns per thread
        for (int k = threadIdx.x; k < WW; k += blockDim.x) {
            unsigned prev = R.w[k];
            for (int y = 1; y < H; ++y) {
                const unsigned r0 = R.w[y * WW + k];
                const unsigned g = r0 | (prev & Z.w[y * WW + k]);
                if (g != r0) { R.w[y * WW + k] = g; changed = 1; }
                prev = g;
            }
            prev = R.w[(H - 1) * WW + k];
            for (int y = H - 2; y >= 0; --y) {
                const unsigned r0 = R.w[y * WW + k];
                const unsigned g = r0 | (prev & Z.w[y * WW + k]);
                if (g != r0) { R.w[y * WW + k] = g; changed = 1; }
                prev = g;
            }
        }
        if (!__syncthreads_or(changed)) break;
        if (iter > 4 * H * WW * 32) { if (threadIdx.x == 0) *flag = 1; break; }   // cannot happen
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) F.w[i] = B.w[i] | (Z.w[i] & ~R.w[i]);
    __syncthreads();
}

struct MorphArgs {
    Img B;                    // raster ("rev" image: set where the matrix has entries)
    Img F, O2, D, E;          // filled, open-open, subtracted, eye-opened
    Img T1, T2, T3;           // scratch
    int open_len, eye;
    int use_smem;
    int *flag;
};

__global__ void __launch_bounds__(1024) morph_kernel(MorphArgs a)
{
    extern __shared__ unsigned sm[];
    const int n = a.B.H * a.B.WW;
    Img B = a.B, F = a.F, O2 = a.O2, D = a.D, E = a.E, T1 = a.T1, T2 = a.T2, T3 = a.T3;
    if (a.use_smem) {   // work on shared copies; results are written back
        B.w = sm; T1.w = sm + n; T2.w = sm + 2 * n; T3.w = sm + 3 * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) B.w[i] = a.B.w[i];
        __syncthreads();
    }
    // F = imfill(B)                (T1 = zeros, T2 = reached)
    Img Fw = a.use_smem ? T3 : F;
    hole_fill(B, T1, T2, Fw, a.flag);
    if (a.use_smem) for (int i = threadIdx.x; i < n; i += blockDim.x) F.w[i] = Fw.w[i];
    // O1 = open 30x1 (F)  -> T1 ; O2 = open 1x30 (O1) -> T3
    erode_dilate_h(Fw, T2, T1, a.open_len);
    Img O2w = a.use_smem ? T3 : O2;
    erode_dilate_v(T1, T2, O2w, a.open_len);
    if (a.use_smem) for (int i = threadIdx.x; i < n; i += blockDim.x) O2.w[i] = O2w.w[i];
    // D = B - O2 (saturating) -> T1
    for (int i = threadIdx.x; i < n; i += blockDim.x) T1.w[i] = B.w[i] & ~O2w.w[i];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) D.w[i] = T1.w[i];
    // E = open eye(5) (D)
    Img Ew = a.use_smem ? T3 : E;
    erode_dilate_eye(T1, T2, Ew, a.eye);
    if (a.use_smem) for (int i = threadIdx.x; i < n; i += blockDim.x) E.w[i] = Ew.w[i];
}

// Bytes (nonzero = set) -> bits, and bits -> 0/255 bytes.
__global__ void pack_kernel(const unsigned char *__restrict__ in, Img img)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= img.H * img.WW) return;
    const int y = i / img.WW, k = i % img.WW;
    unsigned v = 0;
    for (int b = 0; b < 32; ++b) {
        const int x = k * 32 + b;
        if (x < img.W && in[(size_t)y * img.W + x]) v |= 1u << b;
    }
    img.w[i] = v;
}

__global__ void unpack_kernel(Img img, unsigned char *__restrict__ out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)img.H * img.W) return;
    const int y = (int)(i / img.W), x = (int)(i % img.W);
    out[i] = img.pix(y, x) ? 255 : 0;
}

// ----------------------------------------------------------------- contours
// Labels: index 0 is the zero frame around the image, pixel (y,x) is 1+y*W+x.
__device__ __forceinline__ int uf_find(int *L, int a)
{
    int b = __ldcg(L + a);
    while (b != a) { a = b; b = __ldcg(L + a); }
    return a;
}

__device__ void uf_union(int *L, int a, int b, int *flag)
{
    for (int it = 0; it < (1 << 24); ++it) {
        a = uf_find(L, a);
        b = uf_find(L, b);
        if (a == b) return;
        if (a < b) {
            const int old = atomicMin(L + b, a);
            if (old == b) return;
            b = old;
        } else {
            const int old = atomicMin(L + a, b);
            if (old == a) return;
            a = old;
        }
    }
    *flag = 2;   // no progress (cannot happen): reported, never waited on
}

__global__ void ccl_init(int *L, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) L[i] = i;
}

// ones: 8-connected; zeros: 4-connected, and zeros on the image border join
// the frame (OpenCV pads the image with a zero frame).
__global__ void ccl_union(Img img, int *L, int *flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int W = img.W, H = img.H;
    if (i >= H * W) return;
    const int y = i / W, x = i % W, me = i + 1;
    const int v = img.pix(y, x);
    if (v) {
        if (x > 0 && img.pix(y, x - 1)) uf_union(L, me, me - 1, flag);
        if (y > 0) {
            if (img.pix(y - 1, x)) uf_union(L, me, me - W, flag);
            if (x > 0 && img.pix(y - 1, x - 1)) uf_union(L, me, me - W - 1, flag);
            if (x + 1 < W && img.pix(y - 1, x + 1)) uf_union(L, me, me - W + 1, flag);
        }
    } else {
        if (x > 0 && !img.pix(y, x - 1)) uf_union(L, me, me - 1, flag);
        if (y > 0 && !img.pix(y - 1, x)) uf_union(L, me, me - W, flag);
        if (x == 0 || y == 0 || x == W - 1 || y == H - 1) uf_union(L, me, 0, flag);
    }
}

__global__ void ccl_flatten(int *L, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) L[i] = uf_find(L, i);
}

// Border start flags: 1 = outer border (first pixel of a component of ones),
// 2 = hole border (pixel left of the first pixel of an enclosed zero region).
__global__ void border_starts(Img img, const int *L, int *flags, int *parent_pix)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int W = img.W;
    if (i >= img.H * W) return;
    const int y = i / W, x = i % W;
    if (img.pix(y, x)) {
        if (L[i + 1] == i + 1) flags[i] = 1;
    } else if (L[i + 1] == i + 1 && x > 0) {
        flags[i - 1] = 2;
        parent_pix[i - 1] = L[i] - 1;        // first pixel of the enclosing ones
    }
}

struct Border {
    int start;      // pixel index y*W+x
    int hole;       // 0 outer, 1 hole
    int parent;     // hole: start pixel of the enclosing outer border
    int len;        // points of the traced contour
    int mid;        // pixel index of point len/2
    long long area2;   // twice the signed area of the contour polygon (shoelace sum)
};

__global__ void nonzero01(const int *__restrict__ f, int *__restrict__ o, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = f[i] != 0;
    if (i == n) o[n] = 0;
}

__global__ void border_compact(const int *flags, const int *order, const int *parent_pix, int n,
                               Border *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flags[i]) return;
    Border b;
    b.start = i;
    b.hole = flags[i] == 2;
    b.parent = b.hole ? parent_pix[i] : -1;
    b.len = 0;
    b.mid = i;
    b.area2 = 0;
    out[order[i]] = b;
}

// Directions: 0 = +x, counter-clockwise on screen (y grows downward).
__constant__ int c_dx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
__constant__ int c_dy[8] = {0, -1, -1, -1, 0, 1, 1, 1};

// Follows one border (Suzuki & Abe steps 3.1-3.5).  With want < 0 returns the
// number of points; otherwise returns the pixel index of point `want`.
// area2 (optional, with want < 0): the shoelace sum over the closed polygon
// of the points, sum of x_i y_{i+1} - x_{i+1} y_i (twice the signed area).
__device__ long follow(const Img &img, int sy, int sx, int hole, long want, long cap, int *flag,
                       long long *area2 = nullptr)
{
    const int W = img.W;
    int s = hole ? 0 : 4;
    const int s0 = s;
    bool found = false;
    do {
        s = (s - 1) & 7;
        if (img.pix(sy + c_dy[s], sx + c_dx[s])) { found = true; break; }
    } while (s != s0);
    if (!found) return want < 0 ? 1 : (long)sy * W + sx;
    const int ly = sy + c_dy[s], lx = sx + c_dx[s];
    int cy = sy, cx = sx;
    for (long n = 0; n < cap; ++n) {
        if (n == want) return (long)cy * W + cx;
        int k = s, ny, nx;
        for (int t = 0; t < 8; ++t) {
            ++k;
            ny = cy + c_dy[k & 7];
            nx = cx + c_dx[k & 7];
            if (img.pix(ny, nx)) break;
        }
        s = k & 7;
        if (area2) *area2 += (long long)cx * ny - (long long)nx * cy;
        if (ny == sy && nx == sx && cy == ly && cx == lx) return want < 0 ? n + 1 : -1;
        cy = ny;
        cx = nx;
        s = (s + 4) & 7;
    }
    *flag = 3;   // longer than any border can be: reported
    return want < 0 ? cap : -1;
}

__global__ void trace_kernel(Img img, Border *bs, int nb, int *flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    Border b = bs[i];
    const int y = b.start / img.W, x = b.start % img.W;
    const long cap = 8L * img.H * img.W + 16;
    long long a2 = 0;
    const long len = follow(img, y, x, b.hole, -1, cap, flag, &a2);
    b.len = (int)len;
    b.area2 = a2;
    const long m = follow(img, y, x, b.hole, len / 2, cap, flag);
    b.mid = m < 0 ? b.start : (int)m;
    bs[i] = b;
}

// ------------------------------------------------------------------ shapes
__device__ __forceinline__ bool is_unclaimed(float v)
{
    const float d = v - FLT_MAX;          // TaiChi.cu:730
    return fabs((double)d) > 1e-8;
}

__global__ void claim_init(const float *__restrict__ val, unsigned char *__restrict__ claimed, long nnz)
{
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nnz) claimed[j] = val ? (is_unclaimed(val[j]) ? 0 : 1) : 0;
}

struct ShapeBox {
    int x, y, a, b;   // row / column corner, column extent (a) and row extent (b)
    int w;            // band half-width
    int nd;           // 2w - 1 candidate diagonals
};

// Per-diagonal counts of unclaimed entries inside the box and the band
// (TaiChi.cu:723-734); one thread per row of the box.
__global__ void band_hist(const int *__restrict__ rowptr, const int *__restrict__ col,
                          const unsigned char *__restrict__ claimed, ShapeBox sb,
                          unsigned *__restrict__ cnt)
{
    extern __shared__ unsigned sh[];
    const bool local = sb.nd <= 8192;
    if (local) {
        for (int i = threadIdx.x; i < sb.nd; i += blockDim.x) sh[i] = 0;
        __syncthreads();
    }
    const int dof = sb.y - sb.x;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x + sb.x; r < (long)sb.x + sb.b;
         r += (long)gridDim.x * blockDim.x) {
        const int b = __ldg(rowptr + r), e = __ldg(rowptr + r + 1);
        const long lo = r + dof - sb.w + 1, hi = r + dof + sb.w - 1;
        for (int j = b; j < e; ++j) {
            const int c = __ldg(col + j);
            if (c < sb.y || c >= sb.y + sb.a || c < lo || c > hi || claimed[j]) continue;
            const int n = (int)(c - r - dof + sb.w - 1);
            if (local) atomicAdd(sh + n, 1u);
            else atomicAdd(cnt + n, 1u);
        }
    }
    if (local) {
        __syncthreads();
        for (int i = threadIdx.x; i < sb.nd; i += blockDim.x)
            if (sh[i]) atomicAdd(cnt + i, sh[i]);
    }
}

// Claims the entries of the dense diagonals (TaiChi.cu:848-874) and counts,
// per dense diagonal and local row, the entries found (for the hole rows).
__global__ void band_claim(const int *__restrict__ rowptr, const int *__restrict__ col,
                           unsigned char *__restrict__ claimed, ShapeBox sb,
                           const int *__restrict__ dense_idx, int *__restrict__ rowcnt,
                           int *__restrict__ dup)
{
    const int dof = sb.y - sb.x;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x + sb.x; r < (long)sb.x + sb.b;
         r += (long)gridDim.x * blockDim.x) {
        const int b = __ldg(rowptr + r), e = __ldg(rowptr + r + 1);
        const long lo = r + dof - sb.w + 1, hi = r + dof + sb.w - 1;
        for (int j = b; j < e; ++j) {
            const int c = __ldg(col + j);
            if (c < sb.y || c >= sb.y + sb.a || c < lo || c > hi || claimed[j]) continue;
            const int d = dense_idx[c - r - dof + sb.w - 1];
            if (d < 0) continue;
            claimed[j] = 1;
            const int old = atomicAdd(rowcnt + (long)d * sb.b + (r - sb.x), 1);
            if (old) *dup = 1;
        }
    }
}

// hole flag of local row r of dense diagonal d: no entry counted there.
__global__ void hole_flags(const int *__restrict__ rowcnt, int b, int start, int len,
                           int *__restrict__ flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < len) flags[i] = rowcnt[start + i] == 0;
    if (i == len) flags[len] = 0;
}

// Duplicate entries: the reference's row walk (TaiChi.cu:809-827) consumes one
// listed entry per row once the row reaches it; a row is a hole when no entry
// is pending.  Sequential per diagonal (only runs when duplicates exist).
__global__ void hole_flags_dups(const int *__restrict__ rowcnt, int start, int len,
                                int *__restrict__ flags)
{
    if (threadIdx.x || blockIdx.x) return;
    long pending = 0;
    for (int i = 0; i < len; ++i) {
        pending += rowcnt[start + i];
        if (pending > 0) { flags[i] = 0; --pending; }
        else flags[i] = 1;
    }
    flags[len] = 0;
}

__global__ void hole_compact(const int *__restrict__ flags, const int *__restrict__ pos, int len,
                             int start, int keep, int *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < len && flags[i] && pos[i] < keep) out[pos[i]] = start + i;
}

// --------------------------------------------------------------- assembly
__global__ void unclaimed_flags(const unsigned char *__restrict__ claimed, long nnz, int *__restrict__ f)
{
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nnz) f[j] = !claimed[j];
    if (j == nnz) f[nnz] = 0;
}

__global__ void hole_row_count(const int *__restrict__ holes, int n, int xStart, int *__restrict__ zc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(zc + xStart + holes[i], 1);
}

__global__ void row_totals(const int *__restrict__ rowptr, const int *__restrict__ sp,
                           const int *__restrict__ zc, int M, int *__restrict__ cnt)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < M) cnt[r] = zc[r] + sp[rowptr[r + 1]] - sp[rowptr[r]];
    if (r == M) cnt[M] = 0;
}

// Holes of one dense diagonal: at most one per row, so rows are distinct.
__global__ void hole_scatter(const int *__restrict__ holes, int n, int xStart, int yStart, int off,
                             const int *__restrict__ rp_out, int *__restrict__ fill,
                             int *__restrict__ cols)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int rs = holes[i], r = xStart + rs;
    cols[rp_out[r] + fill[r]] = (yStart + rs + off) << 1;
    fill[r] += 1;
}

__global__ void sparse_scatter(const int *__restrict__ rowptr, const int *__restrict__ col,
                               const unsigned char *__restrict__ claimed, const int *__restrict__ sp,
                               const int *__restrict__ rp_out, const int *__restrict__ zc, int M,
                               int *__restrict__ cols)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const int b = rowptr[r], e = rowptr[r + 1];
        const int base = rp_out[r] + zc[r] - sp[b];
        for (int j = b; j < e; ++j)
            if (!claimed[j]) cols[base + sp[j]] = (col[j] << 1) + 1;
    }
}

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// Input check: rowptr[0] == 0, non-decreasing, rowptr[M] == nnz, 0 <= col < N.
__global__ void validate_csr(const int *__restrict__ rowptr, const int *__restrict__ col, int M,
                             int N, long nnz, int *__restrict__ bad)
{
    const long stride = (long)gridDim.x * blockDim.x;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < M; r += stride)
        if (rowptr[r + 1] < rowptr[r]) atomicOr(bad, 1);
    for (long j = (long)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride) {
        const int c = col[j];
        if (c < 0 || c >= N) atomicOr(bad, 2);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (rowptr[0] != 0 || rowptr[M] != nnz)) atomicOr(bad, 4);
}

int band_width(int s)     // TaiChi.cu:689-699
{
    double w;
    if (s >= 10000000) w = s * 0.000001;
    else if (s >= 1000000) w = s * 0.00001;
    else if (s >= 100000) w = s * 0.001;
    else if (s >= 10000) w = s * 0.01;
    else w = s * 0.1;
    return (int)w;
}

void start_end(int M_sub, int N_sub, int width, int off, int n, int &start, int &end)   // TaiChi.cu:881-916
{
    const int ao = off < 0 ? -off : off;
    if (M_sub >= N_sub) {
        if (n >= width - 1) { start = 0; end = N_sub - off; }
        else if (ao > M_sub - N_sub) { start = ao; end = M_sub; }
        else { start = ao; end = N_sub + ao; }
    } else {
        if (n <= width - 1) { start = ao; end = M_sub; }
        else if (ao > N_sub - M_sub) { start = 0; end = N_sub - ao; }
        else { start = 0; end = M_sub; }
    }
}

void shape_size(int M, int N, int mF, int x1, int y1, int a1, int b1, int &x, int &y, int &a, int &b)
{   // TaiChi.cu:280-311
    if (M > mF) {
        const float g = (float)M / (float)mF;
        x = (int)((float)x1 * g); y = (int)((float)y1 * g);
        a = (int)((float)a1 * g); b = (int)((float)b1 * g);
    } else if (M < mF) {
        const float g = (float)mF / (float)M;
        x = (int)((float)x1 / g); y = (int)((float)y1 / g);
        a = (int)((float)a1 / g); b = (int)((float)b1 / g);
    } else {
        x = x1; y = y1; a = a1; b = b1;
    }
    if (x < 0) x = 0;
    if (x > M - 1) x = M - 1;
    if (y < 0) y = 0;
    if (y > N - 1) y = N - 1;
    if (y + a > N) a = N - y;
    if (x + b > M) b = M - x;
    if (a > b) a = b; else b = a;
}

}  // namespace

// ======================================================================
// Contours of a bit image already on the device: ordered (len, start, mid).
// ======================================================================
struct ContourList {
    std::vector<int> lens, first, mid;   // pixel indices y*W+x
    std::vector<long long> area2;        // twice the polygon area (signed)
};

static tc_status contours_on_device(const Img &img, cudaStream_t s, ContourList &out)
{
    const int n = img.H * img.W;
    DevBuf lab, flags, order, parent, tmp, bord, flag;
    TC_CHECK(lab.alloc(sizeof(int) * ((size_t)n + 1)));
    TC_CHECK(flags.alloc(sizeof(int) * ((size_t)n + 1)));
    TC_CHECK(order.alloc(sizeof(int) * ((size_t)n + 1)));
    TC_CHECK(parent.alloc(sizeof(int) * ((size_t)n + 1)));
    TC_CHECK(tmp.alloc(sizeof(int) * scan_tmp_ints(n)));
    TC_CHECK(flag.alloc(sizeof(int)));
    TC_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(int) * ((size_t)n + 1), s));
    TC_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
    const int T = 256;
    ccl_init<<<cdiv(n + 1, T), T, 0, s>>>(lab.as<int>(), n);
    ccl_union<<<cdiv(n, T), T, 0, s>>>(img, lab.as<int>(), flag.as<int>());
    ccl_flatten<<<cdiv(n + 1, T), T, 0, s>>>(lab.as<int>(), n);
    border_starts<<<cdiv(n, T), T, 0, s>>>(img, lab.as<int>(), flags.as<int>(), parent.as<int>());
    TC_CUDA(cudaGetLastError());
    // discovery order = raster order of the start pixels
    {
        DevBuf ones;
        TC_CHECK(ones.alloc(sizeof(int) * ((size_t)n + 1)));
        nonzero01<<<cdiv(n + 1, T), T, 0, s>>>(flags.as<int>(), ones.as<int>(), n);
        TC_CUDA(cudaGetLastError());
        TC_CHECK(exclusive_scan(ones.as<int>(), order.as<int>(), n, tmp.as<int>(), s));
    }
    int nb = 0;
    TC_CUDA(cudaMemcpyAsync(&nb, order.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    TC_CUDA(cudaStreamSynchronize(s));
    TC_CHECK(bord.alloc(sizeof(Border) * (size_t)std::max(nb, 1)));
    border_compact<<<cdiv(n, T), T, 0, s>>>(flags.as<int>(), order.as<int>(), parent.as<int>(), n,
                                            bord.as<Border>());
    trace_kernel<<<cdiv(std::max(nb, 1), 64), 64, 0, s>>>(img, bord.as<Border>(), nb, flag.as<int>());
    TC_CUDA(cudaGetLastError());
    std::vector<Border> hb(nb);
    int hflag = 0;
    if (nb) TC_CUDA(cudaMemcpyAsync(hb.data(), bord.p, sizeof(Border) * nb, cudaMemcpyDeviceToHost, s));
    TC_CUDA(cudaMemcpyAsync(&hflag, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    TC_CUDA(cudaStreamSynchronize(s));
    if (hflag) return fail(TC_ERR_UNSUPPORTED, "contour labelling gave up (code %d)", hflag);
    // OpenCV order: outer borders newest first, each followed by its holes
    // newest first.  hb is in discovery order.
    std::vector<int> head(nb, -1), next(nb, -1);
    {
        // outer start pixels are unique and sorted (discovery order)
        std::vector<std::pair<int, int>> os;
        for (int i = 0; i < nb; ++i)
            if (!hb[i].hole) os.push_back({hb[i].start, i});
        for (int i = 0; i < nb; ++i) {
            if (!hb[i].hole) continue;
            auto it = std::lower_bound(os.begin(), os.end(), std::make_pair(hb[i].parent, -1));
            if (it == os.end() || it->first != hb[i].parent)
                return fail(TC_ERR_FORMAT, "hole border without an outer border");
            const int p = it->second;
            next[i] = head[p];
            head[p] = i;
        }
    }
    out.lens.clear(); out.first.clear(); out.mid.clear(); out.area2.clear();
    auto put = [&](const Border &b) {
        out.lens.push_back(b.len); out.first.push_back(b.start); out.mid.push_back(b.mid);
        out.area2.push_back(b.area2);
    };
    for (int i = nb - 1; i >= 0; --i) {
        if (hb[i].hole) continue;
        put(hb[i]);
        for (int j = head[i]; j >= 0; j = next[j]) put(hb[j]);
    }
    return TC_OK;
}


// ======================================================================
// getSdf on the device
// ======================================================================
struct SdfOut {
    int mF = 0, W = 0;
    std::vector<int> corners;               // 4 per kept contour
    std::vector<double> widths;             // per kept contour: area / corner distance
    std::vector<unsigned char> stages;      // 5*H*W when requested
    int ncontours = 0;                      // all contours before the length filter
};

static tc_status getsdf_device(int M, int N, const int *d_rowptr, const int *d_col, const tc_params &p,
                               bool keep_stages, cudaStream_t s, SdfOut &out)
{
    const int H = p.thumb_height;
    out = SdfOut();
    if (M <= H) return TC_OK;                 // morohutils.cu:192-196: no thumbnail
    const int pM = M / H;
    const double scale = (double)H / (double)M;
    const int W = (int)(scale * N);
    if (W <= 0) return fail(TC_ERR_UNSUPPORTED, "thumbnail width is 0 (N < M/%d)", H);
    if ((long)H * W > (1L << 26)) return fail(TC_ERR_UNSUPPORTED, "thumbnail %d x %d too large", H, W);
    const int pN = N / W;
    const int WW = (W + 31) / 32;
    const size_t nw = (size_t)H * WW;
    DevBuf imgs, flag;
    TC_CHECK(imgs.alloc(sizeof(unsigned) * nw * 8));
    TC_CHECK(flag.alloc(sizeof(int)));
    TC_CUDA(cudaMemsetAsync(imgs.p, 0, sizeof(unsigned) * nw * 8, s));
    TC_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
    auto img = [&](int k) { return Img{imgs.as<unsigned>() + k * nw, H, W, WW}; };
    MorphArgs a;
    a.B = img(0); a.F = img(1); a.O2 = img(2); a.D = img(3); a.E = img(4);
    a.T1 = img(5); a.T2 = img(6); a.T3 = img(7);
    a.open_len = p.open_len;
    a.eye = p.eye_size;
    a.flag = flag.as<int>();
    raster_kernel<<<H, 256, sizeof(unsigned) * WW, s>>>(d_rowptr, d_col, M, pM, pN, a.B);
    TC_CUDA(cudaGetLastError());
    const size_t smem = sizeof(unsigned) * nw * 4;
    a.use_smem = smem <= 200 * 1024;
    if (a.use_smem) TC_CHECK(ensure_smem((const void *)morph_kernel, smem));
    morph_kernel<<<1, 1024, a.use_smem ? smem : 0, s>>>(a);
    TC_CUDA(cudaGetLastError());
    ContourList cl;
    TC_CHECK(contours_on_device(a.E, s, cl));
    int hflag = 0;
    TC_CUDA(cudaMemcpyAsync(&hflag, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    TC_CUDA(cudaStreamSynchronize(s));
    if (hflag) return fail(TC_ERR_UNSUPPORTED, "hole fill did not converge");
    out.mF = H;
    out.W = W;
    out.ncontours = (int)cl.lens.size();
    for (size_t i = 0; i < cl.lens.size(); ++i) {
        if (cl.lens[i] < p.min_contour) continue;           // morohutils.cu:138-151
        out.corners.push_back(cl.first[i] % W);             // contour[0].x (column)
        out.corners.push_back(cl.first[i] / W);             // contour[0].y (row)
        out.corners.push_back(cl.mid[i] % W);               // contour[size/2]
        out.corners.push_back(cl.mid[i] / W);
        // morohutils.cu:268-272: contourArea(contour) / |contour[0] - contour[size/2]|
        const double dx = cl.first[i] % W - cl.mid[i] % W, dy = cl.first[i] / W - cl.mid[i] / W;
        const double area = 0.5 * std::fabs((double)cl.area2[i]);
        out.widths.push_back(area / std::sqrt(dx * dx + dy * dy));
    }
    if (keep_stages) {
        DevBuf bytes;
        const size_t px = (size_t)H * W;
        TC_CHECK(bytes.alloc(px * 5));
        for (int k = 0; k < 5; ++k)
            unpack_kernel<<<cdiv((long)px, 256), 256, 0, s>>>(img(k), bytes.as<unsigned char>() + k * px);
        out.stages.resize(px * 5);
        TC_CUDA(cudaMemcpyAsync(out.stages.data(), bytes.p, px * 5, cudaMemcpyDeviceToHost, s));
        TC_CUDA(cudaStreamSynchronize(s));
    }
    return TC_OK;
}

// ======================================================================
// One shape: dense diagonals, holes, claims (TaiChi.cu:677-879)
// ======================================================================
struct ShapeResult {
    int xStart = 0, yStart = 0, Msub = 0, Nsub = 0, width = 0, neg = 0;
    long nnz = 0;
    std::vector<int> offs, start, end, nzero;
    std::vector<long> hole_off;      // offset of each diagonal's holes in `holes`
    DevBuf holes;                    // local hole rows, ascending per diagonal
};

static int g_sms = 0;
static int sm_count()
{
    if (!g_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_sms <= 0) g_sms = 148;
    }
    return g_sms;
}

static tc_status process_shape(const int *d_rowptr, const int *d_col, unsigned char *d_claim, int x,
                               int y, int a, int b, double density, cudaStream_t s, ShapeResult &R)
{
    R.xStart = x; R.yStart = y; R.Msub = b; R.Nsub = a;
    const int small = b < a ? b : a;
    const int w = band_width(small);
    R.width = w;
    const int nd = 2 * w - 1;
    if (nd <= 0 || b <= 0) return TC_OK;
    ShapeBox sb{x, y, a, b, w, nd};
    const int T = 256;
    const int grid = std::max(1, std::min(cdiv(b, T), sm_count() * 8));
    DevBuf cnt, didx, rowcnt, dup;
    TC_CHECK(cnt.alloc(sizeof(unsigned) * nd));
    TC_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned) * nd, s));
    const size_t hsm = nd <= 8192 ? sizeof(unsigned) * nd : 0;
    band_hist<<<grid, T, hsm, s>>>(d_rowptr, d_col, d_claim, sb, cnt.as<unsigned>());
    TC_CUDA(cudaGetLastError());
    std::vector<unsigned> hc(nd);
    TC_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, sizeof(unsigned) * nd, cudaMemcpyDeviceToHost, s));
    TC_CUDA(cudaStreamSynchronize(s));
    std::vector<int> dense_idx(nd, -1);
    for (int n = 0; n < nd; ++n) {
        const int off = n - w + 1;
        int st, en;
        start_end(b, a, w, off, n, st, en);
        const float dens = (float)hc[n] / (float)(en - st);
        if ((double)dens >= density) {           // TaiChi.cu:756-757
            dense_idx[n] = R.neg++;
            R.offs.push_back(off);
            R.start.push_back(st);
            R.end.push_back(en);
            R.nzero.push_back(en - st - (int)hc[n]);
            R.nnz += hc[n];
        }
    }
    if (R.neg == 0) return TC_OK;
    TC_CHECK(didx.alloc(sizeof(int) * nd));
    TC_CHECK(rowcnt.alloc(sizeof(int) * (size_t)R.neg * b));
    TC_CHECK(dup.alloc(sizeof(int)));
    TC_CUDA(cudaMemcpyAsync(didx.p, dense_idx.data(), sizeof(int) * nd, cudaMemcpyHostToDevice, s));
    TC_CUDA(cudaMemsetAsync(rowcnt.p, 0, sizeof(int) * (size_t)R.neg * b, s));
    TC_CUDA(cudaMemsetAsync(dup.p, 0, sizeof(int), s));
    band_claim<<<grid, T, 0, s>>>(d_rowptr, d_col, d_claim, sb, didx.as<int>(), rowcnt.as<int>(),
                                  dup.as<int>());
    TC_CUDA(cudaGetLastError());
    int hdup = 0;
    TC_CUDA(cudaMemcpyAsync(&hdup, dup.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    long total = 0;
    for (int d = 0; d < R.neg; ++d) { R.hole_off.push_back(total); total += std::max(R.nzero[d], 0); }
    TC_CHECK(R.holes.alloc(sizeof(int) * (size_t)std::max(total, 1L)));
    int maxlen = 0;
    for (int d = 0; d < R.neg; ++d) maxlen = std::max(maxlen, R.end[d] - R.start[d]);
    DevBuf flags, pos, tmp;
    TC_CHECK(flags.alloc(sizeof(int) * ((size_t)maxlen + 1)));
    TC_CHECK(pos.alloc(sizeof(int) * ((size_t)maxlen + 1)));
    TC_CHECK(tmp.alloc(sizeof(int) * scan_tmp_ints(maxlen)));
    TC_CUDA(cudaStreamSynchronize(s));
    for (int d = 0; d < R.neg; ++d) {
        const int len = R.end[d] - R.start[d];
        if (R.nzero[d] <= 0 || len <= 0) continue;
        const int *rc = rowcnt.as<int>() + (size_t)d * b;
        if (hdup) hole_flags_dups<<<1, 1, 0, s>>>(rc, R.start[d], len, flags.as<int>());
        else hole_flags<<<cdiv(len + 1, T), T, 0, s>>>(rc, b, R.start[d], len, flags.as<int>());
        TC_CUDA(cudaGetLastError());
        TC_CHECK(exclusive_scan(flags.as<int>(), pos.as<int>(), len, tmp.as<int>(), s));
        hole_compact<<<cdiv(len, T), T, 0, s>>>(flags.as<int>(), pos.as<int>(), len, R.start[d],
                                                R.nzero[d], R.holes.as<int>() + R.hole_off[d]);
        TC_CUDA(cudaGetLastError());
    }
    TC_CUDA(cudaStreamSynchronize(s));
    return TC_OK;
}

// ======================================================================
// The whole partition
// ======================================================================
tc_status gpu_partition(int M, int N, int64_t nnz, const int *d_rowptr, const int *d_col,
                        const float *d_val, const tc_params &prm, bool keep_stages,
                        bool want_claimed, cudaStream_t s, PartitionOut &out)
{
    auto t0 = std::chrono::steady_clock::now();
    out = PartitionOut();
    if (M < 0 || N < 0 || nnz < 0) return fail(TC_ERR_INVALID, "negative sizes");
    DevBuf claim, bad;
    TC_CHECK(claim.alloc((size_t)std::max<int64_t>(nnz, 1)));
    TC_CHECK(bad.alloc(sizeof(int)));
    const int T = 256;
    TC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    validate_csr<<<std::max(1, std::min(cdiv(std::max<long>(nnz, M), T), sm_count() * 16)), T, 0, s>>>(
        d_rowptr, d_col, M, N, nnz, bad.as<int>());
    int hbad = 0;
    TC_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    TC_CUDA(cudaStreamSynchronize(s));
    if (hbad) return fail(TC_ERR_FORMAT, "invalid CSR input (code %d: 1 rowptr decreases, 2 column "
                                         "outside [0, N), 4 rowptr[0]/rowptr[M] wrong)", hbad);
    if (nnz) claim_init<<<cdiv(nnz, T), T, 0, s>>>(d_val, claim.as<unsigned char>(), nnz);
    TC_CUDA(cudaGetLastError());

    SdfOut sdf;
    TC_CHECK(getsdf_device(M, N, d_rowptr, d_col, prm, keep_stages, s, sdf));
    out.thumb_W = sdf.W;
    out.thumb_H = sdf.mF ? prm.thumb_height : 0;
    out.corners = sdf.corners;
    out.stages.swap(sdf.stages);
    out.ncontours = sdf.ncontours;

    const int ns = (int)sdf.corners.size() / 4;
    std::vector<ShapeResult> shapes(ns);
    long dense = 0;
    for (int i = 0; i < ns; ++i) {     // TaiChi.cu:361-421, in shape order
        const int x1 = sdf.corners[4 * i], y1 = sdf.corners[4 * i + 1];
        const int a1 = sdf.corners[4 * i + 2] - x1, b1 = sdf.corners[4 * i + 3] - y1;
        int x, y, a, b;
        shape_size(M, N, sdf.mF, x1, y1, a1, b1, x, y, a, b);
        if (a < prm.min_shape_side || b < prm.min_shape_side) continue;
        TC_CHECK(process_shape(d_rowptr, d_col, claim.as<unsigned char>(), x, y, a, b, prm.density,
                               s, shapes[i]));
        if (shapes[i].nnz > 0) {
            out.dia_shapes++;
            out.num_negs += shapes[i].neg;
            dense += shapes[i].nnz;
        }
    }
    out.dense_nnz = (int)dense;
    out.sparse_nnz = (int)(nnz - dense);
    long zeros = 0;
    out.nDiasPtr.push_back(0);
    for (int i = 0; i < ns; ++i) {
        const ShapeResult &S = shapes[i];
        if (S.nnz <= 0) continue;
        out.xStart.push_back(S.xStart);
        out.yStart.push_back(S.yStart);
        out.xStop.push_back(S.xStart + S.Msub);
        out.nDiasPtr.push_back(out.nDiasPtr.back() + S.neg);
        for (int d = 0; d < S.neg; ++d) { out.offsets.push_back(S.offs[d]); zeros += S.nzero[d]; }
    }
    if (out.dia_shapes == 0) out.nDiasPtr.clear();
    out.zero_elements = (int)zeros;
    if (out.dia_shapes > 0) {
        out.row_start = *std::min_element(out.xStart.begin(), out.xStart.end());
        out.row_stop = *std::max_element(out.xStop.begin(), out.xStop.end());
    }

    if (dense == 0) {
        out.aliases_input = true;     // TaiChi.cu:575-578
        out.nnz_csr = nnz;
    } else {
        // TaiChi.cu:495-612: per row, holes then unclaimed entries
        DevBuf zc, uf, sp, cnt, tmp, fill;
        TC_CHECK(zc.alloc(sizeof(int) * ((size_t)M + 1)));
        TC_CHECK(uf.alloc(sizeof(int) * ((size_t)nnz + 1)));
        TC_CHECK(sp.alloc(sizeof(int) * ((size_t)nnz + 1)));
        TC_CHECK(cnt.alloc(sizeof(int) * ((size_t)M + 1)));
        TC_CHECK(tmp.alloc(sizeof(int) * scan_tmp_ints(std::max<long>(nnz, M))));
        TC_CHECK(fill.alloc(sizeof(int) * ((size_t)M + 1)));
        TC_CUDA(cudaMemsetAsync(zc.p, 0, sizeof(int) * ((size_t)M + 1), s));
        TC_CUDA(cudaMemsetAsync(fill.p, 0, sizeof(int) * ((size_t)M + 1), s));
        for (int i = 0; i < ns; ++i) {
            const ShapeResult &S = shapes[i];
            if (S.nnz <= 0) continue;
            for (int d = 0; d < S.neg; ++d)
                if (S.nzero[d] > 0)
                    hole_row_count<<<cdiv(S.nzero[d], T), T, 0, s>>>(S.holes.as<int>() + S.hole_off[d],
                                                                     S.nzero[d], S.xStart, zc.as<int>());
        }
        unclaimed_flags<<<cdiv(nnz + 1, T), T, 0, s>>>(claim.as<unsigned char>(), nnz, uf.as<int>());
        TC_CUDA(cudaGetLastError());
        TC_CHECK(exclusive_scan(uf.as<int>(), sp.as<int>(), nnz, tmp.as<int>(), s));
        row_totals<<<cdiv((long)M + 1, T), T, 0, s>>>(d_rowptr, sp.as<int>(), zc.as<int>(), M, cnt.as<int>());
        TC_CUDA(cudaGetLastError());
        TC_CUDA(cudaMalloc(&out.d_rowptr, sizeof(int) * ((size_t)M + 1) + 16));
        TC_CHECK(exclusive_scan(cnt.as<int>(), out.d_rowptr, M, tmp.as<int>(), s));
        int total = 0;
        TC_CUDA(cudaMemcpyAsync(&total, out.d_rowptr + M, sizeof(int), cudaMemcpyDeviceToHost, s));
        TC_CUDA(cudaStreamSynchronize(s));
        out.nnz_csr = total;
        TC_CUDA(cudaMalloc(&out.d_cols, sizeof(int) * (size_t)std::max(total, 1) + 16));
        for (int i = 0; i < ns; ++i) {
            const ShapeResult &S = shapes[i];
            if (S.nnz <= 0) continue;
            for (int d = 0; d < S.neg; ++d)
                if (S.nzero[d] > 0)
                    hole_scatter<<<cdiv(S.nzero[d], T), T, 0, s>>>(
                        S.holes.as<int>() + S.hole_off[d], S.nzero[d], S.xStart, S.yStart, S.offs[d],
                        out.d_rowptr, fill.as<int>(), out.d_cols);
        }
        sparse_scatter<<<std::max(1, std::min(cdiv(M, T), sm_count() * 8)), T, 0, s>>>(
            d_rowptr, d_col, claim.as<unsigned char>(), sp.as<int>(), out.d_rowptr, zc.as<int>(), M,
            out.d_cols);
        TC_CUDA(cudaGetLastError());
    }
    if (want_claimed && nnz) {
        out.claimed.resize((size_t)nnz);
        TC_CUDA(cudaMemcpyAsync(out.claimed.data(), claim.p, (size_t)nnz, cudaMemcpyDeviceToHost, s));
    }
    TC_CUDA(cudaStreamSynchronize(s));
    out.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return TC_OK;
}

// One shape on host arrays, for the reference's partition_dia_shape entry.
tc_status gpu_one_shape(int M, int64_t nnz, const int *h_rowptr, const int *h_col, float *h_val,
                        int x, int y, int a, int b, double density, OneShape &o)
{
    cudaStream_t s = 0;
    DevBuf rp, cl, va, claim;
    TC_CHECK(rp.alloc(sizeof(int) * ((size_t)M + 1)));
    TC_CHECK(cl.alloc(sizeof(int) * (size_t)std::max<int64_t>(nnz, 1)));
    TC_CHECK(va.alloc(sizeof(float) * (size_t)std::max<int64_t>(nnz, 1)));
    TC_CHECK(claim.alloc((size_t)std::max<int64_t>(nnz, 1)));
    TC_CUDA(cudaMemcpy(rp.p, h_rowptr, sizeof(int) * ((size_t)M + 1), cudaMemcpyHostToDevice));
    if (nnz) {
        TC_CUDA(cudaMemcpy(cl.p, h_col, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice));
        TC_CUDA(cudaMemcpy(va.p, h_val, sizeof(float) * (size_t)nnz, cudaMemcpyHostToDevice));
        claim_init<<<cdiv(nnz, 256), 256, 0, s>>>(va.as<float>(), claim.as<unsigned char>(), nnz);
    }
    ShapeResult R;
    TC_CHECK(process_shape(rp.as<int>(), cl.as<int>(), claim.as<unsigned char>(), x, y, a, b, density, s, R));
    o.width = R.width; o.neg = R.neg; o.nnz = R.nnz;
    o.offs = R.offs; o.start = R.start; o.end = R.end; o.nzero = R.nzero;
    o.holes.assign(R.neg, std::vector<int>());
    for (int d = 0; d < R.neg; ++d) {
        o.holes[d].resize(std::max(R.nzero[d], 0));
        if (R.nzero[d] > 0)
            TC_CUDA(cudaMemcpy(o.holes[d].data(), R.holes.as<int>() + R.hole_off[d],
                               sizeof(int) * R.nzero[d], cudaMemcpyDeviceToHost));
    }
    if (nnz && R.neg > 0) {
        std::vector<unsigned char> c((size_t)nnz);
        TC_CUDA(cudaMemcpy(c.data(), claim.p, (size_t)nnz, cudaMemcpyDeviceToHost));
        for (int64_t j = 0; j < nnz; ++j)
            if (c[j]) h_val[j] = FLT_MAX;
    }
    return TC_OK;
}

}  // namespace tc

using tc::fail;

extern "C" tc_status tc_getsdf(int M, int N, const int *d_rowptr, const int *d_col, const tc_params *p,
                               int *mF, int *W, int *corners, int max_corners, int *ncorners,
                               unsigned char *stages, void *stream)
{
    if (!mF || !W || !ncorners || M < 0 || N < 0) return fail(TC_ERR_INVALID, "tc_getsdf: bad arguments");
    tc_params prm;
    tc_params_default(&prm);
    if (p) prm = *p;
    TC_CHECK(tc::check_params(prm));
    tc::SdfOut o;
    TC_CHECK(tc::getsdf_device(M, N, d_rowptr, d_col, prm, stages != nullptr, (cudaStream_t)stream, o));
    *mF = o.mF;
    *W = o.W;
    const int n = (int)o.corners.size() / 4;
    *ncorners = n;
    if (corners) memcpy(corners, o.corners.data(), sizeof(int) * 4 * (size_t)std::min(n, max_corners));
    if (stages && !o.stages.empty()) memcpy(stages, o.stages.data(), o.stages.size());
    return n > max_corners && corners ? fail(TC_ERR_CAPACITY, "%d corners, room for %d", n, max_corners) : TC_OK;
}

extern "C" tc_status tc_trace_contours(const unsigned char *img, int H, int W, int *lens, int *ends,
                                       int max_contours, int *ncontours)
{
    if (!img || H <= 0 || W <= 0 || !ncontours) return fail(TC_ERR_INVALID, "tc_trace_contours: bad arguments");
    if ((long)H * W > (1L << 26)) return fail(TC_ERR_UNSUPPORTED, "image too large");
    const int WW = (W + 31) / 32;
    tc::DevBuf bytes, bits;
    TC_CHECK(bytes.alloc((size_t)H * W));
    TC_CHECK(bits.alloc(sizeof(unsigned) * (size_t)H * WW));
    TC_CUDA(cudaMemcpy(bytes.p, img, (size_t)H * W, cudaMemcpyHostToDevice));
    tc::Img im{bits.as<unsigned>(), H, W, WW};
    tc::pack_kernel<<<tc::cdiv((long)H * WW, 256), 256>>>(bytes.as<unsigned char>(), im);
    TC_CUDA(cudaGetLastError());
    tc::ContourList cl;
    TC_CHECK(tc::contours_on_device(im, 0, cl));
    const int n = (int)cl.lens.size();
    *ncontours = n;
    for (int i = 0; i < n && i < max_contours; ++i) {
        if (lens) lens[i] = cl.lens[i];
        if (ends) {
            ends[4 * i + 0] = cl.first[i] % W;
            ends[4 * i + 1] = cl.first[i] / W;
            ends[4 * i + 2] = cl.mid[i] % W;
            ends[4 * i + 3] = cl.mid[i] / W;
        }
    }
    return n > max_contours ? fail(TC_ERR_CAPACITY, "%d contours, room for %d", n, max_contours) : TC_OK;
}

// ======================================================================
// Thumbnail stages without any allocation
// ======================================================================
// Some callers cannot allocate device memory at the point where they need
// the partitioner's thumbnail: code running while another framework owns the
// device allocator, or a caller that must not add cudaMalloc/cudaFree (which
// synchronize the device) to a latency-critical path.  This variant of the
// raster + morphology stages takes its scratch -- the eight bit-packed
// working images and a status word -- from the fixed array below instead of
// cudaMalloc.  The array holds at most a 512 x 1024 thumbnail (512 KB); it
// lives on every GPU that loads the library until the process exits.
namespace tc {
namespace {

constexpr int kNoAllocMaxH = 512, kNoAllocMaxW = 1024;
constexpr int kNoAllocWords = 8 * kNoAllocMaxH * (kNoAllocMaxW / 32);
static __device__ __align__(256) unsigned g_thumb_scratch[kNoAllocWords + 64];

ContextAddressCache<> g_noalloc_cache;

// Id of the CUDA context current on this thread (0 when there is none yet or
// the driver entry points are unavailable).  Read through the driver's entry
// points, so the library does not link libcuda itself.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess && qb == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrent>(a);
            get_id = reinterpret_cast<GetId>(b);
        }
        (void)cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_thumb_scratch in the current context: looked up once
// per device and context (the host-side name is not a device address, and a
// context created after cudaDeviceReset gets a new lookup).
tc_status noalloc_scratch(unsigned **out)
{
    int dev = 0;
    TC_CUDA(cudaGetDevice(&dev));
    TC_CUDA(cudaSetDevice(dev));                 // initialises and makes current its primary context
    void *p = nullptr;
    cudaError_t err = cudaSuccess;
    const int rc = g_noalloc_cache.get(dev, current_context_id(), [&](void **a) {
        err = cudaGetSymbolAddress(a, g_thumb_scratch);
        return err == cudaSuccess ? 0 : 1;
    }, &p);
    if (rc < 0) return fail(TC_ERR_UNSUPPORTED, "device index %d", dev);
    if (rc != 0) {
        (void)cudaGetLastError();
        return fail(TC_ERR_CUDA, "cudaGetSymbolAddress(thumbnail scratch): %s", cudaGetErrorString(err));
    }
    *out = static_cast<unsigned *>(p);
    return TC_OK;
}

}  // namespace
}  // namespace tc

// Same images as tc_getsdf's `stages`, written to caller-owned device memory;
// allocates nothing.  The first call on a device looks up the scratch array's
// address (make it before any stream capture).  All calls share that array,
// so calls that overlap on the GPU (other streams, other threads) race; each
// call rewrites every word it reads before reading it and clears the status
// word itself.  Synchronizes `stream` to read the status word.
extern "C" tc_status tc_thumbnail_noalloc(int M, int N, const int *d_rowptr, const int *d_col,
                                          const tc_params *params, unsigned char *d_stages, int *W_out,
                                          void *stream)
{
    if (!W_out || M < 0 || N < 0 || (M > 0 && !d_rowptr)) return tc::fail(TC_ERR_INVALID, "tc_thumbnail_noalloc: bad arguments");
    *W_out = 0;
    tc_params p;
    tc_params_default(&p);
    if (params) p = *params;
    TC_CHECK(tc::check_params(p));
    const int H = p.thumb_height;
    if (M <= H) return TC_OK;                      // no thumbnail (morohutils.cu:192-196)
    const int W = (int)((double)H / (double)M * N);
    if (W <= 0) return tc::fail(TC_ERR_UNSUPPORTED, "thumbnail width is 0 (N < M/%d)", H);
    if (H > tc::kNoAllocMaxH || W > tc::kNoAllocMaxW)
        return tc::fail(TC_ERR_CAPACITY, "thumbnail %d x %d exceeds the fixed scratch (%d x %d)", H, W,
                        tc::kNoAllocMaxH, tc::kNoAllocMaxW);
    if (!d_stages || !d_col) return tc::fail(TC_ERR_INVALID, "tc_thumbnail_noalloc: null buffer");
    unsigned *scratch = nullptr;
    TC_CHECK(tc::noalloc_scratch(&scratch));
    cudaStream_t s = (cudaStream_t)stream;
    const int pM = M / H, pN = N / W, WW = (W + 31) / 32;
    const size_t nw = (size_t)H * WW;
    auto img = [&](int k) { return tc::Img{scratch + k * nw, H, W, WW}; };
    int *flag = reinterpret_cast<int *>(scratch + tc::kNoAllocWords);
    TC_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    tc::MorphArgs a;
    a.B = img(0); a.F = img(1); a.O2 = img(2); a.D = img(3); a.E = img(4);
    a.T1 = img(5); a.T2 = img(6); a.T3 = img(7);
    a.open_len = p.open_len;
    a.eye = p.eye_size;
    a.flag = flag;
    tc::raster_kernel<<<H, 256, sizeof(unsigned) * WW, s>>>(d_rowptr, d_col, M, pM, pN, a.B);
    TC_CUDA(cudaGetLastError());
    const size_t smem = sizeof(unsigned) * nw * 4;
    a.use_smem = smem <= 200 * 1024;
    if (a.use_smem) {   // raise (never lower) the kernel's shared-memory limit
        cudaFuncAttributes fa;
        TC_CUDA(cudaFuncGetAttributes(&fa, tc::morph_kernel));
        if ((size_t)fa.maxDynamicSharedSizeBytes < smem)
            TC_CUDA(cudaFuncSetAttribute(tc::morph_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    tc::morph_kernel<<<1, 1024, a.use_smem ? smem : 0, s>>>(a);
    TC_CUDA(cudaGetLastError());
    const size_t px = (size_t)H * W;
    for (int k = 0; k < 5; ++k)
        tc::unpack_kernel<<<tc::cdiv((long)px, 256), 256, 0, s>>>(img(k), d_stages + k * px);
    TC_CUDA(cudaGetLastError());
    int hflag = 0;
    TC_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    TC_CUDA(cudaStreamSynchronize(s));
    if (hflag) return tc::fail(TC_ERR_UNSUPPORTED, "hole fill did not converge");
    *W_out = W;
    return TC_OK;
}

// ======================================================================
// getSdf with the reference's C++ signature (morphutils.h:40-41)
// ======================================================================
#include "morphutils.h"

void getSdf(std::string path, int M, int N, int nnz, int *&csrRowIndexHostPtr, int *&csrColIndexHostPtr,
            float *&csrValHostPtr, std::string &category, Point_t &size, int &shapeNum,
            std::vector<Point_t> &shapePoints, std::vector<double> &widths)
{
    (void)path;
    (void)csrValHostPtr;
    category = "diagonal";                        // morohutils.cu:186
    tc_params prm;
    tc_params_default(&prm);
    if (M <= prm.thumb_height) {                  // morohutils.cu:192-196
        printf("the matrix is too small! exit\n");
        return;
    }
    shapeNum = 0;
    auto report = [](tc_status st) {
        if (st != TC_OK) printf("getSdf: %s\n", tc_last_error());
    };
    if (M < 0 || N < 0 || nnz < 0 || !csrRowIndexHostPtr || (nnz > 0 && !csrColIndexHostPtr)) {
        report(tc::fail(TC_ERR_INVALID, "bad arguments"));
        return;
    }
    tc::DevBuf drp, dcol;
    tc_status st = drp.alloc(sizeof(int) * ((size_t)M + 1));
    if (st == TC_OK) st = dcol.alloc(sizeof(int) * (size_t)std::max(nnz, 1));
    if (st == TC_OK && cudaMemcpy(drp.p, csrRowIndexHostPtr, sizeof(int) * ((size_t)M + 1),
                                  cudaMemcpyHostToDevice) != cudaSuccess)
        st = tc::fail(TC_ERR_CUDA, "row pointer upload");
    if (st == TC_OK && nnz > 0 &&
        cudaMemcpy(dcol.p, csrColIndexHostPtr, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice) != cudaSuccess)
        st = tc::fail(TC_ERR_CUDA, "column upload");
    tc::SdfOut o;
    if (st == TC_OK) st = tc::getsdf_device(M, N, drp.as<int>(), dcol.as<int>(), prm, false, nullptr, o);
    if (st != TC_OK) {
        report(st);
        return;
    }
    size.x = o.mF;                                // morohutils.cu:262-263
    size.y = o.W;
    shapeNum = (int)o.corners.size() / 4;
    for (int i = 0; i < shapeNum; ++i) {
        shapePoints.push_back(Point_t{o.corners[4 * i], o.corners[4 * i + 1]});
        shapePoints.push_back(Point_t{o.corners[4 * i + 2], o.corners[4 * i + 3]});
        widths.push_back(o.widths[i]);
    }
}
