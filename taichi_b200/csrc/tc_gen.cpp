// tc_gen.cpp -- multi-threaded generators of the synthetic benchmark matrices
// (R-MAT graphs and banded-plus-random patterns) for the batched and served
// workloads, whose pools hold matrices of up to 4M rows.  A counter-based
// hash (splitmix64) makes every entry a function of (seed, position), so the
// output does not depend on the thread count.  Output: malloc'd CSR with
// sorted, duplicate-free columns (free with tc_free).

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "tc_internal.h"

namespace {

inline uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

inline double unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

unsigned threads_for(int64_t work)
{
    unsigned t = std::max(1u, std::thread::hardware_concurrency());
    if (work < (1 << 16)) t = 1;
    return std::min(t, 64u);
}

template <class F>
void parallel_for(int64_t n, F f)
{
    const unsigned nt = threads_for(n);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] { f(n * t / nt, n * (t + 1) / nt, t); });
    for (auto &x : th) x.join();
}

tc_status to_csr(int64_t n_rows, std::vector<uint64_t> &keys, int64_t n_cols, int **rowptr, int **col)
{
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    if ((int64_t)keys.size() > INT32_MAX) return tc::fail(TC_ERR_UNSUPPORTED, "too many entries");
    int *rp = (int *)calloc((size_t)n_rows + 1, sizeof(int));
    int *cl = (int *)malloc(sizeof(int) * std::max<size_t>(keys.size(), 1));
    if (!rp || !cl) { free(rp); free(cl); return tc::fail(TC_ERR_ALLOC, "host allocation"); }
    for (size_t i = 0; i < keys.size(); ++i) {
        rp[keys[i] / n_cols + 1]++;
        cl[i] = (int)(keys[i] % n_cols);
    }
    for (int64_t r = 0; r < n_rows; ++r) rp[r + 1] += rp[r];
    *rowptr = rp;
    *col = cl;
    return TC_OK;
}

}  // namespace

// R-MAT (Chakrabarti, Zhan, Faloutsos 2004): each of ef * 2^scale edges picks
// a quadrant per level with probabilities a, b, c, 1-a-b-c.
extern "C" tc_status tc_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                                 uint64_t seed, int self_loops, int *M, int **rowptr, int **col)
{
    if (scale < 1 || scale > 30 || edge_factor < 1 || !M || !rowptr || !col)
        return tc::fail(TC_ERR_INVALID, "tc_gen_rmat: bad arguments");
    const int64_t n = 1LL << scale, E = (int64_t)edge_factor * n;
    const double ab = a + b, abc = a + b + c;
    const unsigned nt = threads_for(E);
    std::vector<std::vector<uint64_t>> part(nt);
    parallel_for(E, [&](int64_t lo, int64_t hi, unsigned t) {
        auto &out = part[t];
        out.reserve((size_t)((hi - lo) / (self_loops ? 1 : 16) + 16));
        for (int64_t e = lo; e < hi; ++e) {
            uint64_t r = 0, cc = 0;
            uint64_t h = mix64(seed * 0x632BE59BD9B4E019ULL + (uint64_t)e);
            for (int l = 0; l < scale; ++l) {
                h = mix64(h + (uint64_t)l);
                const double u = unit(h);
                const uint64_t bit = 1ULL << (scale - 1 - l);
                if (u >= ab) r |= bit;
                if ((u >= a && u < ab) || u >= abc) cc |= bit;
            }
            if (self_loops || r != cc) out.push_back(r * (uint64_t)n + cc);
        }
    });
    std::vector<uint64_t> keys;
    size_t tot = 0;
    for (auto &p : part) tot += p.size();
    keys.reserve(tot);
    for (auto &p : part) keys.insert(keys.end(), p.begin(), p.end());
    *M = (int)n;
    return to_csr(n, keys, n, rowptr, col);
}

// Dense diagonals -k..+k plus `per_row` uniform random columns per row,
// duplicates removed.
extern "C" tc_status tc_gen_banded(int n, int k, int per_row, uint64_t seed, int **rowptr, int **col)
{
    if (n < 1 || k < 0 || per_row < 0 || !rowptr || !col)
        return tc::fail(TC_ERR_INVALID, "tc_gen_banded: bad arguments");
    std::vector<int> len((size_t)n);
    const int w = 2 * k + 1 + per_row;
    auto row_cols = [&](int64_t r, int *buf) {
        int m = 0;
        for (int d = -k; d <= k; ++d)
            if (r + d >= 0 && r + d < n) buf[m++] = (int)(r + d);
        for (int i = 0; i < per_row; ++i)
            buf[m++] = (int)(mix64(seed * 0xD1B54A32D192ED03ULL + (uint64_t)r * 131 + (uint64_t)i) % (uint64_t)n);
        std::sort(buf, buf + m);
        return (int)(std::unique(buf, buf + m) - buf);
    };
    parallel_for(n, [&](int64_t lo, int64_t hi, unsigned) {
        std::vector<int> buf(w);
        for (int64_t r = lo; r < hi; ++r) len[r] = row_cols(r, buf.data());
    });
    int *rp = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    if (!rp) return tc::fail(TC_ERR_ALLOC, "host allocation");
    int64_t run = 0;
    for (int r = 0; r < n; ++r) { rp[r] = (int)run; run += len[r]; }
    if (run > INT32_MAX) { free(rp); return tc::fail(TC_ERR_UNSUPPORTED, "too many entries"); }
    rp[n] = (int)run;
    int *cl = (int *)malloc(sizeof(int) * std::max<int64_t>(run, 1));
    if (!cl) { free(rp); return tc::fail(TC_ERR_ALLOC, "host allocation"); }
    parallel_for(n, [&](int64_t lo, int64_t hi, unsigned) {
        std::vector<int> buf(w);
        for (int64_t r = lo; r < hi; ++r) {
            const int m = row_cols(r, buf.data());
            memcpy(cl + rp[r], buf.data(), sizeof(int) * m);
        }
    });
    *rowptr = rp;
    *col = cl;
    return TC_OK;
}
