// tc_mtx.cpp -- Matrix Market coordinate file -> host CSR.
//
// Same result as readMtx (TaiChi.cu:120-278): the banner and size line follow
// mmio.cpp:96-218 (5 banner tokens, case-insensitive; '%' comment lines; an
// "M N nnz" line), entries are 1-based and become 0-based, symmetric and
// hermitian files are expanded (the mirrored entry follows the stored one),
// pattern entries get value 1.0, and rows keep file order (a stable counting
// sort, no column sort, no duplicate removal).
//
// The entry section is parsed as a stream of whitespace-separated numbers --
// what the reference's fscanf("%d %d %lg\n") loop reads -- split over host
// threads at line boundaries when every line holds exactly one entry.

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "tc_internal.h"

namespace {

enum Field { F_REAL, F_INT, F_PATTERN };

using Entry = tc::MtxEntry;

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Parses entries from [p, e) as a token stream.  Returns false on a malformed
// token.  When one_per_line, also fails if a line does not hold exactly one
// entry (the caller then re-parses serially).
bool parse_span(const char *p, const char *e, Field fld, bool one_per_line, std::vector<Entry> &out)
{
    const int ntok = fld == F_PATTERN ? 2 : 3;
    char *endp = nullptr;
    while (true) {
        while (p < e && is_ws(*p)) ++p;
        if (p >= e) return true;
        Entry en{0, 0, 1.0f};
        const char *line_start = p;
        for (int t = 0; t < ntok; ++t) {
            while (p < e && is_ws(*p)) {
                if (one_per_line && *p == '\n' && t > 0) return false;
                ++p;
            }
            if (p >= e) return false;
            errno = 0;
            if (t < 2 || fld == F_INT) {
                long v = strtol(p, &endp, 10);
                if (endp == p || errno || v < INT32_MIN || v > INT32_MAX) return false;
                if (t == 0) en.i = (int)v;
                else if (t == 1) en.j = (int)v;
                else en.v = (float)(double)v;
            } else {
                double v = strtod(p, &endp);
                if (endp == p) return false;
                en.v = (float)v;
            }
            if (endp > e) return false;
            p = endp;
        }
        (void)line_start;
        if (one_per_line) {
            while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
            if (p < e && *p != '\n') return false;
        }
        out.push_back(en);
    }
}

}  // namespace

namespace tc {

tc_status mtx_parse(const char *path, MtxCoo &out, int *ref_code)
{
    *ref_code = 0;
    FILE *f = fopen(path, "r");
    if (!f) { *ref_code = -1; return tc::fail(TC_ERR_IO, "cannot open %s", path); }
    char line[1025];
    char t[5][64];
    if (!fgets(line, sizeof line, f) ||
        sscanf(line, "%63s %63s %63s %63s %63s", t[0], t[1], t[2], t[3], t[4]) != 5) {
        fclose(f); *ref_code = -2; return tc::fail(TC_ERR_IO, "%s: no Matrix Market banner", path);
    }
    for (int k = 1; k < 5; ++k)
        for (char *c = t[k]; *c; ++c) *c = (char)tolower((unsigned char)*c);
    Field fld;
    bool sym = false, cplx = false;
    bool ok = strncmp(t[0], "%%MatrixMarket", 14) == 0 && strcmp(t[1], "matrix") == 0 &&
              (strcmp(t[2], "coordinate") == 0 || strcmp(t[2], "array") == 0);
    if (!strcmp(t[3], "real")) fld = F_REAL;
    else if (!strcmp(t[3], "integer")) fld = F_INT;
    else if (!strcmp(t[3], "pattern")) fld = F_PATTERN;
    else if (!strcmp(t[3], "complex")) { fld = F_REAL; cplx = true; }
    else { fld = F_REAL; ok = false; }
    if (!strcmp(t[4], "symmetric") || !strcmp(t[4], "hermitian")) sym = true;
    else if (strcmp(t[4], "general") != 0 && strcmp(t[4], "skew-symmetric") != 0) ok = false;
    if (!ok) { fclose(f); *ref_code = -2; return tc::fail(TC_ERR_IO, "%s: unsupported banner", path); }
    if (cplx) { fclose(f); *ref_code = -3; return tc::fail(TC_ERR_IO, "%s: complex matrices are not supported", path); }

    int M = 0, N = 0;
    unsigned long nz = 0;
    do {
        if (!fgets(line, sizeof line, f)) { fclose(f); *ref_code = -4; return tc::fail(TC_ERR_IO, "%s: no size line", path); }
    } while (line[0] == '%');
    if (sscanf(line, "%d %d %lu", &M, &N, &nz) != 3) {
        int got;
        do {
            got = fscanf(f, "%d %d %lu", &M, &N, &nz);
            if (got == EOF) { fclose(f); *ref_code = -4; return tc::fail(TC_ERR_IO, "%s: bad size line", path); }
        } while (got != 3);
    }
    if (M < 0 || N < 0 || nz > (unsigned long)INT32_MAX) {
        fclose(f); *ref_code = -4; return tc::fail(TC_ERR_IO, "%s: size out of range", path);
    }
    // the rest of the file
    long pos = ftell(f);
    fseek(f, 0, SEEK_END);
    long end = ftell(f);
    fseek(f, pos, SEEK_SET);
    std::vector<char> buf((size_t)std::max(0L, end - pos) + 1);
    size_t got = fread(buf.data(), 1, buf.size() - 1, f);
    fclose(f);
    buf[got] = '\n';
    const char *b = buf.data(), *e = buf.data() + got;

    // parallel parse at line boundaries; serial token stream if lines are irregular
    unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (got < (1u << 20)) nth = 1;
    std::vector<std::vector<Entry>> parts(nth);
    std::vector<char> part_ok(nth, 1);
    std::vector<const char *> cut(nth + 1);
    cut[0] = b;
    cut[nth] = e;
    for (unsigned k = 1; k < nth; ++k) {
        const char *c = b + (size_t)(got * k / nth);
        while (c < e && *c != '\n') ++c;
        cut[k] = std::max(cut[k - 1], c);
    }
    {
        std::vector<std::thread> th;
        for (unsigned k = 0; k < nth; ++k)
            th.emplace_back([&, k] {
                parts[k].reserve((size_t)(nz / nth) + 16);
                part_ok[k] = parse_span(cut[k], cut[k + 1], fld, nth > 1, parts[k]);
            });
        for (auto &x : th) x.join();
    }
    std::vector<MtxEntry> &all = out.entries;
    all.clear();
    bool par_ok = std::all_of(part_ok.begin(), part_ok.end(), [](char c) { return c != 0; });
    if (par_ok) {
        size_t tot = 0;
        for (auto &p : parts) tot += p.size();
        all.reserve(tot);
        for (auto &p : parts) all.insert(all.end(), p.begin(), p.end());
    } else {
        all.clear();
        if (!parse_span(b, e, fld, false, all) && all.size() < nz) {
            *ref_code = -5;
            return tc::fail(TC_ERR_IO, "%s: malformed entry %zu", path, all.size() + 1);
        }
    }
    if (all.size() < nz) {
        *ref_code = -5;
        return tc::fail(TC_ERR_IO, "%s: %zu entries, size line says %lu", path, all.size(), nz);
    }
    all.resize(nz);   // like the reference, read exactly nz entries
    for (auto &en : all) {
        if (en.i < 1 || en.i > M || en.j < 1 || en.j > N || (sym && en.i != en.j && en.j > M)) {
            *ref_code = -5;
            return tc::fail(TC_ERR_IO, "%s: entry (%d,%d) outside %d x %d", path, en.i, en.j, M, N);
        }
    }
    out.M = M;
    out.N = N;
    out.symmetric = sym;
    return TC_OK;
}

}  // namespace tc

extern "C" tc_status tc_read_mtx(const char *path, int *Mo, int *No, int64_t *nnzo, int **rowptr,
                                 int **col, float **val, int *ref_code)
{
    int dummy;
    if (!ref_code) ref_code = &dummy;
    *ref_code = 0;
    if (!path || !Mo || !No || !nnzo || !rowptr || !col || !val)
        return tc::fail(TC_ERR_INVALID, "tc_read_mtx: null argument");
    tc::MtxCoo coo;
    TC_CHECK(tc::mtx_parse(path, coo, ref_code));
    const int M = coo.M, N = coo.N;
    const bool sym = coo.symmetric;
    const std::vector<tc::MtxEntry> &all = coo.entries;

    std::vector<int64_t> cnt((size_t)M + 1, 0);
    for (auto &en : all) {
        cnt[en.i - 1]++;
        if (sym && en.i != en.j) cnt[en.j - 1]++;
    }
    int64_t run = 0;
    int *rp = (int *)malloc(sizeof(int) * ((size_t)M + 1));
    if (!rp) return tc::fail(TC_ERR_ALLOC, "host allocation");
    for (int r = 0; r < M; ++r) { rp[r] = (int)run; run += cnt[r]; }
    if (run > INT32_MAX) { free(rp); return tc::fail(TC_ERR_UNSUPPORTED, "more than 2^31 entries"); }
    rp[M] = (int)run;
    int *co = (int *)malloc(sizeof(int) * (size_t)std::max<int64_t>(run, 1));
    float *va = (float *)malloc(sizeof(float) * (size_t)std::max<int64_t>(run, 1));
    if (!co || !va) { free(rp); free(co); free(va); return tc::fail(TC_ERR_ALLOC, "host allocation"); }
    std::fill(cnt.begin(), cnt.end(), 0);
    for (auto &en : all) {
        int i = en.i - 1, j = en.j - 1;
        int64_t at = rp[i] + cnt[i]++;
        co[at] = j; va[at] = en.v;
        if (sym && i != j) {
            at = rp[j] + cnt[j]++;
            co[at] = i; va[at] = en.v;
        }
    }
    *Mo = M; *No = N; *nnzo = run;
    *rowptr = rp; *col = co; *val = va;
    return TC_OK;
}

extern "C" void tc_free(void *p) { free(p); }
