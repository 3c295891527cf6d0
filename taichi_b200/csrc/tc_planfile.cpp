// tc_planfile.cpp -- formatted plans on disk.
//
// No counterpart in the reference, which repartitions every matrix on every
// run (TaiChi.cu:313-638).  A plan file holds the TaiChi_new format of a plan
// (scalars, shape arrays, dense-diagonal offsets, the signed CSR remainder)
// and the parameters it was built with, so a served pool can reload its
// matrices without the partition.  Layout (little-endian):
//
//   "TCPLAN\0\1"                       8 bytes
//   int32  sizeof(tc_params), M, N, dia_shapes, num_negs, dense_nnz,
//          zero_elements, sparse_nnz, row_start, row_stop
//   int64  nnz_csr
//   tc_params                          raw struct
//   int32  xStart[d], yStart[d], xStop[d], nDiasPtr[d+1], offsets[num_negs],
//          csrRow[M+1], csrCol[nnz_csr]
//   uint64 FNV-1a hash of every byte before it
//
// Loading checks the magic, the sizes against the file length and the hash
// before it touches the GPU, then builds the plan with tc_plan_from_format
// (which validates the format itself).

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "tc_internal.h"

using tc::fail;

namespace {

constexpr char kMagic[8] = {'T', 'C', 'P', 'L', 'A', 'N', 0, 1};

struct Hash {
    uint64_t h = 1469598103934665603ULL;
    void add(const void *p, size_t n)
    {
        const unsigned char *b = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ULL;
    }
};

struct Writer {
    FILE *f;
    Hash hash;
    bool ok = true;
    void put(const void *p, size_t n)
    {
        if (!n) return;
        hash.add(p, n);
        ok = ok && fwrite(p, 1, n, f) == n;
    }
};

struct Reader {
    const unsigned char *p, *end;
    bool take(void *dst, size_t n)
    {
        if ((size_t)(end - p) < n) return false;
        memcpy(dst, p, n);
        p += n;
        return true;
    }
};

}  // namespace

extern "C" {

tc_status tc_plan_save(const tc_plan *p, const char *path)
{
    if (!p || !path) return fail(TC_ERR_INVALID, "tc_plan_save: null argument");
    std::vector<int> rp((size_t)p->M + 1), cw((size_t)p->nnz_csr);
    TC_CHECK(tc_plan_export(p, nullptr, nullptr, nullptr, nullptr, nullptr, rp.data(), cw.data()));
    FILE *f = fopen(path, "wb");
    if (!f) return fail(TC_ERR_IO, "cannot open %s for writing", path);
    Writer w{f};
    const int32_t hdr[10] = {(int32_t)sizeof(tc_params), p->M, p->N, p->dia_shapes, p->num_negs, p->dense_nnz,
                             p->zero_elements, p->sparse_nnz, p->row_start, p->row_stop};
    const int64_t nnz_csr = p->nnz_csr;
    w.put(kMagic, sizeof kMagic);
    w.put(hdr, sizeof hdr);
    w.put(&nnz_csr, sizeof nnz_csr);
    w.put(&p->params, sizeof(tc_params));
    auto arr = [&](const std::vector<int> &v) { w.put(v.data(), sizeof(int) * v.size()); };
    arr(p->h_xStart); arr(p->h_yStart); arr(p->h_xStop);
    if (p->dia_shapes > 0) arr(p->h_nDiasPtr);
    arr(p->h_offsets); arr(rp); arr(cw);
    const uint64_t h = w.hash.h;
    w.ok = w.ok && fwrite(&h, 1, sizeof h, f) == sizeof h;
    const bool closed = fclose(f) == 0;
    if (!w.ok || !closed) return fail(TC_ERR_IO, "write to %s failed", path);
    return TC_OK;
}

tc_status tc_plan_load(const char *path, const tc_params *params, void *stream, tc_plan **out)
{
    if (!path || !out) return fail(TC_ERR_INVALID, "tc_plan_load: null argument");
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(TC_ERR_IO, "cannot open %s", path);
    std::vector<unsigned char> buf;
    unsigned char chunk[1 << 16];
    size_t n;
    while ((n = fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + n);
    const bool err = ferror(f) != 0;
    fclose(f);
    if (err) return fail(TC_ERR_IO, "read of %s failed", path);
    if (buf.size() < sizeof kMagic + sizeof(uint64_t) || memcmp(buf.data(), kMagic, sizeof kMagic) != 0)
        return fail(TC_ERR_FORMAT, "%s is not a plan file", path);
    Hash hash;
    hash.add(buf.data(), buf.size() - sizeof(uint64_t));
    uint64_t stored;
    memcpy(&stored, buf.data() + buf.size() - sizeof stored, sizeof stored);
    if (stored != hash.h) return fail(TC_ERR_FORMAT, "%s: checksum mismatch", path);

    Reader r{buf.data() + sizeof kMagic, buf.data() + buf.size() - sizeof(uint64_t)};
    int32_t hdr[10];
    int64_t nnz_csr = 0;
    tc_params saved;
    if (!r.take(hdr, sizeof hdr) || !r.take(&nnz_csr, sizeof nnz_csr))
        return fail(TC_ERR_FORMAT, "%s: truncated header", path);
    if (hdr[0] != (int32_t)sizeof(tc_params) || !r.take(&saved, sizeof saved))
        return fail(TC_ERR_FORMAT, "%s: written by an incompatible library", path);
    const int M = hdr[1], N = hdr[2], dia = hdr[3], negs = hdr[4];
    if (M < 0 || N < 0 || dia < 0 || negs < 0 || nnz_csr < 0 || nnz_csr > (int64_t)1 << 31)
        return fail(TC_ERR_FORMAT, "%s: bad sizes", path);
    const size_t words = 3 * (size_t)dia + (dia > 0 ? (size_t)dia + 1 : 0) + (size_t)negs + (size_t)M + 1 +
                         (size_t)nnz_csr;
    if ((size_t)(r.end - r.p) != words * sizeof(int)) return fail(TC_ERR_FORMAT, "%s: sizes do not match the file", path);
    std::vector<int> xs(dia), ys(dia), xe(dia), ndp(dia > 0 ? dia + 1 : 0), offs(negs), rp((size_t)M + 1),
        cw((size_t)nnz_csr);
    for (std::vector<int> *v : {&xs, &ys, &xe, &ndp, &offs, &rp, &cw}) r.take(v->data(), sizeof(int) * v->size());

    tc_format fmt{};
    fmt.dia_shapes = dia; fmt.num_negs = negs; fmt.dense_nnz = hdr[5];
    fmt.zero_elements = hdr[6]; fmt.sparse_nnz = hdr[7]; fmt.row_start = hdr[8]; fmt.row_stop = hdr[9];
    fmt.xStart = xs.data(); fmt.yStart = ys.data(); fmt.xStop = xe.data();
    fmt.nDiasPtr = ndp.data(); fmt.neg_offsets = offs.data();
    fmt.csrRow = rp.data(); fmt.csrCol = cw.data();
    tc_params prm = params ? *params : saved;
    prm.flags &= ~TC_FLAG_KEEP_HOST;
    if (params && (params->flags & TC_FLAG_KEEP_HOST)) prm.flags |= TC_FLAG_KEEP_HOST;
    return tc_plan_from_format(M, N, &fmt, &prm, stream, out);
}

}  // extern "C"
