"""Seeded generators for the synthetic binary matrices of the benchmark
configurations (the reference's datasets -- SuiteSparse and GTgraph R-MAT
matrices -- are not available here; these stand in with the same shapes,
parameters and value distributions).

Every generator returns ``(M, N, rowptr, col)`` with int32 CSR arrays, columns
sorted within each row and no duplicate entries.  Results depend only on the
arguments (numpy's PCG64 stream, fixed chunking).
"""
import numpy as np

_CHUNK = 1 << 22


def _csr_from_keys(n_rows, n_cols, keys):
    """keys: sorted unique int64 row*n_cols+col."""
    rows = (keys // n_cols).astype(np.int64)
    col = (keys % n_cols).astype(np.int32)
    counts = np.bincount(rows, minlength=n_rows)
    rowptr = np.zeros(n_rows + 1, np.int64)
    np.cumsum(counts, out=rowptr[1:])
    if rowptr[-1] >= 2 ** 31:
        raise ValueError("too many non-zeros for int32 CSR")
    return rowptr.astype(np.int32), col


def rmat(scale, edge_factor=16, a=0.499, b=0.001, c=0.001, seed=1, self_loops=False):
    """R-MAT graph (Chakrabarti et al. 2004): each of edge_factor * 2^scale
    edges picks, level by level, one quadrant with probabilities a, b, c,
    d = 1-a-b-c.  Duplicates are removed; self-loops too unless self_loops."""
    n = 1 << scale
    E = edge_factor * n
    rng = np.random.default_rng(seed)
    ab, abc = a + b, a + b + c
    keys = []
    for lo in range(0, E, _CHUNK):
        m = min(_CHUNK, E - lo)
        r = np.zeros(m, np.int64)
        cc = np.zeros(m, np.int64)
        for lvl in range(scale):
            u = rng.random(m, dtype=np.float32)
            rb = u >= ab
            cb = ((u >= a) & (u < ab)) | (u >= abc)
            bit = np.int64(1) << (scale - 1 - lvl)
            r |= rb * bit
            cc |= cb * bit
        if not self_loops:
            keep = r != cc
            r, cc = r[keep], cc[keep]
        keys.append(np.unique(r * n + cc))
    keys = np.unique(np.concatenate(keys)) if keys else np.zeros(0, np.int64)
    rp, col = _csr_from_keys(n, n, keys)
    return n, n, rp, col


def diag_plus_random(n=65536, offsets=range(-3, 5), extra=10, seed=0):
    """Dense diagonals at `offsets` plus `extra` uniform random columns per
    row, duplicates removed (the small plain configuration)."""
    rng = np.random.default_rng(seed)
    r = np.arange(n, dtype=np.int64)
    parts = []
    for o in offsets:
        c = r + o
        ok = (c >= 0) & (c < n)
        parts.append(r[ok] * n + c[ok])
    rr = np.repeat(r, extra)
    cc = rng.integers(0, n, size=n * extra, dtype=np.int64)
    parts.append(rr * n + cc)
    keys = np.unique(np.concatenate(parts))
    rp, col = _csr_from_keys(n, n, keys)
    return n, n, rp, col


def mesh9(grid=2048, permute_frac=0.02, seed=2):
    """9-point stencil on a grid x grid mesh; then `permute_frac` of the rows
    are chosen at random and their contents permuted among themselves."""
    n = grid * grid
    i = np.arange(n, dtype=np.int64)
    gy, gx = i // grid, i % grid
    # stencil columns i + dy*grid + dx grow with (dy, dx), so rows come out sorted
    offs = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    cols = np.empty((n, 9), np.int64)
    ok = np.empty((n, 9), bool)
    for k, (dy, dx) in enumerate(offs):
        cols[:, k] = i + dy * grid + dx
        ok[:, k] = (gy + dy >= 0) & (gy + dy < grid) & (gx + dx >= 0) & (gx + dx < grid)
    counts = ok.sum(1)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=rp[1:])
    col = cols[ok].astype(np.int32)
    rp = rp.astype(np.int32)
    if permute_frac > 0:
        rng = np.random.default_rng(seed)
        k = int(round(permute_frac * n))
        sel = np.sort(rng.choice(n, size=k, replace=False))
        src = rng.permutation(sel)
        lens = np.diff(rp).astype(np.int64)
        new_lens = lens.copy()
        new_lens[sel] = lens[src]
        perm = np.arange(n)
        perm[sel] = src                   # new row i takes old row perm[i]
        nrp = np.zeros(n + 1, np.int64)
        np.cumsum(new_lens, out=nrp[1:])
        starts = rp[:-1].astype(np.int64)[perm]
        idx = np.repeat(starts - nrp[:-1], new_lens) + np.arange(nrp[-1])
        col = col[idx]
        rp = nrp.astype(np.int32)
    return n, n, rp, col


def segments(n, segs, noise=0, seed=0, n_cols=None):
    """Diagonal segments plus uniform noise.  Each segment is
    (row0, row1, col_offset, halfwidth, keep): rows [row0, row1) get columns
    r + col_offset + d for |d| <= halfwidth, each kept with probability keep
    (missing ones become holes of a dense diagonal).  `noise` random entries
    are added anywhere.  Duplicates are removed."""
    rng = np.random.default_rng(seed)
    N = n if n_cols is None else n_cols
    parts = []
    for (r0, r1, off, hw, keep) in segs:
        r = np.arange(r0, r1, dtype=np.int64)
        for d in range(-hw, hw + 1):
            c = r + off + d
            ok = (c >= 0) & (c < N)
            if keep < 1.0:
                ok &= rng.random(r.size) < keep
            parts.append(r[ok] * N + c[ok])
    if noise:
        parts.append(rng.integers(0, n, noise, dtype=np.int64) * N +
                     rng.integers(0, N, noise, dtype=np.int64))
    keys = np.unique(np.concatenate(parts)) if parts else np.zeros(0, np.int64)
    rp, col = _csr_from_keys(n, N, keys)
    return n, N, rp, col


def banded(n, k, rand_per_row, seed):
    """Dense diagonals -k..+k plus `rand_per_row` uniform random columns per
    row, duplicates removed."""
    return diag_plus_random(n, range(-k, k + 1), rand_per_row, seed)


def to_mtx(path, M, N, rowptr, col, field="pattern", symmetric=False):
    """Writes a Matrix Market coordinate file (1-based)."""
    rows = np.repeat(np.arange(M, dtype=np.int64), np.diff(rowptr)) + 1
    cols = col.astype(np.int64) + 1
    sym = "symmetric" if symmetric else "general"
    with open(path, "w") as f:
        f.write("%%%%MatrixMarket matrix coordinate %s %s\n" % (field, sym))
        f.write("%% written by taichi_b200.matgen\n")
        f.write("%d %d %d\n" % (M, N, len(cols)))
        if field == "pattern":
            np.savetxt(f, np.stack([rows, cols], 1), fmt="%d")
        else:
            np.savetxt(f, np.stack([rows, cols, np.ones_like(rows)], 1), fmt="%d")
