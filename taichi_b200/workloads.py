"""Seeded matrix pools of the batched and served workloads.

batched: 256 binary matrices of uneven size, n log-uniform in [1e3, 2e5];
even-numbered ones R-MAT (a = 0.499, b = c = 0.001, edge factor 8, scale
round(log2 n)), odd-numbered ones banded (dense diagonals -k..+k, k uniform in
1..16, plus 4 random columns per row).

served: 48 resident binary matrices; the first half R-MAT of scales 14..22
(a = 0.499, b = c = 0.001, edge factor 16), the second half banded with n
log-uniform in [1e4, 4e6], k uniform in 1..16 and 2..12 random columns per
row.  Each matrix is seeded by its position.  Generation runs in the
library's multi-threaded host generators (no GPU needed).
"""
import numpy as np


def pool_matrices(kind, count, seed):
    """Seeded matrix pools of the batched (kind='batch') and served
    (kind='serve') workloads."""
    import taichi_b200 as tc
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        if kind == "batch":
            n = int(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
            if i % 2 == 0:
                sc = max(10, int(round(np.log2(n))))
                M, rp, col = tc.gen_rmat(sc, 8, 0.499, 0.001, 0.001, seed=seed * 1000 + i)
                out.append(("rmat%d" % sc, M, rp, col))
            else:
                kk = int(rng.integers(1, 17))
                rp, col = tc.gen_banded(n, kk, 4, seed=seed * 1000 + i)
                out.append(("band%d_k%d" % (n, kk), n, rp, col))
        else:
            if i < count // 2:
                sc = 14 + (i * 9) // (count // 2)          # scales 14..22
                M, rp, col = tc.gen_rmat(sc, 16, 0.499, 0.001, 0.001, seed=seed * 1000 + i)
                out.append(("rmat%d" % sc, M, rp, col))
            else:
                n = int(np.exp(rng.uniform(np.log(1e4), np.log(4e6))))
                kk = int(rng.integers(1, 17))
                rr = int(rng.integers(2, 13))
                rp, col = tc.gen_banded(n, kk, rr, seed=seed * 1000 + i)
                out.append(("band%d_k%d_r%d" % (n, kk, rr), n, rp, col))
    return out


