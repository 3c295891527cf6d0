"""Inputs of the golden fixtures, regenerated identically from seeds by
make_golden.py (which records the expected outputs) and by the tests."""
import numpy as np

from taichi_b200 import matgen


def image(seed, H, W, p, kind):
    """A 0/255 uint8 image.  kind: 'noise' (i.i.d. pixels with density p),
    'blobs' (random filled rectangles and rings), 'diag' (diagonal streaks like
    the partitioner's thumbnails)."""
    rng = np.random.default_rng(seed)
    if kind == "noise":
        return ((rng.random((H, W)) < p) * 255).astype(np.uint8)
    img = np.zeros((H, W), np.uint8)
    if kind == "blobs":
        for _ in range(int(p * 40) + 1):
            y0, x0 = rng.integers(0, H), rng.integers(0, W)
            h, w = rng.integers(1, max(2, H // 3)), rng.integers(1, max(2, W // 3))
            img[y0:y0 + h, x0:x0 + w] = 255
            if rng.random() < 0.5 and h > 2 and w > 2:
                img[y0 + 1:y0 + h - 1, x0 + 1:x0 + w - 1] = 0
                if rng.random() < 0.5 and h > 4 and w > 4:
                    img[y0 + 2:y0 + h - 2, x0 + 2:x0 + w - 2] = 255
        img[rng.random((H, W)) < p * 0.05] = 255
        return img
    # diag: a few thick diagonal streaks with gaps plus speckle
    for _ in range(int(p * 10) + 1):
        off = int(rng.integers(-H // 2, W // 2 + 1))
        t = int(rng.integers(1, 6))
        a, b = sorted(rng.integers(0, H, 2))
        for y in range(a, b):
            for d in range(t):
                x = y + off + d
                if 0 <= x < W and rng.random() < 0.97:
                    img[y, x] = 255
    img[rng.random((H, W)) < p * 0.02] = 255
    return img


IMAGE_CASES = (
    [dict(seed=s, H=int(h), W=int(w), p=float(p), kind="noise")
     for s, (h, w, p) in enumerate([(1, 1, .5), (1, 7, .5), (7, 1, .5), (3, 3, 1.), (2, 2, 0.),
                                    (16, 16, .3), (31, 17, .5), (40, 64, .7), (64, 40, .2),
                                    (128, 128, .5), (100, 257, .45), (512, 512, .5)])] +
    [dict(seed=100 + s, H=int(h), W=int(w), p=float(p), kind="blobs")
     for s, (h, w, p) in enumerate([(32, 32, .2), (64, 96, .5), (128, 128, .8), (200, 150, .3),
                                    (512, 512, .6), (300, 511, .9)])] +
    [dict(seed=200 + s, H=int(h), W=int(w), p=float(p), kind="diag")
     for s, (h, w, p) in enumerate([(64, 64, .3), (128, 128, .5), (256, 256, .5), (512, 512, .4),
                                    (512, 512, .9), (512, 300, .6), (400, 512, .7)])]
)


# Matrices whose partition is pinned against the reference's own code.
MATRIX_CASES = [
    dict(name="tiny_no_thumb", gen="segments", args=dict(n=400, segs=[(0, 400, 0, 2, 1.0)], noise=10, seed=1)),
    dict(name="band_holes", gen="segments", args=dict(n=20000, segs=[(0, 20000, 0, 2, 0.97)], noise=500, seed=2)),
    dict(name="two_segments", gen="segments",
         args=dict(n=60000, segs=[(0, 30000, 0, 1, 1.0), (30000, 60000, -20000, 3, 0.9)], noise=2000, seed=3)),
    dict(name="offdiag_blocks", gen="segments",
         args=dict(n=100000, segs=[(0, 50000, 40000, 2, 0.95), (50000, 100000, -30000, 1, 0.99),
                                   (10000, 90000, 0, 0, 0.7)], noise=5000, seed=4)),
    dict(name="wide_band", gen="segments", args=dict(n=30000, segs=[(0, 30000, 0, 12, 0.8)], noise=100, seed=5)),
    dict(name="overlap", gen="segments",
         args=dict(n=80000, segs=[(0, 60000, 0, 1, 0.98), (20000, 80000, 5, 2, 0.9)], noise=300, seed=6)),
    dict(name="rect_cols", gen="segments",
         args=dict(n=50000, n_cols=80000, segs=[(0, 50000, 10000, 2, 0.95)], noise=400, seed=7)),
    dict(name="multi_shape", gen="segments",
         args=dict(n=200000, segs=[(0, 80000, 100000, 1, 0.99), (100000, 200000, -100000, 2, 0.95),
                                   (20000, 90000, 0, 0, 1.0)], noise=1000, seed=8)),
    dict(name="many_shapes", gen="segments",
         args=dict(n=300000, segs=[(0, 60000, 150000, 0, 1.0), (70000, 140000, 100000, 1, 0.9),
                                   (150000, 230000, -120000, 0, 0.97), (240000, 300000, -200000, 2, 0.9),
                                   (0, 300000, 0, 0, 0.65)], noise=3000, seed=9)),
    dict(name="cfg1_small", gen="diag_plus_random", args=dict(n=65536, seed=0)),
    dict(name="rmat16_selfloops", gen="rmat", args=dict(scale=16, seed=1, self_loops=True)),
    dict(name="rmat20", gen="rmat", args=dict(scale=20, seed=1)),
    dict(name="rmat20_selfloops", gen="rmat", args=dict(scale=20, seed=1, self_loops=True)),
    dict(name="mesh2048", gen="mesh9", args=dict(grid=2048, permute_frac=0.02, seed=2)),
]


def matrix(case):
    fn = getattr(matgen, case["gen"])
    args = dict(case["args"])
    if "segs" in args:
        args["segs"] = [tuple(s) for s in args["segs"]]
    return fn(**args)
