"""Writes the golden fixtures in tests/golden/ from the reference itself.

* morphology / contours: cv2 (OpenCV 4.13.0, the stand-in for the OpenCV C++
  library the reference links) run on the images of cases.IMAGE_CASES with the
  exact calls of morohutils.cu:73-83 and 231-261;
* partition: the reference's own partition_shapes (TaiChi.cu:313-638, built
  from source by oracle/build.py into oracle/_ref) run on cases.MATRIX_CASES,
  with the shape corners that the cv2 restatement of getSdf
  (morohutils.cu:182-291) finds;
* readMtx: the reference's readMtx (TaiChi.cu:120-278) on the small files in
  tests/golden/mtx/.

Needs cv2 and oracle/_ref, i.e. a machine with the reference checkout.
Run from the repository root:  python tests/golden/make_golden.py
(``--widths`` writes only sdf_widths.json, getSdf's per-contour widths,
which needs cv2 alone.)
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import cv2  # noqa: E402

import oracle  # noqa: E402
from oracle import build as obuild  # noqa: E402
from tests.golden import cases  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cv2_imfill(src):
    H, W = src.shape
    pad = np.zeros((H + 2, W + 2), np.uint8)
    pad[1:-1, 1:-1] = src
    cv2.floodFill(pad, None, (0, 0), 255)
    return (src | ~pad[1:-1, 1:-1]).astype(np.uint8)


def cv2_open(img, kernel):
    return cv2.morphologyEx(img, cv2.MORPH_OPEN, kernel)


def cv2_contours(img):
    cs, _ = cv2.findContours(img.copy(), cv2.RETR_CCOMP, cv2.CHAIN_APPROX_NONE)
    return [c.reshape(-1, 2).astype(np.int32) for c in cs]


def contour_summary(cs):
    """Count, hashes of all lengths / end points / points, and the first 40
    contours in clear."""
    lens = np.array([len(c) for c in cs], np.int32)
    ends = np.array([[c[0][0], c[0][1], c[len(c) // 2][0], c[len(c) // 2][1]] for c in cs],
                    np.int32).reshape(-1, 4)
    allp = np.concatenate(cs) if cs else np.zeros((0, 2), np.int32)
    return dict(count=len(cs), lens_sha=sha(lens), ends_sha=sha(ends),
                points_sha=sha(allp.astype(np.int32)), lens_head=lens[:40].tolist(),
                ends_head=ends[:40].tolist())


def cv2_getsdf(M, N, rowptr, col):
    """morohutils.cu:182-291 with cv2 calls."""
    H = 512
    if M <= H:
        return 0, 0, np.zeros((0, 4), np.int32), None
    pM = M // H
    W = int(512.0 / M * N)
    pN = N // W
    img = np.full((H, W), 255, np.uint8)
    rows = np.repeat(np.arange(M), np.diff(rowptr)) // pM
    cols = col // pN
    m = (rows < H) & (cols < W)
    img[rows[m], cols[m]] = 0
    rev = (255 - img).astype(np.uint8)
    filled = cv2_imfill(rev)
    o1 = cv2_open(filled, cv2.getStructuringElement(cv2.MORPH_RECT, (30, 1)))
    o2 = cv2_open(o1, cv2.getStructuringElement(cv2.MORPH_RECT, (1, 30)))
    dele = cv2.subtract(rev, o2)
    eo = cv2_open(dele, np.eye(5, dtype=np.uint8))
    cs = [c for c in cv2_contours(eo) if len(c) >= 80]
    corners = np.array([[c[0][0], c[0][1], c[len(c) // 2][0], c[len(c) // 2][1]] for c in cs],
                       np.int32).reshape(-1, 4)
    cv2_getsdf.widths = [cv2_width(c) for c in cs]
    return 512, W, corners, [rev, filled, o2, dele, eo]


def cv2_width(c):
    """morohutils.cu:268-272: contourArea(contour) / |contour[0] - contour[size/2]|."""
    a, b = c[0].astype(np.float64), c[len(c) // 2].astype(np.float64)
    d = np.sqrt((a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2)
    area = cv2.contourArea(c.reshape(-1, 1, 2))
    return float(area / d) if d > 0 else float("inf")


def sdf_widths():
    """getSdf's widths output (area / corner distance per kept contour) for
    every matrix case, written to sdf_widths.json."""
    out = {}
    for c in cases.MATRIX_CASES:
        M, N, rp, col = cases.matrix(c)
        cv2_getsdf.widths = []
        cv2_getsdf(M, N, rp, col)
        out[c["name"]] = cv2_getsdf.widths
    return out


def images():
    out = []
    for c in cases.IMAGE_CASES:
        img = cases.image(**c)
        rec = dict(case=c)
        rec["imfill"] = sha(cv2_imfill(img))
        rec["open_30x1"] = sha(cv2_open(img, cv2.getStructuringElement(cv2.MORPH_RECT, (30, 1))))
        rec["open_1x30"] = sha(cv2_open(img, cv2.getStructuringElement(cv2.MORPH_RECT, (1, 30))))
        rec["open_eye5"] = sha(cv2_open(img, np.eye(5, dtype=np.uint8)))
        rec["contours"] = contour_summary(cv2_contours(img))
        out.append(rec)
    return out


def partitions():
    out = []
    work = tempfile.mkdtemp()
    for c in cases.MATRIX_CASES:
        M, N, rp, col = cases.matrix(c)
        mF, W, corners, stages = cv2_getsdf(M, N, rp, col)
        fmt, val = oracle.ref_partition(M, N, rp, col, corners=corners, mF=mF, W=W, workdir=work)
        rec = dict(name=c["name"], M=int(M), N=int(N), nnz=int(rp[M]), mF=int(mF), W=int(W),
                   corners=corners.tolist(),
                   stages=[sha(s) for s in stages] if stages is not None else None)
        for k in oracle.FORMAT_KEYS:
            rec[k] = int(fmt[k])
        for k in ("xStart", "yStart", "xStop", "nDiasPtr", "neg_offsets"):
            rec[k] = [int(v) for v in fmt[k]]
        rec["csr_null"] = fmt["csrRow"] is None
        if fmt["csrRow"] is not None:
            rec["nnz_csr"] = int(fmt["csrRow"][M])
            rec["csrRow_sha"] = sha(fmt["csrRow"].astype(np.int32))
            rec["csrCol_sha"] = sha(fmt["csrCol"].astype(np.int32))
        claimed = (val == np.float32(np.finfo(np.float32).max)).astype(np.uint8)
        rec["claimed_count"] = int(claimed.sum())
        rec["claimed_sha"] = sha(claimed)
        out.append(rec)
        print("  %-18s M=%-8d nnz=%-9d shapes=%-3d dia_shapes=%d offsets=%s zeros=%d" % (
            c["name"], M, rp[M], len(corners), rec["dia_shapes"], rec["neg_offsets"][:12],
            rec["zero_elements"]), flush=True)
    return out


MTX_FILES = {
    "pattern_general.mtx": "%%MatrixMarket matrix coordinate pattern general\n% a comment\n5 6 7\n1 1\n3 2\n2 6\n5 5\n1 3\n4 4\n3 1\n",
    "real_symmetric.mtx": "%%MatrixMarket matrix coordinate real symmetric\n4 4 6\n1 1 2.5\n2 1 -1\n3 2 0.5\n4 4 1e3\n4 1 7\n3 3 1\n",
    "integer_general.mtx": "%%MatrixMarket Matrix Coordinate Integer General\n%\n%%\n3 3 4\n1 2 5\n2 3 -2\n3 1 9\n1 2 3\n",
    "pattern_hermitian.mtx": "%%MatrixMarket matrix coordinate pattern hermitian\n3 3 3\n2 1\n3 3\n3 1\n",
    "skew.mtx": "%%MatrixMarket matrix coordinate real skew-symmetric\n3 3 2\n2 1 1.5\n3 2 -4\n",
    "empty_rows.mtx": "%%MatrixMarket matrix coordinate pattern general\n6 6 2\n6 1\n2 2\n",
    "bad_banner.mtx": "%%MatrixMarkett vector coordinate pattern general\n2 2 1\n1 1\n",
    "complex.mtx": "%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1 0\n",
    "no_size.mtx": "%%MatrixMarket matrix coordinate pattern general\n% only comments\n",
}


def mtx():
    out = {}
    for name, text in MTX_FILES.items():
        path = os.path.join(HERE, "mtx", name)
        with open(path, "w") as f:
            f.write(text)
        rc, res = oracle.ref_read_mtx(path)
        rec = dict(rc=int(rc))
        if rc == 0:
            M, N, rp, col, val = res
            rec.update(M=int(M), N=int(N), rowptr=rp.tolist(), col=col.tolist(),
                       val=[float(v) for v in val])
        out[name] = rec
    return out


def main():
    if "--widths" in sys.argv:          # sdf_widths.json only
        with open(os.path.join(HERE, "sdf_widths.json"), "w") as f:
            json.dump(dict(_doc="cv2 4.13.0 getSdf widths (morohutils.cu:268-272) per matrix case, "
                                "made by make_golden.py --widths", widths=sdf_widths()), f, indent=1)
        return
    obuild.build_oracle()
    if obuild.build_ref() is None:
        sys.exit("set TAICHI_REFERENCE to the reference checkout to build oracle/_ref")
    os.makedirs(os.path.join(HERE, "mtx"), exist_ok=True)
    print("images ...")
    im = images()
    print("readMtx ...")
    mm = mtx()
    print("partitions ...")
    pa = partitions()
    meta = dict(cv2=cv2.__version__, numpy=np.__version__,
                note="written by tests/golden/make_golden.py")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(dict(meta=meta, images=im, mtx=mm, partitions=pa), f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
