"""Plan files (tc_plan_save / tc_plan_load): a partitioned matrix reloads
with the same format and multiplies to the same y; damaged or foreign files
are refused before the GPU is touched."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from tests.golden import cases


def _load_status(tc, path):
    h = C.c_void_p()
    return tc.lib().tc_plan_load(os.fsencode(str(path)), None, None, C.byref(h))


def test_refuses_missing_and_foreign_files(tc, tmp_path):
    assert _load_status(tc, tmp_path / "absent.plan") == 4             # TC_ERR_IO
    junk = tmp_path / "junk.plan"
    junk.write_bytes(b"not a plan file at all" * 10)
    assert _load_status(tc, junk) == 5                                 # TC_ERR_FORMAT
    bad = tmp_path / "bad.plan"
    bad.write_bytes(b"TCPLAN\x00\x01" + bytes(64))                      # right magic, wrong hash
    assert _load_status(tc, bad) == 5


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["multi_shape", "rmat16_selfloops", "plain:band_holes"])
def test_roundtrip(tc, dev, tmp_path, name):
    import torch
    plain = name.startswith("plain:")
    case = next(c for c in cases.MATRIX_CASES if c["name"] == name.split(":")[-1])
    M, N, rp, col = cases.matrix(case)
    plan = tc.Plan.from_csr(M, N, rp, col, partition=not plain)
    path = tmp_path / "m.plan"
    plan.save(path)
    again = tc.Plan.load(path)
    a, b = plan.export(), again.export()
    for k in oracle.FORMAT_KEYS:
        assert a[k] == b[k], k
    for k in ("xStart", "yStart", "xStop", "nDiasPtr", "neg_offsets", "csrRow", "csrCol"):
        assert np.array_equal(a[k], b[k]), k
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, N).astype(np.float32)).to(dev)
    y1, y2 = torch.empty(M, device=dev), torch.empty(M, device=dev)
    plan.spmv(x, y1)
    again.spmv(x, y2)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)
    # the saved parameters can be overridden at load time
    other = tc.Plan.load(path, prm=tc.params(tile_mode=1))
    y3 = torch.empty(M, device=dev)
    other.spmv(x, y3)
    torch.cuda.synchronize()
    ref = oracle.spmv_csr_f64(M, rp, col, x.cpu().numpy().astype(np.float64))
    assert np.linalg.norm(y3.cpu().numpy() - ref) <= 1e-5 * np.linalg.norm(ref)
    # one flipped byte is caught by the checksum
    raw = bytearray(path.read_bytes())
    raw[len(raw) // 2] ^= 0x40
    path.write_bytes(bytes(raw))
    with pytest.raises(tc.TcError):
        tc.Plan.load(path)
    for p in (plan, again, other):
        p.close()
