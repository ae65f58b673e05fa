"""GPU parity of the kernel tier (tb_block_multiply, tb_block_assign, fill / axpby /
norm / dot / random fill) against the oracle, through the C ABI.

Tolerance for FP64 contractions: max |gpu - oracle| <= 1e-12 * max |oracle| (the plain
FP64 path must match the reference's block_multiply within 1e-12 relative)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tamm_b200 import _capi as A

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from test_oracle import DIMS, LAB, PATTERNS, _mk  # noqa: E402

FP64_RTOL = 1e-12


def rel_err(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    scale = max(float(np.max(np.abs(ref))) if ref.size else 0.0, 1e-300)
    return float(np.max(np.abs(x - ref))) / scale if ref.size else 0.0


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x).reshape(-1).copy()).cuda()


def i64(v):
    a = np.asarray(list(v) or [0], dtype=np.int64)
    return a


def i32(v):
    return np.asarray(list(v) or [0], dtype=np.int32)


def gpu_block_multiply(alpha, A_, al, B_, bl, beta, C0, cl, is_assign, mode=A.TB_MODE_FP64):
    da, db, dc = dev(A_), dev(B_), dev(C0)
    ad, bd, cd = i64(A_.shape), i64(B_.shape), i64(C0.shape)
    la, lb, lc = i32(al), i32(bl), i32(cl)
    s = torch.cuda.current_stream().cuda_stream
    A.call("tb_block_multiply", alpha, da.data_ptr(), ad.ctypes.data_as(A.i64p), la.ctypes.data_as(A.ip),
           A_.ndim, db.data_ptr(), bd.ctypes.data_as(A.i64p), lb.ctypes.data_as(A.ip), B_.ndim, beta,
           dc.data_ptr(), cd.ctypes.data_as(A.i64p), lc.ctypes.data_as(A.ip), C0.ndim, int(is_assign),
           mode, C.c_void_p(s))
    torch.cuda.synchronize()
    return dc.cpu().numpy().reshape(C0.shape)


@pytest.mark.parametrize("cl,al,bl", PATTERNS)
@pytest.mark.parametrize("beta", [1.0, 0.0, 0.5])
@pytest.mark.parametrize("is_assign", [0, 1])
def test_block_multiply_patterns(cl, al, bl, beta, is_assign):
    A_, B_, C0 = _mk(al, 1), _mk(bl, 2), _mk(cl, 3)
    want = np.array(C0, copy=True)
    assert O.block_multiply(1.3, A_, [LAB[c] for c in al], B_, [LAB[c] for c in bl], beta, want,
                            [LAB[c] for c in cl], is_assign) == 0
    got = gpu_block_multiply(1.3, A_, [LAB[c] for c in al], B_, [LAB[c] for c in bl], beta, C0,
                             [LAB[c] for c in cl], is_assign)
    assert rel_err(got, want) <= FP64_RTOL


@pytest.mark.parametrize("shape", [
    dict(a=10, b=10, c=10, d=10, i=10, j=10),     # config-1 tile pair
    dict(a=24, b=31, c=29, d=37, i=20, j=20),     # uneven ladder tiles crossing 128/64/16 edges
    dict(a=48, b=48, c=48, d=47, i=20, j=20),     # largest ladder tile pair
    dict(a=1, b=1, c=1, d=1, i=1, j=1),           # 1-element blocks
    dict(a=3, b=130, c=17, d=1, i=2, j=65),       # ragged M / N / K
])
@pytest.mark.parametrize("labels", [("abij", "abcd", "cdij"), ("abij", "acid", "cbdj"),
                                    ("ijab", "cadb", "jdci")])
def test_block_multiply_ragged_tiles(shape, labels):
    cl, al, bl = labels
    lab = {c: -ord(c) for c in "abcdij"}
    A_ = np.zeros([shape[c] for c in al])
    B_ = np.zeros([shape[c] for c in bl])
    C0 = np.zeros([shape[c] for c in cl])
    O.fill_uniform(A_.reshape(-1), 11)
    O.fill_uniform(B_.reshape(-1), 12)
    O.fill_uniform(C0.reshape(-1), 13)
    want = np.array(C0, copy=True)
    assert O.block_multiply(0.75, A_, [lab[c] for c in al], B_, [lab[c] for c in bl], 1.0, want,
                            [lab[c] for c in cl], 0) == 0
    got = gpu_block_multiply(0.75, A_, [lab[c] for c in al], B_, [lab[c] for c in bl], 1.0, C0,
                             [lab[c] for c in cl], 0)
    assert rel_err(got, want) <= FP64_RTOL


def test_block_multiply_rejects_bad_args():
    L = A.lib()
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    d = i64([2, 2])
    l1, l2 = i32([-1, -2]), i32([-1, -3])
    rc = L.tb_block_multiply(1.0, None, d.ctypes.data_as(A.i64p), l1.ctypes.data_as(A.ip), 2,
                             x.data_ptr(), d.ctypes.data_as(A.i64p), l2.ctypes.data_as(A.ip), 2, 1.0,
                             x.data_ptr(), d.ctypes.data_as(A.i64p), l1.ctypes.data_as(A.ip), 2, 0, 0, None)
    assert rc == A.TB_ERR_INVALID
    bad = i64([2, 3])  # inner extent mismatch between A and B
    rc = L.tb_block_multiply(1.0, x.data_ptr(), d.ctypes.data_as(A.i64p), l1.ctypes.data_as(A.ip), 2,
                             x.data_ptr(), bad.ctypes.data_as(A.i64p), l2.ctypes.data_as(A.ip), 2, 1.0,
                             x.data_ptr(), d.ctypes.data_as(A.i64p), i32([-2, -3]).ctypes.data_as(A.ip),
                             2, 0, 0, None)
    assert rc == A.TB_ERR_INVALID and "extents" in A.last_error()


@pytest.mark.parametrize("dl,sl,dims", [
    ("ijk", "kij", dict(i=3, j=4, k=5)), ("ij", "ji", dict(i=67, j=45)), ("ij", "ij", dict(i=5, j=7)),
    ("abij", "baji", dict(a=24, b=31, i=20, j=20)), ("abij", "ijab", dict(a=40, b=9, i=33, j=12)),
    ("ij", "ijk", dict(i=3, j=4, k=2)), ("ijk", "ij", dict(i=3, j=4, k=2)), ("", "", {}),
    ("abcd", "dcba", dict(a=8, b=9, c=10, d=11))])
@pytest.mark.parametrize("is_assign", [0, 1])
def test_block_assign(dl, sl, dims, is_assign):
    S = np.zeros([dims[c] for c in sl])
    D0 = np.zeros([dims[c] for c in dl])
    O.fill_uniform(S.reshape(-1), 5)
    O.fill_uniform(D0.reshape(-1), 6)
    lab = {c: -ord(c) for c in "abcdijk"}
    want = np.array(D0, copy=True)
    assert O.assign(want, [lab[c] for c in dl], 0.7, S, [lab[c] for c in sl], is_assign) == 0
    ds, dd = dev(S), dev(D0)
    A.call("tb_block_assign", dd.data_ptr(), i64(D0.shape).ctypes.data_as(A.i64p),
           i32([lab[c] for c in dl]).ctypes.data_as(A.ip), D0.ndim, 0.7, ds.data_ptr(),
           i64(S.shape).ctypes.data_as(A.i64p), i32([lab[c] for c in sl]).ctypes.data_as(A.ip), S.ndim,
           is_assign, None)
    torch.cuda.synchronize()
    # the device may fuse dst + scale*src into one FMA: last-ulp differences only
    np.testing.assert_allclose(dd.cpu().numpy().reshape(D0.shape), want, rtol=1e-15, atol=1e-15)


def test_fill_axpby_norm_dot():
    n = 1_000_003
    x = np.zeros(n)
    y = np.zeros(n)
    O.fill_uniform(x, 1)
    O.fill_uniform(y, 2)
    dx, dy = dev(x), dev(y)
    out = C.c_double()
    A.call("tb_norm2", dx.data_ptr(), n, C.byref(out), None)
    assert abs(out.value - np.linalg.norm(x)) <= 1e-12 * np.linalg.norm(x)
    A.call("tb_dot", dx.data_ptr(), dy.data_ptr(), n, C.byref(out), None)
    assert abs(out.value - float(x @ y)) <= 1e-11 * np.linalg.norm(x) * np.linalg.norm(y)
    A.call("tb_axpby", 2.0, dx.data_ptr(), 0.5, dy.data_ptr(), n, None)
    torch.cuda.synchronize()
    np.testing.assert_allclose(dy.cpu().numpy(), 2.0 * x + 0.5 * y, rtol=1e-15, atol=1e-15)
    A.call("tb_fill", dx.data_ptr(), n, 3.25, 1, None)
    A.call("tb_fill", dx.data_ptr(), n - 1, 1.0, 0, None)
    torch.cuda.synchronize()
    h = dx.cpu().numpy()
    assert np.all(h[:-1] == 4.25) and h[-1] == 3.25
    A.call("tb_norm2", dx.data_ptr(), 0, C.byref(out), None)
    assert out.value == 0.0


def test_fill_random_matches_generator():
    n = 100_000
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    for dist, p0, p1 in [(0, -1.0, 1.0), (1, 0.0, 2.0)]:
        A.call("tb_fill_random", d.data_ptr(), n, 7, 1000, dist, p0, p1, None)
        torch.cuda.synchronize()
        h = np.zeros(n)
        (O.fill_uniform if dist == 0 else O.fill_normal)(h, 7, 1000, p0, p1)
        np.testing.assert_allclose(d.cpu().numpy(), h, rtol=1e-12, atol=1e-14)
