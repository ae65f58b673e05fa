"""GPU test of tb_block_multiply_int8_noalloc, the split-INT8 block multiply for callers
that cannot allocate device memory (their memory already belongs to other allocators,
or they must avoid the synchronisation a cudaMalloc / cudaFree can cause): it keeps its
scratch in a fixed 64 MiB device array instead of allocating.

Calls in a row, on different block shapes and digit counts, must each match both the
oracle's block_multiply (the reference's compiled kernel where it was built) and the
allocating tb_block_multiply in TB_MODE_INT8, within the split-INT8 tolerance of the
other tests (max |diff| <= 1e-11 * max |product|), so nothing one call leaves in the
shared array leaks into the next.  Kept in its own file that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tamm_b200 import _capi as A

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

INT8_TOL = 1e-11


def _i64(v):
    return np.asarray(list(v) or [0], dtype=np.int64)


def _i32(v):
    return np.asarray(list(v) or [0], dtype=np.int32)


def _case(shape, labels, seed):
    cl, al, bl = labels
    lab = {c: -ord(c) for c in "abcdijk"}
    a = np.zeros([shape[c] for c in al])
    b = np.zeros([shape[c] for c in bl])
    c0 = np.zeros([shape[c] for c in cl])
    O.fill_uniform(a.reshape(-1), seed)
    O.fill_normal(b.reshape(-1), seed + 1, 0, 0.0, 1e-2)
    O.fill_uniform(c0.reshape(-1), seed + 2)
    return a, b, c0, [lab[x] for x in al], [lab[x] for x in bl], [lab[x] for x in cl]


def _args(a, al, b, bl, c0, cl):
    da = torch.from_numpy(a.reshape(-1).copy()).cuda()
    db = torch.from_numpy(b.reshape(-1).copy()).cuda()
    dc = torch.from_numpy(c0.reshape(-1).copy()).cuda()
    keep = [_i64(a.shape), _i32(al), _i64(b.shape), _i32(bl), _i64(c0.shape), _i32(cl)]
    return (da, db, dc), keep


def _allocating(alpha, a, al, b, bl, c0, cl):
    (da, db, dc), k = _args(a, al, b, bl, c0, cl)
    A.call("tb_block_multiply", alpha, da.data_ptr(), k[0].ctypes.data_as(A.i64p), k[1].ctypes.data_as(A.ip),
           a.ndim, db.data_ptr(), k[2].ctypes.data_as(A.i64p), k[3].ctypes.data_as(A.ip), b.ndim, 1.0,
           dc.data_ptr(), k[4].ctypes.data_as(A.i64p), k[5].ctypes.data_as(A.ip), c0.ndim, 0, A.TB_MODE_INT8,
           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return dc.cpu().numpy().reshape(c0.shape)


def _no_alloc(alpha, a, al, b, bl, c0, cl, nslices=0):
    (da, db, dc), k = _args(a, al, b, bl, c0, cl)
    A.call("tb_block_multiply_int8_noalloc", alpha, da.data_ptr(), k[0].ctypes.data_as(A.i64p),
           k[1].ctypes.data_as(A.ip), a.ndim, db.data_ptr(), k[2].ctypes.data_as(A.i64p),
           k[3].ctypes.data_as(A.ip), b.ndim, dc.data_ptr(), k[4].ctypes.data_as(A.i64p),
           k[5].ctypes.data_as(A.ip), c0.ndim, nslices, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return dc.cpu().numpy().reshape(c0.shape)


def _oracle(alpha, a, al, b, bl, c0, cl):
    c = c0.copy()
    assert O.block_multiply(alpha, a, al, b, bl, 1.0, c, cl, 0, impl="ref" if O.ref() is not None else "port") == 0
    return c


def test_no_alloc_matches_oracle_and_allocating_entry_point():
    cases = [
        # ladder-shaped tile pair; C's last mode a column label (transposed epilogue)
        (dict(a=24, b=31, c=29, d=37, i=20, j=20), ("abij", "abcd", "cdij"), 41, 0),
        # permuted labels, C's last mode a row label
        (dict(a=13, b=9, c=7, d=5, i=3, j=11), ("ijab", "cadb", "jdci"), 42, 0),
        # eight digits: the 64-wide output tiles
        (dict(a=40, b=7, c=33, d=3, i=6, j=17), ("abij", "acbd", "cdji"), 43, 8),
    ]
    for shape, labels, seed, ns in cases:  # calls in a row on the shared scratch
        a, b, c0, al, bl, cl = _case(shape, labels, seed)
        ref = _oracle(0.75, a, al, b, bl, c0, cl)
        want = _allocating(0.75, a, al, b, bl, c0, cl)
        got = _no_alloc(0.75, a, al, b, bl, c0, cl, ns)
        scale = np.max(np.abs(ref - c0))
        assert np.max(np.abs(got - ref)) <= INT8_TOL * scale, f"case {seed}: vs oracle"
        assert np.max(np.abs(got - want)) <= INT8_TOL * scale, f"case {seed}: vs allocating entry point"


def test_no_alloc_rejects_triples_beyond_the_static_scratch():
    L = A.lib()
    dims = _i64([4096, 4096])
    lab_a, lab_b, lab_c = _i32([-1, -3]), _i32([-3, -2]), _i32([-1, -2])
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.tb_block_multiply_int8_noalloc(1.0, x.data_ptr(), dims.ctypes.data_as(A.i64p), lab_a.ctypes.data_as(A.ip),
                                          2, x.data_ptr(), dims.ctypes.data_as(A.i64p), lab_b.ctypes.data_as(A.ip), 2,
                                          x.data_ptr(), dims.ctypes.data_as(A.i64p), lab_c.ctypes.data_as(A.ip), 2, 0,
                                          None)
    assert rc == A.TB_ERR_INVALID
    assert "64 MiB" in A.last_error()


def test_no_alloc_refuses_a_capturing_stream():
    # the call drains its stream, so under capture it must refuse before enqueuing
    # anything: the capture stays valid and C is left as it was
    a, b, c0, al, bl, cl = _case(dict(a=24, b=31, c=29, d=37, i=20, j=20), ("abij", "abcd", "cdij"), 44)
    (da, db, dc), k = _args(a, al, b, bl, c0, cl)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rc = A.lib().tb_block_multiply_int8_noalloc(
            0.75, da.data_ptr(), k[0].ctypes.data_as(A.i64p), k[1].ctypes.data_as(A.ip), a.ndim, db.data_ptr(),
            k[2].ctypes.data_as(A.i64p), k[3].ctypes.data_as(A.ip), b.ndim, dc.data_ptr(),
            k[4].ctypes.data_as(A.i64p), k[5].ctypes.data_as(A.ip), c0.ndim, 0,
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
        dc.add_(0.0)  # the capture holds one node of its own
    assert rc == A.TB_ERR_INVALID
    assert "cannot be captured" in A.last_error()
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(dc.cpu().numpy().reshape(c0.shape), c0)
    del g
