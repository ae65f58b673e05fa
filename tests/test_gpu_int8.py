"""GPU parity of the split-INT8 (Ozaki) contraction against the FP64 oracle.

Error metric (stated in every assertion): max |int8 - oracle| / max |oracle| over the
output block(s).  Bar: <= 1e-11 at the default error target; the forced slice counts
3..8 must show the expected 2^-8 per slice decay."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import _capi as A
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

from test_gpu_kernels import gpu_block_multiply, rel_err  # noqa: E402

INT8_TOL = 1e-11


@pytest.mark.parametrize("labels,shape", [
    (("abij", "abcd", "cdij"), dict(a=24, b=31, c=29, d=37, i=20, j=20)),
    (("abij", "acid", "cbdj"), dict(a=10, b=10, c=10, d=10, i=10, j=10)),
    (("ijab", "cadb", "jdci"), dict(a=13, b=9, c=7, d=5, i=3, j=11)),
    (("abij", "abcd", "cdij"), dict(a=1, b=1, c=1, d=1, i=1, j=1)),
    (("abij", "abcd", "cdij"), dict(a=48, b=48, c=48, d=48, i=20, j=20)),
    (("ab", "ak", "kb"), dict(a=300, b=170, k=700)),
    # both operands with contiguous rows (staged split of A and B): odd K (K = 1369),
    # short rows, one-element rows
    (("abij", "abcd", "ijcd"), dict(a=13, b=11, c=37, d=37, i=7, j=5)),
    (("abij", "abcd", "ijcd"), dict(a=9, b=17, c=5, d=7, i=6, j=3)),
    (("abij", "abcd", "ijcd"), dict(a=19, b=3, c=1, d=1, i=5, j=9)),
    # long contiguous rows: K = 4209 (one warp group's two stages fill shared memory),
    # a ragged last element and rows of padding in the last tile
    (("abij", "abcd", "ijcd"), dict(a=11, b=13, c=61, d=69, i=3, j=7)),
])
def test_int8_block_multiply(labels, shape):
    cl, al, bl = labels
    lab = {c: -ord(c) for c in "abcdijk"}
    A_ = np.zeros([shape[c] for c in al])
    B_ = np.zeros([shape[c] for c in bl])
    C0 = np.zeros([shape[c] for c in cl])
    O.fill_uniform(A_.reshape(-1), 31)
    O.fill_normal(B_.reshape(-1), 32, 0, 0.0, 1e-2)
    O.fill_uniform(C0.reshape(-1), 33)
    want = np.array(C0, copy=True)
    assert O.block_multiply(0.75, A_, [lab[c] for c in al], B_, [lab[c] for c in bl], 1.0, want,
                            [lab[c] for c in cl], 0) == 0
    got = gpu_block_multiply(0.75, A_, [lab[c] for c in al], B_, [lab[c] for c in bl], 1.0, C0,
                             [lab[c] for c in cl], 0, mode=A.TB_MODE_INT8)
    assert rel_err(got - C0, want - C0) <= INT8_TOL


def test_int8_assign_and_zero_blocks():
    lab = {c: -ord(c) for c in "abcdij"}
    shape = dict(a=7, b=9, c=11, d=5, i=4, j=6)
    A_ = np.zeros([shape[c] for c in "abcd"])
    B_ = np.zeros([shape[c] for c in "cdij"])
    O.fill_uniform(B_.reshape(-1), 2)
    C0 = np.full([shape[c] for c in "abij"], 3.0)
    got = gpu_block_multiply(1.0, A_, [lab[c] for c in "abcd"], B_, [lab[c] for c in "cdij"], 1.0, C0,
                             [lab[c] for c in "abij"], 1, mode=A.TB_MODE_INT8)
    assert np.all(got == 0.0)  # zero A: exact zero, assign overwrote C


def _ladder_case(ec, seed=3):
    lad = W.ladder(4, 13, seed=seed, tile_lo=3, tile_hi=6, ec=ec, build_v=False)
    rng = np.random.default_rng(seed)
    vh = rng.normal(0.0, 1e-2, size=lad.v.nelems) * np.exp(rng.uniform(-3, 3, size=lad.v.nelems))
    lad.v.write(vh)
    ov, ot, orr = (O.BlockTensor([s.tile_sizes for s in x.spaces], [s.tile_spins for s in x.spaces], [0, 0, 1, 1])
                   for x in (lad.v, lad.t2, lad.r2))
    ov.data[:ov.total] = vh
    ot.data[:ot.total] = lad.t2_host
    O.mult_bufacc(orr, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [3, 4, 5, 6])
    return lad, orr.data[:orr.total].copy()


def test_int8_spin_ladder_default_target(ec):
    lad, want = _ladder_case(ec)
    a, b, c, d, i, j = lad.labels
    ec.set_precision(tb.Precision.INT8, 1e-11)
    try:
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute()
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert rel_err(lad.r2.read(), want) <= INT8_TOL


def test_int8_cholesky_ladder_with_zero_spin_blocks(ec):
    """v built on the device from Cholesky vectors (its (ab|ba)-type spin blocks are
    exactly zero, its off-diagonal blocks damped): per-task digit counts must keep the
    1e-11 bar and give zero blocks a single digit."""
    lad = W.ladder(4, 13, seed=6, tile_lo=3, tile_hi=6, ec=ec, build_v=True)
    a, b, c, d, i, j = lad.labels
    vh = lad.v.read().copy()
    ov, ot, orr = (O.BlockTensor([s.tile_sizes for s in x.spaces], [s.tile_spins for s in x.spaces], [0, 0, 1, 1])
                   for x in (lad.v, lad.t2, lad.r2))
    ov.data[:ov.total] = vh
    ot.data[:ot.total] = lad.t2_host
    O.mult_bufacc(orr, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [3, 4, 5, 6])
    zero_blocks = [bid for bid in ov.blockids() if not np.any(ov.block(bid))]
    assert zero_blocks  # the spin-flip blocks of a Cholesky-built v
    ec.set_precision(tb.Precision.INT8, 1e-11)
    try:
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute(profile=True)
        st = lad.sch.op_stats(-1)
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert rel_err(lad.r2.read(), orr.data[:orr.total]) <= INT8_TOL
    assert st["slices_min"] == 1 and st["slices_max"] == 6  # 1e-11 needs 6 digits


def test_int8_slice_count_controls_error(ec):
    lad, want = _ladder_case(ec, seed=4)
    a, b, c, d, i, j = lad.labels
    errs = {}
    for s in (3, 4, 5, 6, 7, 8):
        ec.set_precision(tb.Precision.INT8, 1e-11, s)
        lad.sch(lad.r2().assign(0.0))(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute()
        errs[s] = rel_err(lad.r2.read(), want)
    ec.set_precision(tb.Precision.FP64)
    assert errs[3] < 1e-4
    for s in (3, 4, 5):
        assert errs[s + 1] < errs[s] / 50, errs  # ~2^-8 per added slice
    assert errs[6] <= INT8_TOL and errs[8] <= 1e-14, errs
