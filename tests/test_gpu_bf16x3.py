"""GPU checks of the BF16x3 mode (TB_MODE_BF16X3) against the FP64 oracle.

Each operand row is scaled by a power of two and cut into two bf16 pieces
(hi + lo); the products hi*hi, hi*lo and lo*hi run on the tcgen05 tensor cores with
FP32 accumulation and are recombined in FP64.  The dropped lo*lo term and the FP32
accumulation bound the error near 2^-18 of the row-max x col-max products, so the
mode is FP32-class.  Error metric: max |bf16x3 - oracle| / max |oracle| over the
output; bar BF16X3_TOL, with the measured values in the parametrised cases far
below it and far above the split-INT8 errors (which would mean the mode silently ran
another path)."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import _capi as A
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

from test_gpu_kernels import gpu_block_multiply, rel_err  # noqa: E402

BF16X3_TOL = 5e-5  # measured 4.0e-6 .. 7.4e-6 on the cases below


@pytest.mark.parametrize("labels,shape", [
    (("abij", "abcd", "cdij"), dict(a=24, b=31, c=29, d=37, i=20, j=20)),
    (("abij", "acid", "cbdj"), dict(a=10, b=10, c=10, d=10, i=10, j=10)),
    (("ijab", "cadb", "jdci"), dict(a=13, b=9, c=7, d=5, i=3, j=11)),
    (("abij", "abcd", "cdij"), dict(a=48, b=48, c=48, d=48, i=20, j=20)),
    (("ab", "ak", "kb"), dict(a=300, b=170, k=700)),
])
def test_bf16x3_block_multiply(labels, shape):
    cl, al, bl = labels
    lab = {c: -ord(c) for c in "abcdijk"}
    A_ = np.zeros([shape[c] for c in al])
    B_ = np.zeros([shape[c] for c in bl])
    C0 = np.zeros([shape[c] for c in cl])
    O.fill_uniform(A_.reshape(-1), 41)
    O.fill_normal(B_.reshape(-1), 42, 0, 0.0, 1e-2)
    O.fill_uniform(C0.reshape(-1), 43)
    want = np.array(C0, copy=True)
    assert O.block_multiply(0.75, A_, [lab[c] for c in al], B_, [lab[c] for c in bl], 1.0, want,
                            [lab[c] for c in cl], 0) == 0
    got = gpu_block_multiply(0.75, A_, [lab[c] for c in al], B_, [lab[c] for c in bl], 1.0, C0,
                             [lab[c] for c in cl], 0, mode=A.TB_MODE_BF16X3)
    err = rel_err(got - C0, want - C0)
    print(f"bf16x3 {labels} rel err {err:.3e}")
    assert 1e-12 < err <= BF16X3_TOL


def test_bf16x3_spin_ladder(ec):
    lad = W.ladder(4, 13, seed=7, tile_lo=3, tile_hi=6, ec=ec, build_v=True)
    a, b, c, d, i, j = lad.labels
    ov, ot, orr = (O.BlockTensor([s.tile_sizes for s in x.spaces], [s.tile_spins for s in x.spaces], [0, 0, 1, 1])
                   for x in (lad.v, lad.t2, lad.r2))
    ov.data[:ov.total] = lad.v.read()
    ot.data[:ot.total] = lad.t2_host
    O.mult_bufacc(orr, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [3, 4, 5, 6])
    ec.set_precision(tb.Precision.BF16X3)
    try:
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute(profile=True)
        st = lad.sch.op_stats(-1)
    finally:
        ec.set_precision(tb.Precision.FP64)
    err = rel_err(lad.r2.read(), orr.data[:orr.total])
    print(f"bf16x3 spin ladder rel err {err:.3e}")
    assert 1e-12 < err <= BF16X3_TOL
    assert st["mode"] == tb.Precision.BF16X3 and st["slices_min"] == 2 and st["slices_max"] == 2
