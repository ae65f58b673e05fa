"""Owner-computes shares on the device: the two halves of a contraction, each run by
a Scheduler restricted to one rank's output blocks (one after the other on one GPU;
no kernel waits on another), sum to the unsharded result bit for bit, and each
half leaves the other rank's blocks untouched."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W
from tamm_b200.tamm import mult_owned

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [tb.Precision.FP64, tb.Precision.INT8])
def test_shares_sum_to_the_contraction(ec, mode):
    lad = W.ladder(4, 13, seed=8, tile_lo=3, tile_hi=6, ec=ec, build_v=True)
    a, b, c, d, i, j = lad.labels
    op = lambda: lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))
    ec.set_precision(mode, 1e-11)
    try:
        lad.sch(lad.r2().assign(0.0))(op()).execute()
        full = lad.r2.read().copy()
        parts = []
        for r in range(2):
            s = tb.Scheduler(ec).set_owner(r, 2)
            s(lad.r2().assign(0.0))(op()).execute()
            parts.append(lad.r2.read().copy())
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert np.array_equal(parts[0] + parts[1], full)
    keys, offs = lad.r2.block_table()
    ends = dict(zip(offs.tolist(), list(offs[1:].tolist()) + [lad.r2.nelems]))
    for r in range(2):
        owned = set(mult_owned(lad.r2(a, b, i, j), lad.v(a, b, c, d), lad.t2(c, d, i, j), r, 2)[0].tolist())
        for off in offs.tolist():
            if off not in owned:
                assert not np.any(parts[r][off:ends[off]])
