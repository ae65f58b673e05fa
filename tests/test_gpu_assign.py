"""Assignments C = alpha * A * B (queued as Set(0) + Mult, as TAMM's
MultOp::canonicalize does, multop.hpp:255-269).  On one rank the scheduler runs the
pair fused: the contraction kernel (FP64, or the split kernels' epilogue) stores its
result without reading C, and the fill touches only the output blocks that receive no
task.  The output is written both with its last mode a column label of the tile (the
split epilogue's transposed stores) and a row label (one row per thread).

C(a,b) is dense while A(a,c) and B(c,b) conserve spin, so C's mixed-spin blocks have
no task and must still come out zero; C starts out holding garbage.  Checked in FP64
(1e-12), split-INT8 (1e-11) and BF16x3 (5e-5) against numpy, relative to max |C|,
and C = C * B (C read as an operand, which must see the fill first) gives zeros."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dense(t):
    sizes = [int(np.sum(s.tile_sizes)) for s in t.spaces]
    tofs = [np.concatenate([[0], np.cumsum(s.tile_sizes)]) for s in t.spaces]
    nts = [s.num_tiles for s in t.spaces]
    out = np.zeros(sizes)
    keys, offs = t.block_table()
    data = t.read()
    for key, off in zip(keys.tolist(), offs.tolist()):
        bid = []
        for n in reversed(nts):
            bid.append(key % n)
            key //= n
        bid = bid[::-1]
        dims = [int(s.tile_sizes[x]) for s, x in zip(t.spaces, bid)]
        sl = tuple(slice(int(tofs[m][bid[m]]), int(tofs[m][bid[m]]) + dims[m]) for m in range(len(dims)))
        out[sl] = data[off:off + int(np.prod(dims))].reshape(dims)
    return out


@pytest.fixture(scope="module")
def spaces():
    rng = np.random.default_rng(11)
    virt = W.random_tiles(70, 12, 30, rng)
    MO = W.mo_tiled(6, 70, [6], virt)
    return MO("virt")


@pytest.mark.parametrize("transposed", [False, True])
@pytest.mark.parametrize("mode,tol", [(tb.Precision.FP64, 1e-12), (tb.Precision.INT8, 1e-11),
                                      (tb.Precision.BF16X3, 5e-5)])
def test_assign_stores_and_zeroes_blocks_without_tasks(ec, spaces, mode, tol, transposed):
    V = spaces
    rng = np.random.default_rng(5)
    A = tb.Tensor([V, V], spin=(1, 1)).allocate(ec)
    B = tb.Tensor([V, V], spin=(1, 1)).allocate(ec)
    C = tb.Tensor([V, V]).allocate(ec)
    A.write(rng.uniform(-1, 1, size=A.nelems))
    B.write(rng.normal(0, 1e-2, size=B.nelems))
    C.write(np.full(C.nelems, 7.0))
    want = -0.5 * _dense(A) @ _dense(B)
    if transposed:
        want = want.T
    a, b, c = V.labels(3)
    ec.set_precision(mode, 1e-11)
    try:
        sch = tb.Scheduler(ec)
        for _ in range(2):  # the second run reuses the scheduler's cached plan and work list
            C.write(np.full(C.nelems, 7.0))
            lhs = C(b, a) if transposed else C(a, b)
            sch(lhs.assign(-0.5 * A(a, c) * B(c, b))).execute(tb.ExecutionHW.GPU)
            got = _dense(C)
            assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want))
            assert np.all(got[want == 0.0] == 0.0)  # mixed-spin blocks: no task, zero fill
    finally:
        ec.set_precision(tb.Precision.FP64)


def test_assign_reading_its_own_output_sees_the_fill(ec, spaces):
    V = spaces
    rng = np.random.default_rng(6)
    B = tb.Tensor([V, V]).allocate(ec)
    C = tb.Tensor([V, V]).allocate(ec)
    B.write(rng.normal(size=B.nelems))
    C.write(rng.normal(size=C.nelems))
    a, b, c = V.labels(3)
    tb.Scheduler(ec)(C(a, b).assign(C(a, c) * B(c, b))).execute(tb.ExecutionHW.GPU)
    assert np.all(C.read() == 0.0)
