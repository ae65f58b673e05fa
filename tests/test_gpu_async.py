"""Asynchronous host transfers and execution (tb_tensor_write_async / read_async,
tb_sched_execute_async / wait): two buffer sets used in turn, each step writing its
input, contracting and reading its result without waiting, give the same bits as the
synchronous calls."""
import numpy as np
import pytest
import torch

import tamm_b200 as tb
from tamm_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [tb.Precision.FP64, tb.Precision.INT8])
def test_pipelined_steps_match_synchronous(ec, mode):
    lad = W.ladder(4, 13, seed=10, tile_lo=3, tile_hi=6, ec=ec, build_v=True)
    a, b, c, d, i, j = lad.labels
    rng = np.random.default_rng(3)
    inputs = [rng.normal(0, 1e-2, size=lad.t2.nelems) for _ in range(4)]
    ec.set_precision(mode, 1e-11)
    try:
        want = []
        for x in inputs:  # synchronous reference: r2 = v * t2 per step
            lad.t2.write(x)
            lad.sch(lad.r2().assign(0.0))(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute()
            want.append(lad.r2.read().copy())
        t2b = tb.Tensor([lad.V, lad.V, lad.O, lad.O], spin=(2, 2)).allocate(ec)
        r2b = tb.Tensor([lad.V, lad.V, lad.O, lad.O], spin=(2, 2)).allocate(ec)
        bufs = [(lad.t2, lad.r2), (t2b, r2b)]
        pin_in = [torch.from_numpy(x).pin_memory() for x in inputs]
        pin_out = [torch.empty(lad.r2.nelems, dtype=torch.float64).pin_memory() for _ in inputs]
        for k in range(len(inputs)):
            t2x, r2x = bufs[k % 2]
            t2x.write_async(pin_in[k].data_ptr())
            lad.sch(r2x().assign(0.0))(r2x(a, b, i, j).iadd(lad.v(a, b, c, d) * t2x(c, d, i, j))).execute_async()
            r2x.read_async(pin_out[k].data_ptr())
        lad.sch.wait()
    finally:
        ec.set_precision(tb.Precision.FP64)
    for k in range(len(inputs)):
        assert np.array_equal(pin_out[k].numpy(), want[k])
