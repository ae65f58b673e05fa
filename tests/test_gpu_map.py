"""MapOp family on the device (tb_sched_map): exact_copy, apply_ewise_ip and the
apply_ewise element functions, against numpy over the same packed blocks.

Cases: every element function in place on a spin-blocked tensor; out of place into a
tensor without spin symmetry, whose blocks that the spin-blocked source does not store
must come out zero (TAMM's get of a non-admitted block); and a map restricted to a
sub-space label (virt_alpha), which must leave the other blocks untouched.  Bars: 0 for
copy / set / abs / square / scale (exact), 4 ulps relative for the library functions."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W

pytestmark = pytest.mark.gpu

FNS = [(tb.Map.COPY, 0.0, lambda x, p: x), (tb.Map.SCALE, -2.5, lambda x, p: p * x),
       (tb.Map.SET, 3.25, lambda x, p: np.full_like(x, p)), (tb.Map.SQUARE, 0.0, lambda x, p: x * x),
       (tb.Map.SQRT, 0.0, lambda x, p: np.sqrt(x)), (tb.Map.LOG, 0.0, lambda x, p: np.log(x)),
       (tb.Map.LOG10, 0.0, lambda x, p: np.log10(x)), (tb.Map.INVERSE, 0.0, lambda x, p: 1.0 / x),
       (tb.Map.POW, 1.7, lambda x, p: np.power(x, p)), (tb.Map.ABS, 0.0, lambda x, p: np.abs(x))]


def _space():
    return W.mo_tiled(3, 7, [3], [3, 4])


@pytest.mark.parametrize("fn,p,ref", FNS)
def test_map_in_place(ec, fn, p, ref):
    MO = _space()
    V, O_ = MO("virt"), MO("occ")
    t = tb.Tensor([V, V, O_, O_], spin=(2, 2)).allocate(ec)
    x = np.random.default_rng(fn).uniform(0.1, 2.0, size=t.nelems)
    t.write(x)
    a, b = V.labels(2)
    i, j = O_.labels(2)
    if fn == tb.Map.SCALE:
        tb.apply_ewise_ip(t(a, b, i, j), fn, p)
    else:
        tb.Scheduler(ec).map(t(a, b, i, j), t(a, b, i, j), fn, p).execute()
    got, want = t.read(), ref(x, p)
    exact = fn in (tb.Map.COPY, tb.Map.SCALE, tb.Map.SET, tb.Map.SQUARE, tb.Map.ABS, tb.Map.SQRT, tb.Map.INVERSE)
    tol = 0.0 if exact else 4 * np.finfo(float).eps
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) <= tol


def test_exact_copy_into_dense_and_subspace_map(ec):
    MO = _space()
    V, O_ = MO("virt"), MO("occ")
    src = tb.Tensor([V, V, O_, O_], spin=(2, 2)).allocate(ec)
    dst = tb.Tensor([V, V, O_, O_]).allocate(ec)  # no spin symmetry: every block stored
    x = np.random.default_rng(5).normal(size=src.nelems)
    src.write(x)
    dst.write(np.full(dst.nelems, 7.0))
    a, b = V.labels(2)
    i, j = O_.labels(2)
    sch = tb.Scheduler(ec)
    sch.exact_copy(dst(a, b, i, j), src(a, b, i, j)).execute()
    got = dst.read()
    keys, offs = dst.block_table()
    nts = [s.num_tiles for s in dst.spaces]
    for k, off in zip(keys.tolist(), offs.tolist()):
        bid = []
        for n in reversed(nts):
            bid.append(k % n)
            k //= n
        bid = bid[::-1]
        n = int(np.prod(dst.block_dims(bid)))
        want = src.get(bid).reshape(-1)  # zeros where src does not store the block
        assert np.array_equal(got[off:off + n], want)
    # scale only the (alpha, alpha) virtual blocks in place; the others stay as they were
    va = MO("virt_alpha")
    aa, bb = va.labels(2)
    before = dst.read()
    sch.map(dst(aa, bb, i, j), dst(aa, bb, i, j), tb.Map.SCALE, 2.0).execute()
    after = dst.read()
    V_alpha = {int(r) for r in va.root_tiles}
    for k, off in zip(keys.tolist(), offs.tolist()):
        bid = []
        for n in reversed(nts):
            bid.append(k % n)
            k //= n
        bid = bid[::-1]
        n = int(np.prod(dst.block_dims(bid)))
        inside = int(V.root_tiles[bid[0]]) in V_alpha and int(V.root_tiles[bid[1]]) in V_alpha
        want = 2.0 * before[off:off + n] if inside else before[off:off + n]
        assert np.array_equal(after[off:off + n], want)
