"""Multi-factor products on the device (tb_sched_mult_n: OpMin's tree run as binary
contractions through scheduler-owned intermediates) against numpy's einsum on the
dense arrays: a matrix chain, a four-factor coupled-cluster-like term on spin-blocked
tensors (dense reference with the same zero blocks), assignment and update, FP64
within 1e-12 and split-INT8 within 1e-11 of max |result|; queuing the same product
again reuses its intermediates and gives the same bits."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dense(t):
    sizes = [int(np.sum(s.tile_sizes)) for s in t.spaces]
    out = np.zeros(sizes)
    keys, offs = t.block_table()
    data = t.read()
    nts = [s.num_tiles for s in t.spaces]
    tofs = [np.concatenate([[0], np.cumsum(s.tile_sizes)]) for s in t.spaces]
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


def _rel(x, y):
    return float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))


@pytest.mark.parametrize("mode,tol", [(tb.Precision.FP64, 1e-12), (tb.Precision.INT8, 1e-11)])
def test_matrix_chain(ec, mode, tol):
    I, K, L, J = (tb.TiledIndexSpace(tb.IndexSpace(n), t) for n, t in ((7, 4), (90, 30), (110, 40), (5, 5)))
    i, k, l, j = I.label(), K.label(), L.label(), J.label()
    A_, B_, C_, D_ = (tb.Tensor(sp).allocate(ec) for sp in ([I, K], [K, L], [L, J], [I, J]))
    rng = np.random.default_rng(1)
    for t in (A_, B_, C_, D_):
        t.write(rng.uniform(-1, 1, size=t.nelems))
    d0 = _dense(D_)
    want = d0 + 0.5 * np.einsum("ik,kl,lj->ij", _dense(A_), _dense(B_), _dense(C_))
    ec.set_precision(mode, 1e-11)
    try:
        sch = tb.Scheduler(ec)
        sch(D_(i, j).iadd(0.5 * A_(i, k) * B_(k, l) * C_(l, j))).execute()
        got = _dense(D_)
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert _rel(got - d0, want - d0) <= tol


def test_four_factor_spin_term_and_reuse(ec):
    """r2(a,b,i,j) = t2(a,c,i,k) * v(k,l,c,d) * t2(d,b,l,j) * f(j,j') style chain with
    spin-blocked operands (every factor's stored blocks as TAMM's spin rule admits)."""
    MO = W.mo_tiled(3, 6, [3], [3, 3])
    O_, V = MO("occ"), MO("virt")
    a, b, c, d = V.labels(4)
    i, j, k, l = O_.labels(4)
    t2 = tb.Tensor([V, V, O_, O_], spin=(2, 2)).allocate(ec)
    v = tb.Tensor([O_, O_, V, V], spin=(2, 2)).allocate(ec)
    f = tb.Tensor([O_, O_], spin=(1, 1)).allocate(ec)
    r2 = tb.Tensor([V, V, O_, O_], spin=(2, 2)).allocate(ec)
    rng = np.random.default_rng(2)
    for t in (t2, v, f):
        t.write(rng.normal(size=t.nelems))
    T2, Vd, F = _dense(t2), _dense(v), _dense(f)
    want = np.einsum("acik,klcd,dblm,mj->abij", T2, Vd, T2, F)
    (m,) = O_.labels(1)
    sch = tb.Scheduler(ec)
    sch(r2(a, b, i, j).assign(t2(a, c, i, k) * v(k, l, c, d) * t2(d, b, l, m) * f(m, j))).execute()
    got = _dense(r2)
    # every factor conserves spin, so the product vanishes outside r2's stored blocks
    assert _rel(got, want) <= 1e-12
    assert np.count_nonzero(got) > 0
    # queued again: the scheduler's intermediates are reused, the bits are the same
    sch(r2(a, b, i, j).assign(t2(a, c, i, k) * v(k, l, c, d) * t2(d, b, l, m) * f(m, j))).execute()
    assert np.array_equal(_dense(r2), got)
