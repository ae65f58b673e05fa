"""Dependent index spaces on the device.

* Known answers of TAMM's Test_DependentSpace.cpp (test_dependent_space_with_T, full
  dependency of a on the tiles of i, 10 indices, tiles of 3): SetOp 42 everywhere;
  AddOp T1 = 4, T2 = 42, T1 += 3 * T2 -> 130; T1 = 4, T1 -= T2 -> -38; MultOp with a
  scalar factor (T1 += T2 * T3: 8 * 4 = 32) and the full reduction
  T3 += 1.5 * T1 * T2 = 4 + 1.5 * 100 * 9 * 8.
* A DLPNO-like contraction over a PNO space that depends on LMO pairs, with pairs and
  PNO ranges drawn at random, R(i,j,a(i,j),b(i,j)) += t2(i,j,a(i,j),e(i,j)) F(e,b),
  against numpy on dense arrays where the missing blocks are zero: FP64 within 1e-12.
"""
import numpy as np
import pytest

import tamm_b200 as tb
from test_dependent import _pno

pytestmark = pytest.mark.gpu


def _dep_space():
    IS = tb.IndexSpace(10)
    T_IS = tb.TiledIndexSpace(IS, 3)
    REF = tb.TiledIndexSpace(tb.IndexSpace(10), 3)
    DIS = tb.TiledIndexSpace.dependent(REF, [T_IS], {(t,): REF("all") for t in range(T_IS.num_tiles)})
    return T_IS, DIS


def test_dependent_space_known_answers(ec):
    T_IS, DIS = _dep_space()
    (a,) = DIS.labels(1)
    (i,) = T_IS.labels(1)
    T1, T2 = tb.Tensor([a(i), i]).allocate(ec), tb.Tensor([a(i), i]).allocate(ec)
    T3 = tb.Tensor([]).allocate(ec)
    sch = tb.Scheduler(ec)
    sch(T1().assign(42.0)).execute()
    assert T1.nelems == 100 and np.all(T1.read() == 42.0)
    sch(T1().assign(4.0))(T2().assign(42.0))(T1(a, i).iadd(3.0 * T2(a, i))).execute()
    assert np.all(T1.read() == 130.0)
    sch(T1().assign(4.0))(T1().isub(T2())).execute()
    assert np.all(T1.read() == -38.0)
    sch(T1().assign(0.0))(T2().assign(8.0))(T3().assign(4.0))(T1().iadd(T2() * T3())).execute()
    assert np.all(T1.read() == 32.0)
    sch(T1().assign(9.0))(T2().assign(8.0))(T3().assign(4.0))(T3().iadd(1.5 * T1() * T2())).execute()
    assert abs(float(T3.read()[0]) - (4 + 1.5 * 100 * 9 * 8)) <= 1e-12 * 10804


def _dense(t, sizes):
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


def test_dlpno_like_contraction(ec):
    LMO, REF, PNO, allowed = _pno(seed=5, n_lmo=9, lmo_tile=2, n_pno=23, pno_tile=4)
    i, j = LMO.labels(2)
    a, b, e = PNO.labels(3)
    t2 = tb.Tensor([i, j, a(i, j), e(i, j)]).allocate(ec)
    R = tb.Tensor([i, j, a(i, j), b(i, j)]).allocate(ec)
    F = tb.Tensor([REF, REF]).allocate(ec)
    rng = np.random.default_rng(8)
    t2.write(rng.normal(size=t2.nelems))
    F.write(rng.normal(size=F.nelems))
    R.write(rng.normal(size=R.nelems))
    sizes = [9, 9, 23, 23]
    T2d, R0 = _dense(t2, sizes), _dense(R, sizes)
    Fd = _dense(F, [23, 23])
    tb.Scheduler(ec)(R(i, j, a, b).iadd(0.5 * t2(i, j, a, e) * F(e, b))).execute()
    got = _dense(R, sizes)
    # the product restricted to the blocks R stores (a and b listed for the pair)
    mask = (_dense_mask(R, sizes) > 0)
    want = R0 + 0.5 * np.einsum("ijae,eb->ijab", T2d, Fd) * mask
    assert float(np.max(np.abs(got - want))) <= 1e-12 * float(np.max(np.abs(want - R0)))


def _dense_mask(t, sizes):
    keys, _ = t.block_table()
    out = np.zeros(sizes)
    nts = [s.num_tiles for s in t.spaces]
    tofs = [np.concatenate([[0], np.cumsum(s.tile_sizes)]) for s in t.spaces]
    for key in keys.tolist():
        bid = []
        for n in reversed(nts):
            bid.append(key % n)
            key //= n
        bid = bid[::-1]
        dims = [int(s.tile_sizes[x]) for s, x in zip(t.spaces, bid)]
        sl = tuple(slice(int(tofs[m][bid[m]]), int(tofs[m][bid[m]]) + dims[m]) for m in range(len(dims)))
        out[sl] = 1.0
    return out
