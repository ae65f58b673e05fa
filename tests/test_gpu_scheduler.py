"""GPU parity of the runtime tier (LabeledTensor / Scheduler API) against the oracle's
MultOp::execute_bufacc restatement driven by the reference's own block kernel, plus
the reference tests' known answers run through the API."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12


def rel_err(x, ref):
    scale = max(float(np.max(np.abs(ref))), 1e-300)
    return float(np.max(np.abs(np.asarray(x) - np.asarray(ref)))) / scale


def impl():
    return "ref" if O.ref() is not None else "port"


def oracle_tensor(t: tb.Tensor, mask=None):
    return O.BlockTensor([s.tile_sizes for s in t.spaces], [s.tile_spins for s in t.spaces], mask)


def test_config1_contraction(ec):
    """Config 1: C(a,b,i,j) += A(a,c,i,k) * B(c,b,k,j), O=10, V=40, tile 10, dense,
    A, B uniform [-1,1] from seed 0, C = 0."""
    sch = tb.Scheduler(ec)
    Otis = tb.TiledIndexSpace(tb.IndexSpace(10), 10)
    Vtis = tb.TiledIndexSpace(tb.IndexSpace(40), 10)
    a, b, c = Vtis.labels(3)
    i, j, k = Otis.labels(3)
    A_ = tb.Tensor([Vtis, Vtis, Otis, Otis])
    B_ = tb.Tensor([Vtis, Vtis, Otis, Otis])
    C_ = tb.Tensor([Vtis, Vtis, Otis, Otis])
    sch.allocate(A_, B_, C_)
    oa, ob, oc = oracle_tensor(A_), oracle_tensor(B_), oracle_tensor(C_)
    O.fill_uniform(oa.data[:oa.total], 0, 0)
    O.fill_uniform(ob.data[:ob.total], 0, oa.total)
    A_.write(oa.data[:oa.total])
    B_.write(ob.data[:ob.total])
    sch(C_(a, b, i, j).assign(0.0))(C_(a, b, i, j).iadd(A_(a, c, i, k) * B_(c, b, k, j))).execute(
        tb.ExecutionHW.GPU)
    O.mult_bufacc(oc, [1, 2, 5, 6], 1.0, oa, [1, 3, 5, 7], ob, [3, 2, 7, 6], impl=impl())
    assert rel_err(C_.read(), oc.data[:oc.total]) <= FP64_RTOL
    sch.deallocate(A_, B_, C_)


def spin_ladder(ec, oa=4, va=13, seed=3):
    lad = W.ladder(oa, va, seed=seed, tile_lo=3, tile_hi=6, ec=ec, build_v=False)
    rng = np.random.default_rng(seed)
    vh = rng.uniform(-1, 1, size=lad.v.nelems)
    lad.v.write(vh)
    return lad, vh


def test_spin_ladder_matches_oracle(ec):
    lad, vh = spin_ladder(ec)
    a, b, c, d, i, j = lad.labels
    lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute()
    ov, ot, orr = (oracle_tensor(x, [0, 0, 1, 1]) for x in (lad.v, lad.t2, lad.r2))
    ov.data[:ov.total] = vh
    ot.data[:ot.total] = lad.t2_host
    O.mult_bufacc(orr, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [3, 4, 5, 6], impl=impl())
    assert rel_err(lad.r2.read(), orr.data[:orr.total]) <= FP64_RTOL


def test_permuted_outputs_and_subspace_labels(ec):
    """Output written in a permuted label order and labels on a sub-space (v_alpha)."""
    lad, vh = spin_ladder(ec, seed=5)
    a, b, c, d, i, j = lad.labels
    r2p = tb.Tensor([lad.O, lad.V, lad.V, lad.O], spin_mask=[0, 0, 1, 1]).allocate(ec)
    lad.sch(r2p(j, a, b, i).assign(0.0))(r2p(j, a, b, i).iadd(0.5 * lad.v(b, a, c, d) * lad.t2(d, c, j, i)))
    va = lad.MO("virt_alpha")
    aa, bb, cc, dd = va.labels(4)
    lad.sch(lad.r2(aa, bb, i, j).iadd(lad.v(aa, bb, cc, dd) * lad.t2(cc, dd, i, j))).execute()
    ov, ot, orp, orr = (oracle_tensor(x, [0, 0, 1, 1]) for x in (lad.v, lad.t2, r2p, lad.r2))
    ov.data[:ov.total] = vh
    ot.data[:ot.total] = lad.t2_host
    O.mult_bufacc(orp, [6, 1, 2, 5], 0.5, ov, [2, 1, 3, 4], ot, [4, 3, 6, 5], impl=impl())
    assert rel_err(r2p.read(), orp.data[:orp.total]) <= FP64_RTOL
    vmap = [list(lad.V.root_tiles).index(r) for r in va.root_tiles]
    O.mult_bufacc(orr, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [3, 4, 5, 6],
                  tmaps=([vmap, vmap, None, None], [vmap] * 4, [vmap, vmap, None, None]), impl=impl())
    assert rel_err(lad.r2.read(), orr.data[:orr.total]) <= FP64_RTOL


def test_known_answer_mult_ops_norm(ec):
    """Test_Mult_Ops.cpp:176-204 through the API: |C| == 2.625e8 within 1e-9."""
    sch = tb.Scheduler(ec)
    tis = tb.TiledIndexSpace(tb.IndexSpace(50), 20)
    i, j, k, l, m, o = tis.labels(6)
    A_ = tb.Tensor([i, j, m, o])
    B_ = tb.Tensor([m, o, k, l])
    C_ = tb.Tensor([i, j, k, l])
    sch.allocate(A_, B_, C_)
    sch(A_().assign(21.0))(B_().assign(2.0))(C_().assign(0.0)).execute()
    sch(C_(j, i, k, l).iadd(A_(i, j, m, o) * B_(m, o, k, l))).execute(tb.ExecutionHW.GPU)
    assert abs(C_.norm() - 2.625e8) <= 1e-9 * 2.625e8
    sch.deallocate(A_, B_, C_)


def test_known_answer_ops(ec):
    """Test_Ops.cpp:1396-1555: constant-input 3-D / 4-D mults with batch labels."""
    sch = tb.Scheduler(ec)
    IS = tb.IndexSpace(10, named={"nr1": [(0, 5)], "nr2": [(5, 10)]})
    TIS = tb.TiledIndexSpace(IS, 1)
    i, j, k, l, m = TIS.labels(5)
    T1, T2, T3 = (tb.Tensor([TIS] * 3) for _ in range(3))
    sch.allocate(T1, T2, T3)
    sch(T1().assign(2))(T2().assign(3))(T3().assign(4))(T1(i, j, k).iadd(1.7 * T2(j, l, i) * T3(l, i, k))).execute()
    assert np.max(np.abs(T1.read() - (2 + 1.7 * 3 * 4 * 10))) < 1e-10
    S1, S2, S3 = (tb.Tensor([TIS] * 4) for _ in range(3))
    sch.allocate(S1, S2, S3)
    sch(S1().assign(2))(S2().assign(3))(S3().assign(4))
    sch(S1(i, j, k, l).iadd(1.7 * S2(j, l, k, m) * S3(l, i, k, m))).execute()
    assert np.max(np.abs(S1.read() - (2 + 1.7 * 3 * 4 * 10))) < 1e-10
    s0 = tb.Tensor([])
    sch.allocate(s0)
    sch(s0().assign(4))(T1().assign(2))(T1().iadd(6.9 * T2() * s0())).execute()
    assert np.max(np.abs(T1.read() - (2 + 6.9 * 3 * 4))) < 1e-10


def test_addop_setop_match_oracle(ec):
    lad, vh = spin_ladder(ec, seed=9)
    a, b, c, d, i, j = lad.labels
    x = tb.Tensor([lad.V, lad.V, lad.O, lad.O], spin=(2, 2)).allocate(ec)
    lad.sch(x().assign(1.5))(x(a, b, i, j).iadd(-2.0 * lad.t2(b, a, j, i))).execute()
    ot = oracle_tensor(lad.t2, [0, 0, 1, 1])
    ox = oracle_tensor(x, [0, 0, 1, 1])
    ot.data[:ot.total] = lad.t2_host
    ox.set(1.5)
    for bid in ox.blockids():
        src = ot.block((bid[1], bid[0], bid[3], bid[2]))
        dst = ox.block(bid)
        assert O.assign(dst, [1, 2, 5, 6], -2.0, np.ascontiguousarray(src), [2, 1, 6, 5], 0) == 0
    np.testing.assert_allclose(x.read(), ox.data[:ox.total], rtol=1e-15, atol=1e-15)
    # flat AddOp (same labels, same layout) and assignment
    lad.sch(x(a, b, i, j).assign(3.0 * lad.t2(a, b, i, j))).execute()
    np.testing.assert_allclose(x.read(), 3.0 * lad.t2_host, rtol=1e-15, atol=0)


def test_block_get_put_add(ec):
    lad, vh = spin_ladder(ec, seed=2)
    ot = oracle_tensor(lad.t2, [0, 0, 1, 1])
    ot.data[:ot.total] = lad.t2_host
    for bid in ot.blockids()[:5]:
        np.testing.assert_array_equal(lad.t2.get(bid), ot.block(bid))
    bid = ot.blockids()[0]
    blk = np.full(lad.t2.block_dims(bid), 0.25)
    lad.t2.put(bid, blk)
    lad.t2.add(bid, blk)
    np.testing.assert_array_equal(lad.t2.get(bid), 0.5)
    # a non-admitted block reads as zeros and ignores writes (tensor_impl.hpp:324-329)
    nz = (0, lad.V.num_tiles - 1, 0, 0)
    assert not lad.t2.is_non_zero(nz)
    assert np.all(lad.t2.get(nz) == 0)


def test_unallocated_tensor_is_a_state_error(ec):
    sch = tb.Scheduler(ec)
    T = tb.TiledIndexSpace(tb.IndexSpace(8), 4)
    x = tb.Tensor([T, T])
    with pytest.raises(tb.TambError) as e:
        sch(x().assign(1.0)).execute()
    assert e.value.code == 7
