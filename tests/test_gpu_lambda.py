"""Lambda tensors (Tensor(tis, Func): blocks on demand) read by contractions.

The integrals v(a,b,c,d) = sum_Q L(Q,a,c) L(Q,b,d) of a spin-blocked ladder are given
three ways: stored (built once by a contraction), as a per-block lambda (a host
function of the block id, as TAMM's LambdaTensorImpl calls it), and as a batch builder
(each batch queued as the same contraction into the batch tensor).  With batch budgets
small enough to force several batches:
  * r2(a,b,i,j) += v(a,b,c,d) t2(c,d,i,j) (first lambda mode an output label): the
    built form is bit-identical to the stored form in FP64 (each output block is
    computed in one batch by the same tasks), the per-block form within 1e-12, and
    split-INT8 within 1e-11 of the oracle (execute_bufacc restatement);
  * g(a,b,i,j) += v(c,d,a,b) t2(c,d,i,j) with v's first mode summed: batches add
    partial sums; within 1e-12 of the oracle;
  * a CUDA graph of the lambda contraction replays bit-identically to the eager run.
"""
import math

import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel_err(x, ref):
    return float(np.max(np.abs(np.asarray(x) - ref))) / max(float(np.max(np.abs(ref))), 1e-300)


@pytest.fixture(scope="module")
def setup(ec):
    lad = W.ladder(4, 13, seed=21, tile_lo=3, tile_hi=6, ec=ec, build_v=False)
    V = lad.V
    Q = 30
    CI = tb.TiledIndexSpace(tb.IndexSpace(Q), 16)
    q = CI.label()
    L = tb.Tensor([CI, V, V], spin_mask=[2, 0, 1]).allocate(ec)
    L.write(np.random.default_rng(4).normal(size=L.nelems) / math.sqrt(Q))
    a, b, c, d = V.labels(4)
    lad.sch(lad.v(a, b, c, d).assign(L(q, a, c) * L(q, b, d))).execute()
    v_host = lad.v.read()
    # dense L over (Q, virtual, virtual) for the per-block host function
    Ld = np.zeros((Q, int(np.sum(V.tile_sizes)), int(np.sum(V.tile_sizes))))
    keys, offs = L.block_table()
    nts = [s.num_tiles for s in L.spaces]
    tofs = [np.concatenate([[0], np.cumsum(s.tile_sizes)]) for s in L.spaces]
    data = L.read()
    for k, off in zip(keys.tolist(), offs.tolist()):
        bid = []
        for n in reversed(nts):
            bid.append(k % n)
            k //= n
        bid = bid[::-1]
        dims = [int(s.tile_sizes[x]) for s, x in zip(L.spaces, bid)]
        sl = tuple(slice(int(tofs[m][bid[m]]), int(tofs[m][bid[m]]) + dims[m]) for m in range(3))
        Ld[sl] = data[off:off + int(np.prod(dims))].reshape(dims)
    return lad, L, Ld, v_host, q


def _oracle(lad, v_host, clab, alab, blab):
    def ot(t):
        return O.BlockTensor([s.tile_sizes for s in t.spaces], [s.tile_spins for s in t.spaces], [0, 0, 1, 1])
    ov, o2, orr = ot(lad.v), ot(lad.t2), ot(lad.r2)
    ov.data[:ov.total] = v_host
    o2.data[:o2.total] = lad.t2_host
    O.mult_bufacc(orr, clab, 1.0, ov, alab, o2, blab, impl="ref" if O.ref() is not None else "port")
    return orr.data[:orr.total].copy()


def _lambdas(lad, L, Ld, q):
    V = lad.V
    vofs = np.concatenate([[0], np.cumsum(V.tile_sizes)])

    def block(bid, dims):
        r = [slice(int(vofs[x]), int(vofs[x]) + dims[m]) for m, x in enumerate(bid)]
        return np.einsum("qac,qbd->abcd", Ld[:, r[0], r[2]], Ld[:, r[1], r[3]])

    def build(batch, first, last, sch):
        ap = batch.spaces[0].label()
        b2, c2, d2 = V.labels(3)
        sch(batch(ap, b2, c2, d2).assign(L(q, ap, c2) * L(q, b2, d2)))

    nbytes = 8 * lad.v.nelems // 3  # at least three batches
    vl = tb.Tensor.lambda_([V, V, V, V], block, spin=(2, 2), batch_bytes=nbytes)
    vb = tb.Tensor.built([V, V, V, V], build, spin=(2, 2), batch_bytes=nbytes)
    return vl, vb


def test_lambda_ladder_output_label(ec, setup):
    lad, L, Ld, v_host, q = setup
    a, b, c, d, i, j = lad.labels
    vl, vb = _lambdas(lad, L, Ld, q)

    def run(v):
        lad.sch(lad.r2().assign(0.0)).execute()
        lad.sch(lad.r2(a, b, i, j).iadd(v(a, b, c, d) * lad.t2(c, d, i, j))).execute(tb.ExecutionHW.GPU, True)
        return lad.r2.read(), lad.sch.op_stats(-1)

    stored, st0 = run(lad.v)
    built, stb = run(vb)
    per_block, stl = run(vl)
    assert np.array_equal(built, stored)
    assert stb["flops"] == st0["flops"] and stl["flops"] == st0["flops"]
    want = _oracle(lad, v_host, [1, 2, 5, 6], [1, 2, 3, 4], [3, 4, 5, 6])
    assert rel_err(stored, want) <= 1e-12 and rel_err(per_block, want) <= 1e-12
    ec.set_precision(tb.Precision.INT8, 1e-11)
    try:
        got8, _ = run(vb)
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert rel_err(got8, want) <= 1e-11


def test_lambda_first_mode_summed(ec, setup):
    lad, L, Ld, v_host, q = setup
    a, b, c, d, i, j = lad.labels
    _, vb = _lambdas(lad, L, Ld, q)
    lad.sch(lad.r2().assign(0.0)).execute()
    lad.sch(lad.r2(a, b, i, j).iadd(vb(c, d, a, b) * lad.t2(c, d, i, j))).execute()
    want = _oracle(lad, v_host, [1, 2, 5, 6], [3, 4, 1, 2], [3, 4, 5, 6])
    assert rel_err(lad.r2.read(), want) <= 1e-12


def test_lambda_graph_replay(ec, setup):
    lad, L, Ld, v_host, q = setup
    a, b, c, d, i, j = lad.labels
    _, vb = _lambdas(lad, L, Ld, q)
    sch = tb.Scheduler(ec)
    sch(lad.r2().assign(0.0))(lad.r2(a, b, i, j).iadd(vb(a, b, c, d) * lad.t2(c, d, i, j))).execute()
    eager = lad.r2.read()
    sch(lad.r2().assign(0.0))(lad.r2(a, b, i, j).iadd(vb(a, b, c, d) * lad.t2(c, d, i, j)))
    g = sch.graph()
    lad.r2.write(np.full(lad.r2.nelems, 5.0))
    g.launch().sync()
    assert np.array_equal(lad.r2.read(), eager)
    del g
