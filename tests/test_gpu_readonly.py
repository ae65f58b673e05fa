"""Read-only tensors and exactly-zero blocks (tb_tensor_set_read_only).

A spin-blocked ladder r2 += v * t2 whose v has its (alpha beta | beta alpha) and
(beta alpha | alpha beta) blocks exactly zero, as a v built from same-spin Cholesky
vectors has: TAMM's spin rule admits those blocks, so its MultOp multiplies them.
With v marked read-only the contraction skips those tasks.  Checks:
  * FP64 result bit-identical to the unmarked contraction, and within 1e-12 of the
    oracle (the execute_bufacc restatement driving the reference's block kernel);
  * split-INT8 within 1e-11 of the oracle;
  * tb_stats.flops stays the admitted count, flops_run drops by exactly the FLOPs of
    the tasks over zero blocks (counted on the host from the block table);
  * writes to a marked tensor fail with TB_ERR_STATE; clearing the mark allows them.
"""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import _capi as A
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel_err(x, ref):
    return float(np.max(np.abs(np.asarray(x) - ref))) / max(float(np.max(np.abs(ref))), 1e-300)


def _blockid(key, nts):
    out = []
    for n in reversed(nts):
        out.append(key % n)
        key //= n
    return out[::-1]


def _ladder_with_zero_blocks(ec, seed=7):
    lad = W.ladder(4, 13, seed=seed, tile_lo=3, tile_hi=6, ec=ec, build_v=False)
    rng = np.random.default_rng(seed)
    vh = rng.uniform(-1, 1, size=lad.v.nelems)
    keys, offs = lad.v.block_table()
    nts = [s.num_tiles for s in lad.v.spaces]
    zero = []
    for bi, (k, off) in enumerate(zip(keys, offs)):
        bid = _blockid(int(k), nts)
        sp = [lad.v.spaces[m].spin(bid[m]) for m in range(4)]
        if sp[0] != sp[2]:  # (a c) of different spin: the Cholesky factor vanishes
            n = int(np.prod(lad.v.block_dims(bid)))
            vh[off:off + n] = 0.0
            zero.append(tuple(bid))
    # a block of -0.0 entries counts as zero too
    k0 = sorted(zero)[0]
    off0 = int(offs[[tuple(_blockid(int(k), nts)) for k in keys].index(k0)])
    vh[off0:off0 + int(np.prod(lad.v.block_dims(list(k0))))] = -0.0
    lad.v.write(vh)
    return lad, vh, set(zero)


def _oracle(lad, vh):
    def ot(t):
        return O.BlockTensor([s.tile_sizes for s in t.spaces], [s.tile_spins for s in t.spaces], [0, 0, 1, 1])
    ov, o2, orr = ot(lad.v), ot(lad.t2), ot(lad.r2)
    ov.data[:ov.total] = vh
    o2.data[:o2.total] = lad.t2_host
    O.mult_bufacc(orr, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], o2, [3, 4, 5, 6],
                  impl="ref" if O.ref() is not None else "port")
    return orr.data[:orr.total].copy()


def _skipped_flops(lad, zero):
    """FP64 FLOPs of the admitted (a,b,c,d,i,j) tuples whose v block is in `zero`."""
    V, Oc = lad.V, lad.O
    vs = [V.spin(x) for x in range(V.num_tiles)]
    os_ = [Oc.spin(x) for x in range(Oc.num_tiles)]
    vz = [V.tile_size(x) for x in range(V.num_tiles)]
    oz = [Oc.tile_size(x) for x in range(Oc.num_tiles)]
    fl = 0.0
    for (a, b, c, d) in zero:
        for i in range(Oc.num_tiles):
            for j in range(Oc.num_tiles):
                if vs[a] + vs[b] == os_[i] + os_[j]:
                    fl += 2.0 * vz[a] * vz[b] * vz[c] * vz[d] * oz[i] * oz[j]
    return fl


def test_zero_blocks_skipped_fp64_bitwise_and_int8_vs_oracle(ec):
    lad, vh, zero = _ladder_with_zero_blocks(ec)
    assert zero, "the test ladder must have zero blocks"
    a, b, c, d, i, j = lad.labels
    want = _oracle(lad, vh)

    def run(profile=True):
        lad.sch(lad.r2().assign(0.0)).execute()
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute(tb.ExecutionHW.GPU,
                                                                                          profile)
        return lad.r2.read(), lad.sch.op_stats(-1)

    base, st0 = run()
    lad.v.set_read_only(True)
    on, nzb, nze = lad.v.read_only_info()
    assert on and nzb == len(zero)
    fast, st1 = run()
    assert np.array_equal(fast, base), "skipping exactly-zero tasks must not change the FP64 result"
    assert rel_err(fast, want) <= 1e-12
    assert st1["flops"] == st0["flops"] and st0["flops_run"] == st0["flops"]
    skip = _skipped_flops(lad, zero)
    assert skip > 0 and abs((st1["flops"] - st1["flops_run"]) - skip) <= 1e-9 * skip

    ec.set_precision(tb.Precision.INT8, 1e-11)
    try:
        got8, st8 = run()
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert rel_err(got8, want) <= 1e-11
    assert st8["flops_run"] == st1["flops_run"]

    # work lists are cached per read-only marking: clearing the mark runs every task again
    lad.v.set_read_only(False)
    again, st2 = run()
    assert np.array_equal(again, base) and st2["flops_run"] == st2["flops"]


def test_read_only_tensor_rejects_writes(ec):
    lad, vh, _ = _ladder_with_zero_blocks(ec, seed=9)
    a, b, c, d, i, j = lad.labels
    lad.v.set_read_only(True)
    bid = [0, 0, 0, 0]
    with pytest.raises(tb.TambError) as e:
        lad.v.write(vh)
    assert e.value.code == A.TB_ERR_STATE
    with pytest.raises(tb.TambError):
        lad.v.put(bid, np.zeros(int(np.prod(lad.v.block_dims(bid)))))
    with pytest.raises(tb.TambError):
        lad.sch(lad.v(a, b, c, d).assign(0.0)).execute()
    lad.sch.clear()
    # reading and contracting with it still work; clearing the mark restores writes
    assert np.array_equal(lad.v.read(), vh)
    lad.v.set_read_only(False)
    lad.v.write(vh)


def test_structural_zeros_within_one_execute(ec):
    """v = L*L assigned in the same execute as r2 += v*t2: the (alpha beta|beta alpha)
    blocks of v get no task in the assignment (L vanishes between spins), so the
    contraction skips them; the FP64 result is bit-identical to running the two ops in
    separate executes (where nothing is known about v), split-INT8 within 1e-11."""
    lad = W.ladder(4, 13, seed=11, tile_lo=3, tile_hi=6, ec=ec, build_v=False)
    a, b, c, d, i, j = lad.labels
    V = lad.V
    CI = tb.TiledIndexSpace(tb.IndexSpace(40), 16)
    q = CI.label()
    L = tb.Tensor([CI, V, V], spin_mask=[2, 0, 1]).allocate(ec)
    L.write(np.random.default_rng(3).normal(size=L.nelems))

    def run(together, profile=True):
        lad.sch(lad.r2().assign(0.0)).execute()
        lad.sch(lad.v(a, b, c, d).assign(L(q, a, c) * L(q, b, d)))
        if not together:
            lad.sch.execute()
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute(tb.ExecutionHW.GPU, profile)
        return lad.r2.read(), lad.sch.op_stats(-1)

    apart, st0 = run(False)
    joint, st1 = run(True)
    assert st0["flops_run"] == st0["flops"]
    assert st1["flops"] == st0["flops"] and st1["flops_run"] < st1["flops"]
    assert np.array_equal(apart, joint)
    ec.set_precision(tb.Precision.INT8, 1e-11)
    try:
        joint8, st8 = run(True)
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert st8["flops_run"] == st1["flops_run"]
    assert rel_err(joint8, apart) <= 1e-11


def test_digit_cache_bitwise_and_bounded(ec):
    """With the digit cache on, the read-only v is split once and kept: two contractions
    in a row give the bits of the per-call split, the cache holds bytes, a budget too
    small keeps nothing, and clearing the mark releases them at once, while the
    scheduler still holds the contraction's cached layout."""
    lad, vh, zero = _ladder_with_zero_blocks(ec, seed=13)
    a, b, c, d, i, j = lad.labels
    want = _oracle(lad, vh)
    lad.v.set_read_only(True)

    def run():
        lad.sch(lad.r2().assign(0.0)).execute()
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute()
        return lad.r2.read()

    ec.set_precision(tb.Precision.INT8, 1e-11)
    try:
        plain = run()
        ec.set_digit_cache(1 << 30)
        first, second = run(), run()
        used, limit = ec.digit_cache_info()
        assert used > 0 and limit == 1 << 30
        assert np.array_equal(first, plain) and np.array_equal(second, plain)
        assert rel_err(second, want) <= 1e-11
        lad.v.set_read_only(False)  # drops the entries (and the work lists keyed by the mark)
        assert ec.digit_cache_info()[0] == 0
        assert rel_err(run(), want) <= 1e-11
        lad.v.set_read_only(True)
        ec.set_digit_cache(1)  # too small for any entry: split per call, same bits
        assert np.array_equal(run(), plain)
    finally:
        ec.set_digit_cache(0)
        ec.set_precision(tb.Precision.FP64)
        lad.v.set_read_only(False)
