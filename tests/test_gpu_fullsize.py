"""Parity at the sizes that are benchmarked, against the oracle (the reference's
compiled block_multiply where it was built, else the C restatement).

* Config 2, full size (O=40, V=360, virtual tiles U{24..48}, seed 1 — the bench's
  workload, v read-only so its exactly-zero spin blocks are skipped as in the bench):
  18 output blocks of r2, three per spin case (the widest, the narrowest and one
  seeded pair of virtual tiles), each recomputed on the host from the device's v and
  t2 blocks by the oracle's block_multiply over every admitted (c, d).  FP64 within
  1e-12 and split-INT8 within 1e-11 of max |r2| over the sampled blocks; the FP64
  result with v marked read-only bit-identical to the unmarked one.
* Config 3 shapes at O=20, V=160, tiles U{20..64}: one doubles-residual iteration
  against the oracle's iteration (every contraction through the reference's block
  kernel): FP64 1e-12, split-INT8 1e-11.
* Config 5 shapes at tile 40 (O=20, V=160, j blocks of 2, the summed d one tile per
  spin block): the W of one streaming step against a dense numpy restatement:
  FP64 1e-12, split-INT8 1e-11 of max |W|.
Each case prints one line with its errors."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import ccsd, triples
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

IMPL = "ref" if O.ref() is not None else "port"


@pytest.fixture(scope="module")
def big_ec():
    ctx = tb.ExecutionContext(0, 110 << 30)
    yield ctx
    ctx.close()


def _sample_blocks(lad, seed=5):
    V, Oc = lad.V, lad.O
    vz = [V.tile_size(x) for x in range(V.num_tiles)]
    rng = np.random.default_rng(seed)
    out = []
    for sa, sb, si, sj in ((1, 1, 1, 1), (2, 2, 2, 2), (1, 2, 1, 2), (1, 2, 2, 1), (2, 1, 1, 2), (2, 1, 2, 1)):
        va = [x for x in range(V.num_tiles) if V.spin(x) == sa]
        vb = [x for x in range(V.num_tiles) if V.spin(x) == sb]
        i = [x for x in range(Oc.num_tiles) if Oc.spin(x) == si][0]
        j = [x for x in range(Oc.num_tiles) if Oc.spin(x) == sj][0]
        wide = (max(va, key=lambda x: vz[x]), max(vb, key=lambda x: vz[x]))
        narrow = (min(va, key=lambda x: vz[x]), min(vb, key=lambda x: vz[x]))
        rand = (int(rng.choice(va)), int(rng.choice(vb)))
        for a, b in (wide, narrow, rand):
            out.append((a, b, i, j))
    return out


def _reference_block(lad, bid):
    a, b, i, j = bid
    V = lad.V
    ref = np.zeros(lad.r2.block_dims(list(bid)))
    for c in range(V.num_tiles):
        for d in range(V.num_tiles):
            if not (lad.v.is_non_zero([a, b, c, d]) and lad.t2.is_non_zero([c, d, i, j])):
                continue
            vb = lad.v.get([a, b, c, d])
            tb_ = lad.t2.get([c, d, i, j])
            assert O.block_multiply(1.0, vb, [1, 2, 3, 4], tb_, [3, 4, 5, 6], 1.0, ref, [1, 2, 5, 6], 0,
                                    impl=IMPL) == 0
    return ref


def test_config2_full_size_sampled_blocks(big_ec):
    ec = big_ec
    lad = W.ladder(20, 180, seed=1, ec=ec)
    a, b, c, d, i, j = lad.labels

    def run():
        lad.sch(lad.r2().assign(0.0)).execute()
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute(tb.ExecutionHW.GPU, True)
        return lad.sch.op_stats(-1)

    try:
        run()
        plain = lad.r2.read()
        lad.v.set_read_only(True)
        st = run()
        got64 = {bid: lad.r2.get(list(bid)) for bid in _sample_blocks(lad)}
        assert np.array_equal(lad.r2.read(), plain), "skipping zero v blocks changed the FP64 result"
        del plain
        ec.set_precision(tb.Precision.INT8, 1e-11)
        try:
            st8 = run()
        finally:
            ec.set_precision(tb.Precision.FP64)
        got8 = {bid: lad.r2.get(list(bid)) for bid in got64}
        refs = {bid: _reference_block(lad, bid) for bid in got64}
        scale = max(float(np.max(np.abs(r))) for r in refs.values())
        e64 = max(float(np.max(np.abs(got64[x] - refs[x]))) for x in refs) / scale
        e8 = max(float(np.max(np.abs(got8[x] - refs[x]))) for x in refs) / scale
        print(f"config2 O=40 V=360: {len(refs)} blocks, admitted {st['flops']:.3e} run {st['flops_run']:.3e} "
              f"FLOP, max rel err FP64 {e64:.2e} split-INT8 {e8:.2e} (slices {st8['slices_min']}-{st8['slices_max']})")
        assert st["flops_run"] < st["flops"]
        assert e64 <= 1e-12 and e8 <= 1e-11
    finally:
        lad.v.set_read_only(False)
        lad.sch.deallocate(lad.v, lad.t2, lad.r2)


def test_config3_iteration_O20_V160(big_ec):
    from test_gpu_ccsd import _oracle_iteration, _run, rel
    ec = big_ec
    P = ccsd.build(10, 80, seed=2, tile_lo=20, tile_hi=64, ec=ec, batch_tiles=1)
    t2_0 = P.T["t2"].read().copy()
    want_r2, want_t2, want_e, want_n = _oracle_iteration(P, t2_0, impl=IMPL)
    errs = {}
    for name, mode, tol in (("fp64", tb.Precision.FP64, 1e-12), ("int8", tb.Precision.INT8, 1e-11)):
        ec.set_precision(mode, 1e-11)
        try:
            r2, t2, e, n = _run(P, tb.Scheduler(ec), t2_0)
        finally:
            ec.set_precision(tb.Precision.FP64)
        errs[name] = (rel(r2, want_r2), rel(t2, want_t2), abs(e - want_e) / abs(want_e), abs(n - want_n) / want_n)
        assert max(errs[name]) <= tol, f"{name}: {errs[name]}"
    print(f"config3 O=20 V=160 tiles U{{20..64}}: max rel err (r2, t2, E, |r2|) FP64 "
          f"{max(errs['fp64']):.2e} split-INT8 {max(errs['int8']):.2e}")


def _dense_from(t, sizes=None):
    """Dense copy of a tensor over its modes (zeros where not stored), dims in each
    mode's own tile numbering."""
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


def test_config5_w_step_tile40(big_ec):
    ec = big_ec
    oa, va, seed = 10, 80, 4
    P = triples.build(oa, va, tile=40, jtile=2, dtile=0, seed=seed, ec=ec)
    no = 2 * oa
    step = (3, 6)  # i = 3 (alpha), j block 6 (beta)
    jlo = int(P.Oj.tile_offsets[step[1]])
    jw = int(P.Oj.tile_sizes[step[1]])
    Lvv, Lvo, Loo = (_dense_from(P.T[n]) for n in ("L_vv", "L_vo", "L_oo"))
    t2 = triples._dense_t2(oa, va, P.eps, seed)
    v1 = np.einsum("qbd,qck->bcdk", Lvv, Lvo, optimize=True)
    v2 = np.einsum("qlj,qck->lcjk", Loo[:, :, jlo:jlo + jw], Lvo, optimize=True)
    i = step[0]
    want = (np.einsum("adj,bcdk->abcjk", t2[:, :, i, jlo:jlo + jw], v1, optimize=True)
            - np.einsum("abl,lcjk->abcjk", t2[:, :, i, :], v2, optimize=True))
    errs = {}
    for name, mode, tol in (("fp64", tb.Precision.FP64, 1e-12), ("int8", tb.Precision.INT8, 1e-11)):
        ec.set_precision(mode, 1e-11)
        try:
            sch = tb.Scheduler(ec)
            Wt, _ = triples.queue_pair(P, sch, *step, fused=False)  # W itself: both terms stored
            sch.execute(tb.ExecutionHW.GPU)
            got = _dense_from(Wt)[:, :, :, 0, :, :]
            Wt.deallocate()
        finally:
            ec.set_precision(tb.Precision.FP64)
        # W's spin rule stores only admitted t3 blocks; the formula is zero elsewhere
        errs[name] = float(np.max(np.abs(got - want))) / float(np.max(np.abs(want)))
        assert errs[name] <= tol, f"{name}: {errs[name]:.3e}"
    P.release()
    assert no == 20
    print(f"config5 tile 40 O=20 V=160 step {step}: max rel err of W FP64 {errs['fp64']:.2e} "
          f"split-INT8 {errs['int8']:.2e}")
