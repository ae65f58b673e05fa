"""GPU checks of the doubles-residual iteration (tamm_b200.ccsd) on a small spin-blocked
MO space: every op of the iteration against the oracle (contractions through the
oracle's MultOp restatement, the four P(ab)P(ij) adds and the orbital-energy update
in numpy over its block tensors), then a CUDA-graph replay against the eager run and
the autotuned split-INT8 iteration against the FP64 one.

Bars: FP64 residual, updated amplitudes, energy and residual norm within 1e-12 of
the oracle (max |diff| / max |ref|); graph replay bit-identical to the eager run;
split-INT8 within 1e-11 of the FP64 iteration."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import ccsd
from oracle import oracle as O

pytestmark = pytest.mark.gpu

a, b, c, d, i, j, k, l, q = range(1, 10)
MASKS = {"L_vo": [2, 0, 1], "L_oo": [2, 0, 1], "L_vv": [2, 0, 1], "f_oo": [0, 1], "f_vv": [0, 1],
         "F_vv": [0, 1], "F_oo": [0, 1]}


def rel(x, y):
    return float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))


def _ob(t, mask, data=None):
    o = O.BlockTensor([s.tile_sizes for s in t.spaces], [s.tile_spins for s in t.spaces], mask)
    if data is not None:
        o.data[:o.total] = data
    return o


def _add(dst, dlabels, alpha, src, slabels):
    """dst(dlabels) += alpha * src(slabels) over dst's stored blocks (host AddOp)."""
    for bid in dst.blockids():
        tile = dict(zip(dlabels, bid))
        blk = src.block(tuple(tile[x] for x in slabels))
        if blk is None:
            continue
        dst.block(bid)[...] += alpha * blk.transpose([slabels.index(x) for x in dlabels])


def _oracle_iteration(P, t2_0, impl="port"):
    """One iteration on the oracle's block tensors; impl "ref" runs every block triple
    through the reference's compiled block_multiply."""
    T = P.T
    ot = {n: _ob(t, MASKS.get(n, [0, 0, 1, 1]), t.read()) for n, t in T.items()
          if n in ("L_vo", "L_oo", "L_vv", "f_oo", "f_vv", "v_vvoo", "v_oooo", "v_ovvo")}
    V, O_ = T["t2"].spaces[0], T["t2"].spaces[2]
    t2 = _ob(T["t2"], [0, 0, 1, 1], t2_0)
    v = ot["v_vvoo"]
    mk = lambda like, mask=(0, 0, 1, 1): _ob(like, list(mask))
    F_vv = mk(T["F_vv"], (0, 1)); F_vv.data[:] = ot["f_vv"].data
    O.mult_bufacc(F_vv, [b, c], -0.5, v, [c, d, k, l], t2, [b, d, k, l], impl=impl)
    F_oo = mk(T["F_oo"], (0, 1)); F_oo.data[:] = ot["f_oo"].data
    O.mult_bufacc(F_oo, [k, j], 0.5, v, [c, d, k, l], t2, [c, d, j, l], impl=impl)
    W_oo = mk(T["W_oo"]); W_oo.data[:] = 0.5 * ot["v_oooo"].data
    O.mult_bufacc(W_oo, [k, l, i, j], 0.25, v, [c, d, k, l], t2, [c, d, i, j], impl=impl)
    W_ov = mk(T["W_ov"]); W_ov.data[:] = ot["v_ovvo"].data
    O.mult_bufacc(W_ov, [k, b, c, j], 0.5, v, [c, d, k, l], t2, [d, b, l, j], impl=impl)
    r2 = mk(T["r2"]); r2.data[:] = v.data
    O.mult_bufacc(r2, [a, b, i, j], 1.0, F_vv, [b, c], t2, [a, c, i, j], impl=impl)
    O.mult_bufacc(r2, [a, b, i, j], -1.0, F_vv, [a, c], t2, [b, c, i, j], impl=impl)
    O.mult_bufacc(r2, [a, b, i, j], -1.0, F_oo, [k, j], t2, [a, b, i, k], impl=impl)
    O.mult_bufacc(r2, [a, b, i, j], 1.0, F_oo, [k, i], t2, [a, b, j, k], impl=impl)
    O.mult_bufacc(r2, [a, b, i, j], 1.0, W_oo, [k, l, i, j], t2, [a, b, k, l], impl=impl)
    X = mk(T["X"])
    O.mult_bufacc(X, [a, b, i, j], 1.0, t2, [a, c, i, k], W_ov, [k, b, c, j], impl=impl)
    for alpha, sl in ((1.0, [a, b, i, j]), (-1.0, [b, a, i, j]), (-1.0, [a, b, j, i]), (1.0, [b, a, j, i])):
        _add(r2, [a, b, i, j], alpha, X, sl)
    v4 = O.BlockTensor([V.tile_sizes] * 4, [V.tile_spins] * 4, [0, 0, 1, 1])
    O.mult_bufacc(v4, [a, b, c, d], 1.0, ot["L_vv"], [q, a, c], ot["L_vv"], [q, b, d], impl=impl)
    O.mult_bufacc(r2, [a, b, i, j], 0.5, v4, [a, b, c, d], t2, [c, d, i, j], impl=impl)
    energy = 0.25 * float(np.dot(v.data[:v.total], t2.data[:t2.total]))
    norm = float(np.sqrt(np.dot(r2.data[:r2.total], r2.data[:r2.total])))
    t2n = _ob(T["t2"], [0, 0, 1, 1], t2_0)
    starts = [s.tile_offsets for s in (V, V, O_, O_)]
    for bid in t2n.blockids():
        e = [P.eps[starts[m][bid[m]]:starts[m][bid[m]] + t2n.block_dims(bid)[m]] for m in range(4)]
        D = e[0][:, None, None, None] + e[1][None, :, None, None] - e[2][None, None, :, None] - e[3][None, None, None, :]
        t2n.block(bid)[...] -= r2.block(bid) / D
    return r2.data[:r2.total].copy(), t2n.data[:t2n.total].copy(), energy, norm


@pytest.fixture(scope="module")
def problem(ec):
    return ccsd.build(4, 13, seed=2, tile_lo=3, tile_hi=6, ec=ec, batch_tiles=2)


def _run(P, sch, t2_0):
    P.T["t2"].write(t2_0)
    ccsd.queue_iteration(P, sch)
    sch.execute(tb.ExecutionHW.GPU)
    e, n = sch.scalars(2)
    return P.T["r2"].read().copy(), P.T["t2"].read().copy(), e, n


def test_iteration_matches_oracle(ec, problem):
    P = problem
    t2_0 = P.T["t2"].read().copy()
    want_r2, want_t2, want_e, want_n = _oracle_iteration(P, t2_0)
    r2, t2, e, n = _run(P, tb.Scheduler(ec), t2_0)
    P.T["t2"].write(t2_0)
    assert rel(r2, want_r2) <= 1e-12
    assert rel(t2, want_t2) <= 1e-12
    assert abs(e - want_e) <= 1e-12 * abs(want_e)
    assert abs(n - want_n) <= 1e-12 * want_n


@pytest.mark.parametrize("mode", [tb.Precision.FP64, tb.Precision.INT8])
def test_graph_replay_matches_eager(ec, problem, mode):
    P = problem
    t2_0 = P.T["t2"].read().copy()
    ec.set_precision(mode, 1e-11)
    try:
        sch = tb.Scheduler(ec)
        r2_e, t2_e, e_e, n_e = _run(P, sch, t2_0)
        P.T["t2"].write(t2_0)
        ccsd.queue_iteration(P, sch)
        g = sch.graph()
        for _ in range(2):  # replays start from the same amplitudes
            P.T["t2"].write(t2_0)
            g.launch().sync()
            assert np.array_equal(P.T["r2"].read(), r2_e)
            assert np.array_equal(P.T["t2"].read(), t2_e)
            assert tuple(sch.scalars(2)) == (e_e, n_e)
        del g
    finally:
        ec.set_precision(tb.Precision.FP64)
        P.T["t2"].write(t2_0)


def test_autotuned_int8_iteration(ec, problem):
    P = problem
    t2_0 = P.T["t2"].read().copy()
    r2_f, t2_f, e_f, n_f = _run(P, tb.Scheduler(ec), t2_0)
    ec.set_precision(tb.Precision.INT8, 1e-11)
    try:
        sch = tb.Scheduler(ec).autotune(True)
        r2, t2, e, n = _run(P, sch, t2_0)
        tuned = ccsd.tune_report(sch)
    finally:
        ec.set_precision(tb.Precision.FP64)
        P.T["t2"].write(t2_0)
    assert rel(r2, r2_f) <= 1e-11 and rel(t2, t2_f) <= 1e-11
    assert abs(e - e_f) <= 1e-11 * abs(e_f) and abs(n - n_f) <= 1e-11 * n_f
    chosen = [x for x in tuned if x is not None]
    assert chosen  # every plain contraction of the list went through the autotuner
    for x in chosen:
        assert len(x["candidates"]) >= 2 and x["candidates"][0][0] == tb.Precision.FP64
        assert min(ms for _, _, ms in x["candidates"]) == min(
            ms for m, t, ms in x["candidates"] if (m, t) == (x["mode"], x["tile_n"]))
