"""GPU checks of the tape (tb_tape_*): the gradient of the coupled-cluster energy
functional E(t2) = sum w(i,j,a,b) t2(a,b,i,j) + 1/4 sum t2(a,b,i,j) [v(a,b,c,d) t2(c,d,i,j)]
with respect to t2, against

* the oracle: dE/dt2 = w(i,j,a,b) + 1/4 v.t2 + 1/4 sum_ab v(a,b,c,d) t2(a,b,i,j), the
  last term being the swapped-operand contraction run through the reference's
  compiled block_multiply (oracle/_ref);
* central finite differences (step 1e-5) on 64 random amplitudes.

Bars: FP64 gradient within 1e-12 of the oracle (max |diff| / max |g|), split-INT8
within 1e-11; finite differences within 1e-7 of the gradient (max |diff| / max |g|
over the sampled amplitudes) in both modes."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import _capi as A
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FD_TOL = 1e-7


def _oracle_tensor(t, mask):
    return O.BlockTensor([s.tile_sizes for s in t.spaces], [s.tile_spins for s in t.spaces], mask)


def _expected(P):
    """E and dE/dt2 (packed in t2's layout) from the oracle."""
    lad = P.lad
    ov, ot, ox, oy = (_oracle_tensor(x, [0, 0, 1, 1]) for x in (lad.v, lad.t2, lad.t2, lad.t2))
    ow = _oracle_tensor(P.w, [0, 0, 1, 1])
    ov.data[:ov.total] = lad.v.read()
    ot.data[:ot.total] = lad.t2.read()
    ow.data[:ow.total] = P.w_host
    # labels a b c d i j = 1..6
    O.mult_bufacc(ox, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [3, 4, 5, 6])
    O.mult_bufacc(oy, [3, 4, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [1, 2, 5, 6], impl="ref")
    wt = np.zeros(ot.total)
    for bid in ot.blockids():
        off = ot.locate(bid)
        blk = ow.block((bid[2], bid[3], bid[0], bid[1]))
        wt[off:off + blk.size] = blk.transpose(2, 3, 0, 1).reshape(-1)
    t2 = ot.data[:ot.total]
    x = ox.data[:ox.total]
    e = float(np.dot(wt, t2) + 0.25 * np.dot(t2, x))
    g = wt + 0.25 * x + 0.25 * oy.data[:oy.total]
    return e, g


@pytest.fixture(scope="module")
def problem(ec):
    return W.energy_problem(4, 13, seed=5, tile_lo=3, tile_hi=6, ec=ec, build_v=True)


@pytest.mark.parametrize("mode,tol", [(tb.Precision.FP64, 1e-12), (tb.Precision.INT8, 1e-11)])
def test_gradient_matches_oracle(ec, problem, mode, tol):
    P = problem
    want_e, want_g = _expected(P)
    ec.set_precision(mode, 1e-11)
    try:
        e = W.energy(P, gradient=True)
    finally:
        ec.set_precision(tb.Precision.FP64)
    g = P.g.read()
    assert abs(e - want_e) <= tol * max(abs(want_e), 1e-300)
    assert np.max(np.abs(g - want_g)) <= tol * np.max(np.abs(want_g))


@pytest.mark.parametrize("mode", [tb.Precision.FP64, tb.Precision.INT8])
def test_gradient_matches_finite_differences(ec, problem, mode):
    P = problem
    amps = W.fd_amplitudes(P.lad.t2, 64, seed=11)
    ec.set_precision(mode, 1e-11)
    try:
        W.energy(P, gradient=True)
        g = P.g.read()[[off for _, _, off in amps]]
        fd = W.finite_difference(P, amps, h=1e-5)
    finally:
        ec.set_precision(tb.Precision.FP64)
    assert np.max(np.abs(fd - g)) <= FD_TOL * np.max(np.abs(g))


def test_budget_recomputes_the_intermediate(ec):
    full = W.energy_problem(4, 13, seed=6, tile_lo=3, tile_hi=6, ec=ec, build_v=True)
    e_full = W.energy(full, gradient=True)
    g_full = full.g.read().copy()
    info = full.tape.info()
    assert info["recomputed"] == 0 and info["kept_bytes"] == 8 * full.X.nelems
    lean = W.energy_problem(4, 13, seed=6, tile_lo=3, tile_hi=6, ec=ec, build_v=True, budget_bytes=0)
    e_lean = W.energy(lean, gradient=True)
    info = lean.tape.info()
    assert info["recomputed"] == 1 and info["kept_bytes"] == 0
    assert e_lean == e_full
    assert np.array_equal(lean.g.read(), g_full)  # same FP64 arithmetic, recomputed X


def test_gradient_with_broadcast_output_is_rejected(ec):
    V = tb.TiledIndexSpace(tb.IndexSpace(12), 5)
    a, i = V.label(), V.label()
    M = tb.Tensor([V, V]).allocate(ec)
    u = tb.Tensor([V]).allocate(ec)
    y = tb.Tensor([V]).allocate(ec)
    tape = tb.Tape(ec)
    with pytest.raises(tb.TambError) as err:
        tape.contract(y(a), M(a, i) * u(a))  # i is summed inside M alone
    assert err.value.code == A.TB_ERR_NOT_IMPLEMENTED
