"""Streamed triples energy (tamm_b200.triples) against a dense restatement of its
formula, on a small spin-blocked MO space (O=6, V=16, tile 4, j streamed in blocks of 2),
summed over every streaming step:

    W(a,b,c,i,j,k) = sum_d t2(a,d,i,j) v(b,c,d,k) - sum_l t2(a,b,i,l) v(l,c,j,k)
    E = sum W^2 / (e_i + e_j + e_k - e_a - e_b - e_c)

with v(b,c,d,k) = sum_Q L(Q,b,d) L(Q,c,k), v(l,c,j,k) = sum_Q L(Q,l,j) L(Q,c,k), the
Cholesky vectors read back from the device.  TAMM has no triples code, so the
reference is this restatement (numpy einsum).  Bars: FP64 1e-12, split-INT8 1e-10
relative to |E|, for the separate W update and denominator-energy ops and for the
energy fused into the epilogue of the contraction over d (Scheduler.mult_energy)."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import triples

pytestmark = pytest.mark.gpu


def _dense(t, starts):
    """Dense copy of a tensor over its modes' full ranges (zeros where not stored)."""
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
        n = int(np.prod(dims))
        sl = tuple(slice(int(tofs[m][bid[m]]), int(tofs[m][bid[m]]) + dims[m]) for m in range(len(dims)))
        out[sl] = data[off:off + n].reshape(dims)
    return out


def _reference(P, oa, va, seed):
    no = 2 * oa
    T = P.T
    Lvv, Lvo, Loo = (_dense(T[n], None) for n in ("L_vv", "L_vo", "L_oo"))
    t2 = triples._dense_t2(oa, va, P.eps, seed)
    v1 = np.einsum("qbd,qck->bcdk", Lvv, Lvo)
    v2 = np.einsum("qlj,qck->lcjk", Loo, Lvo)
    Wd = np.einsum("adij,bcdk->abcijk", t2, v1) - np.einsum("abil,lcjk->abcijk", t2, v2)
    eo, ev = P.eps[:no], P.eps[no:]
    D = (eo[None, None, None, :, None, None] + eo[None, None, None, None, :, None] + eo[None, None, None, None, None, :]
         - ev[:, None, None, None, None, None] - ev[None, :, None, None, None, None] - ev[None, None, :, None, None, None])
    return float(np.sum(Wd * Wd / D))


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("dtile", [4, 0])
@pytest.mark.parametrize("mode,tol", [(tb.Precision.FP64, 1e-12), (tb.Precision.INT8, 1e-10)])
def test_streamed_triples_energy(ec, mode, tol, dtile, fused):
    oa, va, seed = 3, 8, 4
    # j blocks of 2, 1 (ragged); d on the output tiling (4) or one tile per spin block (0)
    P = triples.build(oa, va, tile=4, jtile=2, dtile=dtile, seed=seed, ec=ec)
    want = _reference(P, oa, va, seed)
    ec.set_precision(mode, 1e-11)
    try:
        e, flops, _ = triples.energy(P, triples.steps(P), tb.Scheduler(ec), fused=fused)
    finally:
        ec.set_precision(tb.Precision.FP64)
        P.release()
    assert flops > 0 and want < 0
    assert abs(e - want) <= tol * abs(want)
