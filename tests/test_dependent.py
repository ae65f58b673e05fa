"""Dependent tiled index spaces on the host (no GPU): the blocks a tensor over a
dependent space stores, and the tasks of a contraction over one, equal a plain
restatement of TAMM's rule (a dependent mode's tile must be listed for the tiles of
the modes it depends on; tiled_index_space.hpp:60-72, translate_blockid_if_possible,
utils.hpp:369), on a DLPNO-like PNO space over LMO pairs (Test_DLPNO_Ops.cpp)."""
import itertools

import numpy as np

import tamm_b200 as tb


def _pno(seed=0, n_lmo=7, lmo_tile=2, n_pno=11, pno_tile=3):
    rng = np.random.default_rng(seed)
    LMO = tb.TiledIndexSpace(tb.IndexSpace(n_lmo), lmo_tile)
    REF = tb.TiledIndexSpace(tb.IndexSpace(n_pno), pno_tile)
    allowed = {}
    for ti in range(LMO.num_tiles):
        for tj in range(LMO.num_tiles):
            if rng.uniform() < 0.2:
                continue  # pair without PNOs
            lo = int(rng.integers(0, REF.num_tiles))
            hi = int(rng.integers(lo + 1, REF.num_tiles + 1))
            allowed[(ti, tj)] = (lo, hi)
    PNO = tb.TiledIndexSpace.dependent(REF, [LMO, LMO], {k: REF.sub(lo, hi) for k, (lo, hi) in allowed.items()})
    return LMO, REF, PNO, allowed


def test_dependent_block_table():
    LMO, REF, PNO, allowed = _pno()
    i, j = LMO.labels(2)
    a, e = PNO.labels(2)
    t2 = tb.Tensor([i, j, a(i, j), e(i, j)])
    nl, npn = LMO.num_tiles, REF.num_tiles
    want = []
    for ti, tj, ta, te in itertools.product(range(nl), range(nl), range(npn), range(npn)):
        r = allowed.get((ti, tj))
        if r and r[0] <= ta < r[1] and r[0] <= te < r[1]:
            want.append(((ti * nl + tj) * npn + ta) * npn + te)
    keys, _ = t2.block_table()
    assert keys.tolist() == want


def test_dependent_contraction_tasks():
    """R(i,j,a(i,j),b(i,j)) += t2(i,j,a(i,j),e(i,j)) * F(e,b): tasks are the (output
    block, e) pairs whose blocks all exist."""
    LMO, REF, PNO, allowed = _pno(seed=3)
    i, j = LMO.labels(2)
    a, b, e = PNO.labels(3)
    t2 = tb.Tensor([i, j, a(i, j), e(i, j)])
    R = tb.Tensor([i, j, a(i, j), b(i, j)])
    F = tb.Tensor([REF, REF])
    ng, nt, fl = tb.tamm.mult_info(R(i, j, a, b), t2(i, j, a, e), F(e, b))
    nl, npn = LMO.num_tiles, REF.num_tiles
    sz = [REF.tile_size(x) for x in range(npn)]
    lz = [LMO.tile_size(x) for x in range(nl)]
    wg = wt = 0
    wf = 0.0
    for ti, tj in itertools.product(range(nl), range(nl)):
        r = allowed.get((ti, tj))
        if not r:
            continue
        for ta, tb_ in itertools.product(range(r[0], r[1]), repeat=2):
            wg += 1
            for te in range(r[0], r[1]):
                wt += 1
                wf += 2.0 * lz[ti] * lz[tj] * sz[ta] * sz[tb_] * sz[te]
    assert (ng, nt) == (wg, wt) and fl == wf
