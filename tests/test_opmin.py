"""OpMin on the host: the binary contraction tree the library picks for a multi-factor
product (tb_opmin_order, the plan tb_sched_mult_n runs) equals the oracle's
restatement of opmin::Optimizer (src/tamm/opmin.hpp:438-560) on seeded random
products of 3 to 6 factors, including ties; no GPU needed."""
import numpy as np
import pytest

import tamm_b200 as tb
from oracle import oracle as O


def _spaces(rng, nlab):
    sizes = [int(rng.integers(2, 9)) * int(rng.choice([1, 5, 20])) for _ in range(nlab)]
    return [tb.TiledIndexSpace(tb.IndexSpace(n), max(1, n // 3)) for n in sizes], sizes


@pytest.mark.parametrize("seed", range(12))
def test_opmin_tree_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    nlab = int(rng.integers(4, 8))
    spaces, sizes = _spaces(rng, nlab)
    labels = [s.label() for s in spaces]
    nf = int(rng.integers(3, 7))
    factors = []
    for _ in range(nf):  # every factor at most 3 modes, labels may repeat across factors
        k = int(rng.integers(1, 4))
        idx = sorted(rng.choice(nlab, size=k, replace=False).tolist())
        factors.append(idx)
    used = sorted({x for f in factors for x in f})
    lhs = sorted(rng.choice(used, size=min(2, len(used)), replace=False).tolist())
    lts = [tb.Tensor([spaces[x] for x in f])(*[labels[x] for x in f]) for f in factors]
    lhs_lt = tb.Tensor([spaces[x] for x in lhs])(*[labels[x] for x in lhs])
    got, cost = tb.tamm.opmin_order(lhs_lt, *lts)
    want, wcost = O.opmin_order(factors, lhs, {x: float(sizes[x]) for x in range(nlab)})
    assert got == [tuple(p) for p in want]
    assert cost == wcost


def test_opmin_prefers_the_cheap_association():
    """A(i,k) B(k,l) C(l,j) with |k| = |l| = 500: with |i| = 2, |j| = 5 the product A B
    first costs 2*500*500 + 2*500*5 against 500*500*5 + 2*500*5 for B C first; with
    |i| = 5, |j| = 2 the other way round."""
    def order(ni, nj):
        I, K, L, J = (tb.TiledIndexSpace(tb.IndexSpace(n), 50) for n in (ni, 500, 500, nj))
        i, k, l, j = I.label(), K.label(), L.label(), J.label()
        lts = [tb.Tensor([I, K])(i, k), tb.Tensor([K, L])(k, l), tb.Tensor([L, J])(l, j)]
        return tb.tamm.opmin_order(tb.Tensor([I, J])(i, j), *lts)[0]
    assert set(order(2, 5)[0]) == {1, 2}  # A B first
    assert set(order(5, 2)[0]) == {2, 4}  # B C first
