"""Orbital-energy denominator ops (tb_sched_denom, tb_sched_denom_energy) against
numpy, on tilings that reach every branch of the device kernel: a last mode longer
than the CTA's thread count and than the shared-memory table of its denominators
(1100), one between the two (400), short last modes whose blocks have more rows than
one work unit holds (3600 rows of 4 and of 3 columns), and ragged last units.

    update:  t += alpha * r / D       energy:  slot += alpha * sum w^2 / D
    D(x_0..x_last) = sum_m signs[m] * eps[orbital index of x_m]

Bars: the update within 8 rounding errors of its terms, element by element (the
device forms 1/D by Newton-Raphson refinement of a hardware approximation); the energy
within 1e-12 relative (a sum in another order)."""
import numpy as np
import pytest

import tamm_b200 as tb

pytestmark = pytest.mark.gpu

CASES = [
    ([[1100, 400], [1100, 400]], [1.0, -0.25]),
    ([[60, 50], [60, 50], [4, 3, 103]], [1.0, 1.0, 1.0]),
]


def _blocks(t, tilings):
    """(offset, dims, first orbital per mode) of every stored block."""
    keys, offs = t.block_table()
    nts = [len(x) for x in tilings]
    starts = [np.concatenate([[0], np.cumsum(x)]) for x in tilings]
    out = []
    for key, off in zip(keys.tolist(), offs.tolist()):
        bid = []
        for n in reversed(nts):
            bid.append(key % n)
            key //= n
        bid = bid[::-1]
        out.append((off, [tilings[m][b] for m, b in enumerate(bid)], [int(starts[m][b]) for m, b in enumerate(bid)]))
    return out


def _denominators(t, tilings, eps, signs):
    D = np.zeros(t.nelems)
    for off, dims, first in _blocks(t, tilings):
        d = np.zeros(dims)
        for m, (n, f) in enumerate(zip(dims, first)):
            shape = [1] * len(dims)
            shape[m] = n
            d = d + signs[m] * eps[f:f + n].reshape(shape)
        D[off:off + d.size] = d.reshape(-1)
    return D


@pytest.mark.parametrize("tilings,signs", CASES)
def test_denominator_update_and_energy(ec, tilings, signs):
    n = sum(tilings[0])
    assert all(sum(x) == n for x in tilings)
    rng = np.random.default_rng(17)
    eps = rng.uniform(1.0, 3.0, size=n)  # |D| >= 0.25 for the signs above
    is_ = tb.IndexSpace(n)  # every mode over one index space, as the ops require
    spaces = [tb.TiledIndexSpace(is_, list(x)) for x in tilings]
    t, r = (tb.Tensor(spaces).allocate(ec) for _ in range(2))
    t0, r0 = rng.normal(size=t.nelems), rng.normal(size=r.nelems)
    t.write(t0)
    r.write(r0)
    D = _denominators(t, tilings, eps, signs)
    assert np.all(np.abs(D) >= 0.25)
    labels = [s.label() for s in spaces]
    sch = tb.Scheduler(ec)
    sch.set_scalar(5, 0.25)
    sch.denom_energy(5, 0.5, t(*labels), eps, signs)
    sch.denom(t(*labels), -0.75, r(*labels), eps, signs)
    sch.execute(tb.ExecutionHW.GPU)
    want_e = 0.25 + 0.5 * float(np.sum(t0 * t0 / D))
    got_e = float(sch.scalars(6)[5])
    assert abs(got_e - want_e) <= 1e-12 * abs(want_e)
    want_t = t0 - 0.75 * r0 / D
    got_t = t.read()
    assert np.max(np.abs(got_t - want_t)) <= 1e-13 * np.max(np.abs(want_t))
    # elementwise: the device forms 1/D by Newton-Raphson refinement of a hardware
    # approximation; with the products and the sum, a few rounding errors of the terms
    bound = 8 * np.finfo(np.float64).eps * (np.abs(t0) + np.abs(0.75 * r0 / D))
    assert np.all(np.abs(got_t - want_t) <= bound)
