"""Permuted AddOps / SetOps on the device, bit-exact against numpy.

TAMM's AddOp runs kernels::block_add / assign per block pair (addop.hpp:230-275,
kernels/assign.hpp:467-485): dst(labels) (=|+=) alpha * src(permuted labels).  Here
all block pairs go through one launch; a pair whose destination stride-1 mode is not
the source's goes through the shared-memory transpose in sub-tiles of at most
64 x 32 (nearly equal extents when a tile is larger), a pair with a mode below 8 or
the same stride-1 mode streams by rows of the destination's last mode (a row longer
than one 2048-element work unit is cut into several).  The product is rounded before
the add, so the result equals numpy's R + alpha * X bit for bit.
"""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _space(tiles):
    return tb.TiledIndexSpace(tb.IndexSpace(int(sum(tiles))), list(tiles))


def _write_dense(t, dense):
    t.write(W.fill_blocks(t, lambda bid, dims, rg: dense[tuple(slice(lo, hi) for lo, hi in rg)]))


def _read_dense(t, shape):
    out = np.full(shape, np.nan)
    keys, offs = t.block_table()
    data = t.read()
    nts = [s.num_tiles for s in t.spaces]
    starts = [s.tile_offsets for s in t.spaces]
    for key, off in zip(keys.tolist(), offs.tolist()):
        bid = []
        for n in reversed(nts):
            bid.append(key % n)
            key //= n
        bid = bid[::-1]
        dims = [int(s.tile_sizes[b]) for s, b in zip(t.spaces, bid)]
        sl = tuple(slice(int(starts[m][b]), int(starts[m][b]) + dims[m]) for m, b in enumerate(bid))
        out[sl] = data[off:off + int(np.prod(dims))].reshape(dims)
    return out


# (tiles of the a-like space, tiles of the i-like space, dst modes, src modes)
CASES = [
    ([20, 24, 30], [20, 12], "abij", "baji"),   # the ladder's r2 += X(b,a,j,i): small planes
    ([20, 24, 30], [20, 12], "abij", "abji"),   # inner swap only
    ([20, 24, 30], [20, 12], "abij", "ijab"),   # p = b, q = j: strided rows on both sides
    ([20, 24, 30], [20, 12], "abij", "baij"),   # same stride-1 mode: streamed
    ([100, 70], [66, 9], "abi", "iba"),         # planes above 64 x 64: ragged sub-tiles
    ([5, 7, 3], [6, 2], "abij", "baji"),        # tiles below 8: streamed
    ([2500, 40], [3, 2], "ia", "ai"),           # streamed rows longer than a work unit
    ([2100, 9], [5, 3], "ija", "jia"),          # long rows and many-row units in one launch
]


@pytest.mark.parametrize("assign", [False, True])
@pytest.mark.parametrize("ta,ti,dm,sm", CASES)
def test_permuted_add_bit_exact(ec, ta, ti, dm, sm, assign):
    A, I = _space(ta), _space(ti)
    space = {"a": A, "b": A, "i": I, "j": I}
    n = {"a": int(sum(ta)), "b": int(sum(ta)), "i": int(sum(ti)), "j": int(sum(ti))}
    rng = np.random.default_rng(len(dm) * 7 + len(ta))
    R = tb.Tensor([space[m] for m in dm]).allocate(ec)
    X = tb.Tensor([space[m] for m in sm]).allocate(ec)
    Rd = rng.normal(size=[n[m] for m in dm])
    Xd = rng.normal(size=[n[m] for m in sm])
    _write_dense(R, Rd)
    _write_dense(X, Xd)
    lab = {"a": A.label(), "b": A.label(), "i": I.label(), "j": I.label()}
    alpha = -0.37
    lhs, rhs = R(*[lab[m] for m in dm]), alpha * X(*[lab[m] for m in sm])
    sch = tb.Scheduler(ec)
    for rep in range(2):  # the second run reuses the cached device list of block pairs
        _write_dense(R, Rd)
        sch(lhs.assign(rhs) if assign else lhs.iadd(rhs)).execute(tb.ExecutionHW.GPU)
        got = _read_dense(R, Rd.shape)
        moved = np.transpose(Xd, [sm.index(m) for m in dm])
        want = alpha * moved if assign else Rd + alpha * moved
        assert np.array_equal(got, want), f"rep {rep}: max diff {np.max(np.abs(got - want)):.3e}"
    R.deallocate()
    X.deallocate()
