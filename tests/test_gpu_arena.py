"""Arena sub-allocation through the C ABI (tb_ctx_alloc / tb_ctx_free): 256-byte
aligned blocks, occupancy accounting, allocation after free, and a clear out-of-memory
status when the arena cannot serve a request."""
import pytest

import tamm_b200 as tb
from tamm_b200 import _capi as A

pytestmark = pytest.mark.gpu


def test_alloc_free_accounting(ec):
    used0, _, cap = ec.arena_info()
    p = ec.alloc(1000)
    q = ec.alloc(1)
    assert p % 256 == 0 and q % 256 == 0 and p != q
    used1, peak, _ = ec.arena_info()
    assert used1 - used0 == 1024 + 256 and peak >= used1
    ec.free(p)
    r = ec.alloc(512)  # best fit over the free list (the session arena may hold other gaps)
    assert r % 256 == 0
    ec.free(r).free(q)
    assert ec.arena_info()[0] == used0
    with pytest.raises(tb.TambError) as err:
        ec.alloc(cap + 256)
    assert err.value.code == A.TB_ERR_NO_MEMORY


def test_best_fit_and_coalescing():
    """On a fresh 1 MiB arena: a freed 512-byte gap is preferred to a larger free block
    for a 256-byte request (best fit, lowest offset among equal sizes), and freeing every
    block coalesces the arena back into one block that a full-size request takes."""
    ec = tb.ExecutionContext(0, 1 << 20)
    try:
        used0, _, cap = ec.arena_info()  # (anything the context holds itself sits below)
        a = ec.alloc(256)
        b = ec.alloc(512)
        c = ec.alloc(256)
        d = ec.alloc(1024)
        e = ec.alloc(256)
        assert [a, b, c, d, e] == [a, a + 256, a + 768, a + 1024, a + 2048]
        ec.free(b).free(d)                      # gaps of 512 and 1024 bytes, then the tail
        x = ec.alloc(256)
        assert x == b                           # the smallest gap that holds it
        y = ec.alloc(1024)
        assert y == d                           # an exact fit ahead of the tail
        z = ec.alloc(256)
        assert z == b + 256                     # the rest of the first gap
        for p in (a, c, e, x, y, z):
            ec.free(p)
        assert ec.arena_info()[0] == used0
        whole = ec.alloc(cap - used0)           # one block again: every neighbour merged
        assert whole == a
        ec.free(whole)
    finally:
        ec.close()
