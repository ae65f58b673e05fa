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
