"""Checkpoint / restart of a block-sparse tensor (tb_tensor_save / tb_tensor_load):
the file payload is the tensor's admitted blocks in row-major tile order (TAMM's
tammio element order, checked against the oracle's Distribution_NW packing), a load
restores the values bit for bit, and a tensor with other spaces refuses the file."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import _capi as A
from tamm_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_save_load_round_trip(ec, tmp_path):
    lad = W.ladder(4, 13, seed=9, tile_lo=3, tile_hi=6, ec=ec, build_v=False)
    t2 = lad.t2
    path = tmp_path / "t2.ckpt"
    t2.save(path)
    raw = np.fromfile(path, dtype=np.uint8)
    payload = raw[raw.size - 8 * t2.nelems:].view(np.float64)
    ot = O.BlockTensor([s.tile_sizes for s in t2.spaces], [s.tile_spins for s in t2.spaces], [0, 0, 1, 1])
    assert raw[:8].tobytes() == b"TBTENS01" and ot.total == t2.nelems
    assert np.array_equal(payload, lad.t2_host)  # packed in the oracle's block order
    lad.sch(t2().assign(0.0)).execute()
    t2.load(path)
    assert np.array_equal(t2.read(), lad.t2_host)
    other = tb.Tensor([lad.V, lad.V, lad.O, lad.O]).allocate(ec)  # no spin symmetry
    with pytest.raises(tb.TambError) as err:
        other.load(path)
    assert err.value.code == A.TB_ERR_INVALID
