"""CPU tests of the product library: it loads, exports every C-ABI symbol the header
declares, and its host logic (tiling, spin sparsity, Distribution_NW block tables,
MultOp enumeration, argument checking) matches the oracle bit-exactly.  No GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import _capi as A
from tamm_b200 import workloads as W
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "tamm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = A.lib()
    syms = header_symbols()
    assert len(syms) > 40
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(syms) - {"tb_status_string"} <= set(A.PROTOS), set(syms) - set(A.PROTOS)


def test_status_and_last_error():
    L = A.lib()
    assert L.tb_status_string(A.TB_ERR_INVALID) == b"invalid argument"
    lab = (C.c_int * 2)(-1, -1)  # repeated label in C
    plan = A.h()
    rc = L.tb_plan_contraction(lab, 2, lab, 1, lab, 1, 0, 0.0, 0, C.byref(plan))
    assert rc == A.TB_ERR_INVALID
    assert "repeated label" in A.last_error()
    cl = (C.c_int * 1)(-9)  # output label in neither input
    al = (C.c_int * 1)(-1)
    rc = L.tb_plan_contraction(cl, 1, al, 1, al, 1, 0, 0.0, 0, C.byref(plan))
    assert rc == A.TB_ERR_INVALID and "neither input" in A.last_error()
    rc = L.tb_plan_contraction(cl, 1, cl, 1, al, 1, 7, 0.0, 0, C.byref(plan))
    assert rc == A.TB_ERR_INVALID and "mode" in A.last_error()


SPIN_IS = dict(named={"occ": [(0, 10)], "virt": [(10, 20)]},
               spin={2: [(0, 5), (10, 15)], 1: [(5, 10), (15, 20)]})


def test_tiling_matches_oracle():
    for n, named, spin, tile in [(20, SPIN_IS["named"], SPIN_IS["spin"], 3), (50, {}, {}, 20),
                                 (37, {"x": [(0, 11)]}, {}, 4), (7, {}, {}, 10)]:
        is_ = tb.IndexSpace(n, named=named, spin=spin)
        tis = tb.TiledIndexSpace(is_, tile)
        bounds = [x for d in (named, spin) for rs in d.values() for r in rs for x in r]
        want = np.diff(O.tile_offsets_uniform(n, bounds, tile))
        assert list(tis.tile_sizes) == list(want)
    is_ = tb.IndexSpace(20, **SPIN_IS)
    assert list(tb.TiledIndexSpace(is_, [3, 2, 3, 2, 3, 2, 3, 2]).tile_sizes) == [3, 2, 3, 2] * 2
    with pytest.raises(tb.TambError):
        tb.TiledIndexSpace(is_, [4, 4, 4, 4, 4])
    with pytest.raises(tb.TambError):
        tb.TiledIndexSpace(is_, [3, 3])


def test_tile_spins_and_subspaces():
    MO = W.mo_tiled(3, 7, [3], [4, 3])
    assert list(MO.tile_sizes) == [3, 3, 4, 3, 4, 3]
    assert list(MO.tile_spins) == [1, 2, 1, 1, 2, 2]
    occ, virt = MO("occ"), MO("virt")
    assert list(occ.root_tiles) == [0, 1] and list(virt.root_tiles) == [2, 3, 4, 5]
    va = MO("virt_alpha")
    assert list(va.root_tiles) == [2, 3]
    sub = virt.sub(1, 3)
    assert list(sub.root_tiles) == [3, 4] and list(sub.tile_spins) == [1, 2]


def _oracle_tensor(t: tb.Tensor, mask):
    return O.BlockTensor([s.tile_sizes for s in t.spaces], [s.tile_spins for s in t.spaces], mask)


@pytest.mark.parametrize("spin", [None, (2, 2), (1, 1)])
def test_block_table_matches_oracle(spin):
    MO = W.mo_tiled(4, 9, [3, 1], [4, 5])
    O_, V = MO("occ"), MO("virt")
    spaces = [V, V, O_, O_] if spin != (1, 1) else [V, O_]
    t = tb.Tensor(spaces, spin=spin)
    mask = None if spin is None else [0] * spin[0] + [1] * spin[1]
    ot = _oracle_tensor(t, mask)
    keys, offs = t.block_table()
    assert list(keys) == list(ot.keys)
    assert list(offs) == list(ot.offsets)
    assert t.nelems == ot.total
    for bid in ot.blockids()[:20]:
        assert t.is_non_zero(bid)
        assert t.locate(bid) == ot.locate(bid)


def test_mult_enumeration_matches_oracle():
    """Admitted (C,A,B) triples and FLOPs of the ladder, the config-1 shape and a
    sub-space-labelled op equal the oracle's execute_bufacc enumeration."""
    MO = W.mo_tiled(3, 8, [2, 1], [3, 5])
    Ot, V = MO("occ"), MO("virt")
    v = tb.Tensor([V, V, V, V], spin=(2, 2))
    t2 = tb.Tensor([V, V, Ot, Ot], spin=(2, 2))
    r2 = tb.Tensor([V, V, Ot, Ot], spin=(2, 2))
    a, b, c, d = V.labels(4)
    i, j = Ot.labels(2)
    ng, nt, fl = tb.tamm.mult_info(r2(a, b, i, j), v(a, b, c, d), t2(c, d, i, j))
    ov, ot2, or2 = (_oracle_tensor(x, [0, 0, 1, 1]) for x in (v, t2, r2))
    ntr, ofl = O.mult_count(or2, [1, 2, 5, 6], ov, [1, 2, 3, 4], ot2, [3, 4, 5, 6])
    assert (nt, fl) == (ntr, ofl)
    assert ng == len(or2.keys)
    # labels on a sub-space of the tensor's space (translate_blockid)
    va = MO("virt_alpha")
    aa, bb, cc, dd = va.labels(4)
    ng2, nt2, fl2 = tb.tamm.mult_info(r2(aa, bb, i, j), v(aa, bb, cc, dd), t2(cc, dd, i, j))
    vmap = [list(V.root_tiles).index(r) for r in va.root_tiles]
    tm = [vmap, vmap, None, None]
    ntr2, ofl2 = O.mult_count(or2, [1, 2, 5, 6], ov, [1, 2, 3, 4], ot2, [3, 4, 5, 6],
                              tmaps=(tm, tm, [vmap, vmap, vmap, vmap]))
    assert (nt2, fl2) == (ntr2, ofl2)
    assert fl2 < fl


def test_ladder_flops_formula():
    """Config 2 (O=40, V=360) admitted FLOPs: 10 spin combinations x 2 x 180^4 x 20^2."""
    rng = np.random.default_rng(1)
    occ_t = W.random_tiles(20, 24, 48, rng)
    virt_t = W.random_tiles(180, 24, 48, rng)
    assert occ_t == [20] and sum(virt_t) == 180
    MO = W.mo_tiled(20, 180, occ_t, virt_t)
    Ot, V = MO("occ"), MO("virt")
    v = tb.Tensor([V, V, V, V], spin=(2, 2))
    t2 = tb.Tensor([V, V, Ot, Ot], spin=(2, 2))
    r2 = tb.Tensor([V, V, Ot, Ot], spin=(2, 2))
    a, b, c, d = V.labels(4)
    i, j = Ot.labels(2)
    _, _, fl = tb.tamm.mult_info(r2(a, b, i, j), v(a, b, c, d), t2(c, d, i, j))
    assert fl == 10 * 2 * 180 ** 4 * 20 ** 2


def test_invalid_ops_rejected_on_host():
    is_ = tb.IndexSpace(10)
    T = tb.TiledIndexSpace(is_, 5)
    x = tb.Tensor([T, T])
    i, j, k = T.labels(3)
    with pytest.raises(tb.TambError):  # output label in neither input
        tb.tamm.mult_info(x(i, k), x(i, j), x(j, i))
    with pytest.raises(tb.TambError):  # repeated label
        tb.tamm.mult_info(x(i, i), x(i, j), x(j, i))
    with pytest.raises(ValueError):
        x(i, j, k)


def test_front_end_attribute_kinds():
    """The context's stream is a property (bench and tests pass it to torch as an int);
    the digit-cache controls are methods."""
    import tamm_b200 as tb
    assert isinstance(tb.ExecutionContext.stream, property)
    assert callable(tb.ExecutionContext.set_digit_cache) and callable(tb.ExecutionContext.digit_cache_info)
