"""Pins the oracle (CPU): the C restatement against the reference's own compiled
block kernels, the committed golden vectors, and the known answers of TAMM's tests."""
import os

import numpy as np
import pytest

from oracle import oracle as O

# label-pattern cases: (C labels, A labels, B labels); letters map to extents below
PATTERNS = [
    ("abij", "acik", "cbkj"),   # config-1 contraction
    ("abij", "abcd", "cdij"),   # ladder
    ("jikl", "ijmo", "mokl"),   # Test_Mult_Ops 4-D (permuted output)
    ("ijk", "jli", "lik"),      # Test_Ops 3-D with a batch label
    ("ijkl", "jlkm", "likm"),   # Test_Ops 4-D with two batch labels
    ("ijk", "ij", "k"),         # outer product
    ("ij", "ikx", "kjy"),       # A-only / B-only reduction labels
    ("", "ij", "ij"),           # full contraction to a scalar
    ("ij", "ij", ""),           # scale by a scalar tensor
    ("abcij", "adij", "bcdj"),  # 5-D with batch j
]
DIMS = dict(a=3, b=4, c=5, d=2, i=3, j=2, k=4, l=3, m=2, o=3, x=2, y=3)
LAB = {ch: -ord(ch) for ch in DIMS}


def _mk(labels, seed):
    x = np.zeros([DIMS[c] for c in labels], dtype=np.float64)
    O.fill_uniform(x.reshape(-1), seed)
    return x


def _naive(cl, al, bl, A, B):
    return np.einsum(f"{al},{bl}->{cl}", A, B)


@pytest.mark.parametrize("cl,al,bl", PATTERNS)
def test_port_matches_einsum(cl, al, bl):
    A, B, C0 = _mk(al, 1), _mk(bl, 2), _mk(cl, 3)
    for is_assign in (0, 1):
        C = np.array(C0, copy=True)
        assert O.block_multiply(1.3, A, [LAB[c] for c in al], B, [LAB[c] for c in bl], 1.0, C,
                                [LAB[c] for c in cl], is_assign) == 0
        want = (0 if is_assign else C0) + 1.3 * _naive(cl, al, bl, A, B)
        np.testing.assert_allclose(C, want, rtol=1e-13, atol=1e-13)


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (no TAMM source tree)")
@pytest.mark.parametrize("cl,al,bl", PATTERNS)
@pytest.mark.parametrize("beta", [1.0, 0.0, 0.5])
def test_port_matches_reference_block_multiply(cl, al, bl, beta):
    for is_assign in (0, 1):
        A, B, C0 = _mk(al, 1), _mk(bl, 2), _mk(cl, 3)
        Cp, Cr = np.array(C0, copy=True), np.array(C0, copy=True)
        assert O.block_multiply(1.3, A, [LAB[c] for c in al], B, [LAB[c] for c in bl], beta, Cp,
                                [LAB[c] for c in cl], is_assign, "port") == 0
        assert O.block_multiply(1.3, A, [LAB[c] for c in al], B, [LAB[c] for c in bl], beta, Cr,
                                [LAB[c] for c in cl], is_assign, "ref") == 0
        np.testing.assert_allclose(Cp, Cr, rtol=1e-12, atol=1e-13)


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (no TAMM source tree)")
@pytest.mark.parametrize("dl,sl", [("ijk", "kij"), ("ij", "ji"), ("ij", "ij"), ("ij", "ijk"),
                                   ("ijk", "ij"), ("", ""), ("abij", "baji")])
def test_port_matches_reference_assign(dl, sl):
    for is_assign in (0, 1):
        S = _mk(sl, 5)
        D0 = _mk(dl, 6)
        Dp, Dr = np.array(D0, copy=True), np.array(D0, copy=True)
        assert O.assign(Dp, [LAB[c] for c in dl], 0.7, S, [LAB[c] for c in sl], is_assign, "port") == 0
        assert O.assign(Dr, [LAB[c] for c in dl], 0.7, S, [LAB[c] for c in sl], is_assign, "ref") == 0
        np.testing.assert_array_equal(Dp, Dr)


GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "block_multiply_golden.npz")


def test_port_matches_golden_vectors():
    """Outputs of the reference's compiled block_multiply, committed with the script that
    made them (tests/golden/gen_golden.py)."""
    g = np.load(GOLDEN)
    for idx, (cl, al, bl) in enumerate(PATTERNS):
        for beta in (1.0, 0.0, 0.5):
            for is_assign in (0, 1):
                key = f"p{idx}_b{beta}_a{is_assign}"
                A, B, C0 = _mk(al, 1), _mk(bl, 2), _mk(cl, 3)
                C = np.array(C0, copy=True)
                assert O.block_multiply(1.3, A, [LAB[c] for c in al], B, [LAB[c] for c in bl], beta, C,
                                        [LAB[c] for c in cl], is_assign) == 0
                np.testing.assert_allclose(C.reshape(-1), g[key], rtol=1e-12, atol=1e-13, err_msg=key)
    # config-1 block pair and one spin-blocked ladder through the bufacc driver
    np.testing.assert_allclose(config1_block_pair(), g["config1_block"], rtol=1e-12, atol=1e-13)
    lad = small_ladder()
    np.testing.assert_allclose(lad.data[:lad.total], g["ladder_r2"], rtol=1e-12, atol=1e-14)


def config1_block_pair():
    """One tile pair of the config-1 contraction C(a,b,i,j) += A(a,c,i,k) B(c,b,k,j),
    tile 10, A and B uniform [-1, 1] from seed 0."""
    A = np.zeros((10, 10, 10, 10))
    B = np.zeros((10, 10, 10, 10))
    O.fill_uniform(A.reshape(-1), 0, 0)
    O.fill_uniform(B.reshape(-1), 0, A.size)
    C = np.zeros((10, 10, 10, 10))
    lab = {c: -ord(c) for c in "abcijk"}
    assert O.block_multiply(1.0, A, [lab[c] for c in "acik"], B, [lab[c] for c in "cbkj"], 1.0, C,
                            [lab[c] for c in "abij"], 0) == 0
    return C.reshape(-1)


def small_ladder(impl="port"):
    """r2(a,b,i,j) += v(a,b,c,d) t2(c,d,i,j), oa=2 (one occupied tile per spin), va=5 with
    tiles 3,2 per spin, spin mask {2,2}; inputs uniform from fixed seeds."""
    vt, vs = [3, 2, 3, 2], [1, 1, 2, 2]
    ot, os_ = [2, 2], [1, 2]
    v = O.BlockTensor([vt] * 4, [vs] * 4, [0, 0, 1, 1])
    t2 = O.BlockTensor([vt, vt, ot, ot], [vs, vs, os_, os_], [0, 0, 1, 1])
    r2 = O.BlockTensor([vt, vt, ot, ot], [vs, vs, os_, os_], [0, 0, 1, 1])
    O.fill_uniform(v.data[:v.total], 21)
    O.fill_uniform(t2.data[:t2.total], 22)
    a, b, c, d, i, j = -1, -2, -3, -4, -5, -6
    O.mult_bufacc(r2, [a, b, i, j], 1.0, v, [a, b, c, d], t2, [c, d, i, j], impl=impl)
    return r2


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (no TAMM source tree)")
def test_bufacc_port_matches_reference_kernel():
    p = small_ladder("port")
    r = small_ladder("ref")
    np.testing.assert_allclose(p.data, r.data, rtol=1e-12, atol=1e-14)


# ---------------------------------------------------------------- known answers

def test_known_answer_mult_ops_norm():
    """tests/tamm/Test_Mult_Ops.cpp:161-204: N=50 tiled 20 (tiles 20,20,10), A=21, B=2,
    C(j,i,k,l) += A(i,j,m,o) * B(m,o,k,l); |C| = 2.625e8 within 1e-9."""
    tiles = O.tile_offsets_uniform(50, [], 20)
    assert list(np.diff(tiles)) == [20, 20, 10]
    ts = list(np.diff(tiles))
    A = O.BlockTensor([ts] * 4)
    B = O.BlockTensor([ts] * 4)
    C = O.BlockTensor([ts] * 4)
    A.set(21.0)
    B.set(2.0)
    C.set(0.0)
    i, j, k, l, m, o = -1, -2, -3, -4, -5, -6
    impl = "ref" if O.ref() is not None else "port"
    O.mult_bufacc(C, [j, i, k, l], 1.0, A, [i, j, m, o], B, [m, o, k, l], impl=impl)
    assert abs(C.norm() - 2.625e8) <= 1e-9 * 2.625e8 or abs(C.norm() - 2.625e8) <= 1e-9


@pytest.mark.parametrize("case", ["3x3x3", "3x2x1", "4d"])
def test_known_answer_ops(case):
    """tests/tamm/Test_Ops.cpp:1396-1555 (check_value tolerance 1e-10): N=10, tile 1."""
    ts = [1] * 10
    if case == "3x3x3":
        T1, T2, T3 = (O.BlockTensor([ts] * 3) for _ in range(3))
        lab = ([-1, -2, -3], [-2, -4, -1], [-4, -1, -3])  # T1(i,j,k) += 1.7 T2(j,l,i) T3(l,i,k)
        want = 2 + 1.7 * 3 * 4 * 10
    elif case == "3x2x1":
        T1, T2, T3 = O.BlockTensor([ts] * 3), O.BlockTensor([ts] * 2), O.BlockTensor([ts])
        lab = ([-1, -2, -3], [-1, -2], [-3])
        want = 2 + 1.7 * 3 * 4
    else:
        T1, T2, T3 = (O.BlockTensor([ts] * 4) for _ in range(3))
        lab = ([-1, -2, -3, -4], [-2, -4, -3, -5], [-4, -1, -3, -5])  # T1(i,j,k,l) += T2(j,l,k,m) T3(l,i,k,m)
        want = 2 + 1.7 * 3 * 4 * 10
    T1.set(2.0)
    T2.set(3.0)
    T3.set(4.0)
    O.mult_bufacc(T1, lab[0], 1.7, T2, lab[1], T3, lab[2])
    assert np.max(np.abs(T1.data[:T1.total] - want)) < 1e-10


def test_known_answer_spin_tiling():
    """tests/tamm/Test_TiledIndexSpace.cpp:308-328: spin-split tiling 3,2,3,2,..."""
    bounds = [0, 10, 10, 20, 0, 5, 10, 15, 5, 10, 15, 20]
    want = [3, 2, 3, 2, 3, 2, 3, 2]
    assert list(np.diff(O.tile_offsets_uniform(20, bounds, 3))) == want
    assert list(np.diff(O.tile_offsets_list(20, bounds, want))) == want
    with pytest.raises(ValueError):
        O.tile_offsets_list(20, bounds, [4, 4, 4, 4, 4])


def test_spin_rule():
    """TensorBase::is_non_zero: sum of upper spins == sum of lower spins."""
    assert O.is_non_zero([1, 2, 1, 2], [0, 0, 1, 1])
    assert O.is_non_zero([1, 2, 2, 1], [0, 0, 1, 1])
    assert not O.is_non_zero([1, 1, 1, 2], [0, 0, 1, 1])
    assert O.is_non_zero([5, 1, 1], [2, 0, 1])  # ignore position
    assert O.is_non_zero([1, 1, 2, 2], [0, 0, 1, 1], has_spin=False)


def test_distribution_nw_order():
    """Distribution_NW: admitted blocks sorted by row-major tile key, packed."""
    t = O.BlockTensor([[3, 2, 3, 2], [2, 2]], [[1, 1, 2, 2], [1, 2]], [0, 1])
    assert list(t.keys) == [0, 2, 5, 7]  # (0,0),(1,0),(2,1),(3,1)
    assert list(t.offsets) == [0, 6, 10, 16]
    assert t.total == 20
