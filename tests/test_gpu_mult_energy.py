"""Contraction with the denominator energy fused into its epilogue
(Scheduler.mult_energy / tb_sched_mult_energy):

    slot += scale * sum (C + alpha * A * B)^2 / D,   D = sum_m s_m * eps[index of C mode m]

over C's stored elements, C left unchanged.  It stands for TAMM's MultOp C += alpha*A*B
(multop.hpp:576-893) followed by tb_sched_denom_energy over C, so each case checks it
against those two ops run separately on a copy of C (same precision mode), and against
a dense numpy restatement over the admitted blocks.  Cases cover both split-INT8
epilogue layouts (C's last mode a column label: transposed loads; a row label: row
loads) and output blocks whose tasks all fall on exactly-zero blocks of a read-only
operand (no tasks: those blocks enter with their stored values).  Bars against numpy:
FP64 1e-12, split-INT8 1e-10, BF16x3 1e-5 relative to |E|; against the separate ops:
1e-13 (the same products, summed in another order)."""
import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W

pytestmark = pytest.mark.gpu

OA, VA = 3, 10


def _dense(t):
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
        sl = tuple(slice(int(tofs[m][bid[m]]), int(tofs[m][bid[m]]) + dims[m]) for m in range(len(dims)))
        out[sl] = data[off:off + int(np.prod(dims))].reshape(dims)
    return out


def _spaces():
    is_ = W.mo_index_space(OA, VA)
    mo = tb.TiledIndexSpace(is_, 4)  # tiles cut at the spin boundaries: occ 3 3, virt 4 4 2 4 4 2
    return mo("occ"), mo("virt")


def _fill(t, seed, zero_beta_first=False):
    rng = np.random.default_rng(seed)
    no = 2 * OA

    def f(bid, dims, rg):
        if zero_beta_first and rg[0][0] >= no + VA:  # first mode a beta virtual: an exactly-zero block
            return np.zeros(dims)
        return rng.uniform(-1.0, 1.0, size=dims)
    t.write(W.fill_blocks(t, f))


def _eps():
    e_occ, e_virt = W.orbital_energies(OA, VA, 5)
    return np.concatenate([e_occ, e_occ, e_virt, e_virt])


# (C modes, A modes, B modes, C spin, A spin, B spin); o: occupied, v: virtual
CASES = {
    # C(a,b,i,j) += A(a,c,i,k) B(c,b,k,j): C's last mode j is a column label
    "ladder_like": ("abij", "acik", "cbkj", (2, 2), (2, 2), (2, 2)),
    # C(a,b,i,j) += X(a,j,c) Y(c,b,i): j is a row label
    "rows_last": ("abij", "ajc", "cbi", (2, 2), None, None),
}
OCC = set("ijkl")


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("mode,tol", [(tb.Precision.FP64, 1e-12), (tb.Precision.INT8, 1e-10),
                                      (tb.Precision.BF16X3, 1e-5)])
@pytest.mark.parametrize("zero_blocks", [False, True])
def test_mult_energy(ec, case, mode, tol, zero_blocks):
    cm, am, bm, cs, as_, bs = CASES[case]
    O, V = _spaces()
    sp = lambda m: O if m in OCC else V
    kw = lambda s: {} if s is None else {"spin": s}
    Ct = tb.Tensor([sp(m) for m in cm], **kw(cs)).allocate(ec)
    C2 = tb.Tensor([sp(m) for m in cm], **kw(cs)).allocate(ec)
    At = tb.Tensor([sp(m) for m in am], **kw(as_)).allocate(ec)
    Bt = tb.Tensor([sp(m) for m in bm], **kw(bs)).allocate(ec)
    try:
        _fill(Ct, 1)
        _fill(At, 2, zero_beta_first=zero_blocks)
        _fill(Bt, 3)
        if zero_blocks:  # read-only: tasks over its zero blocks are dropped, some outputs keep none
            At.set_read_only(True)
        C2.write(Ct.read())
        c0 = Ct.read()
        eps = _eps()
        signs = [1.0 if m in OCC else -1.0 for m in cm]
        lab = {}
        for m in sorted(set(cm + am + bm)):
            lab[m] = sp(m).label()
        L = lambda t, ms: t(*[lab[m] for m in ms])
        alpha, scale = -0.7, 0.25
        ec.set_precision(mode, 1e-11)
        sch = tb.Scheduler(ec)
        sch.set_scalar(0, 0.0).set_scalar(1, 0.0)
        sch.mult_energy(0, scale, L(Ct, cm).iadd(alpha * L(At, am) * L(Bt, bm)), eps, signs)
        sch(L(C2, cm).iadd(alpha * L(At, am) * L(Bt, bm)))
        sch.denom_energy(1, scale, L(C2, cm), eps, signs)
        sch.execute()
        e_fused, e_sep = (float(x) for x in sch.scalars(2)[:2])
        assert np.array_equal(Ct.read(), c0), "the energy epilogue wrote C"
        # dense restatement over the admitted blocks
        Cd, Ad, Bd = _dense(Ct), _dense(At), _dense(Bt)
        full = Cd + alpha * np.einsum(f"{am},{bm}->{cm}", Ad, Bd)
        mask = _dense(C2) != 0  # admitted positions (random values, never exactly zero)
        D = np.zeros(full.shape)
        for pos, m in enumerate(cm):  # dense positions count from the start of each subspace
            shape = [1] * len(cm)
            shape[pos] = -1
            e = eps[:2 * OA] if m in OCC else eps[2 * OA:]
            D = D + (1.0 if m in OCC else -1.0) * e.reshape(shape)
        want = scale * float(np.sum(np.where(mask, full * full / D, 0.0)))
        assert abs(e_fused - want) <= tol * abs(want), f"fused {e_fused!r} vs numpy {want!r}"
        assert abs(e_fused - e_sep) <= 1e-13 * abs(e_sep), f"fused {e_fused!r} vs separate ops {e_sep!r}"
    finally:
        ec.set_precision(tb.Precision.FP64)
        for t in (Ct, C2, At, Bt):
            t.deallocate()
