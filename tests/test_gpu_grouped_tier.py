"""The grouped tier of the C ABI, driven as a TAMM maintainer would bind it:
tb_plan_contraction -> tb_worklist_build -> tb_contract replace the
MultOp::execute_bufacc loop of block_multiply calls (multop.hpp:576-893).

The block stores are the oracle's Distribution_NW packings of a spin-blocked ladder
r2(a,b,i,j) += alpha * v(a,b,c,d) * t2(c,d,i,j) (uneven tiles, alpha/beta spin
blocks), copied to the device as three flat arrays; the groups (admitted output
blocks) and tasks (admitted reduction tiles c, d) are enumerated on the host here,
in Python, with offsets from the oracle's block table.  Every call goes through
ctypes.  The result must match the oracle's bufacc restatement driving the
reference's block_multiply: FP64 1e-12, split-INT8 1e-11, BF16x3 5e-5 relative to
max |r2|; tb_worklist_info must report the oracle's admitted task count and FLOPs.
"""
import ctypes as C
import itertools

import numpy as np
import pytest

from oracle import oracle as O
from tamm_b200 import _capi as A

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {A.TB_MODE_FP64: 1e-12, A.TB_MODE_INT8: 1e-11, A.TB_MODE_BF16X3: 5e-5}


def _spaces(occ, virt):
    vt, vs = list(virt) * 2, [1] * len(virt) + [2] * len(virt)
    ot, os_ = list(occ) * 2, [1] * len(occ) + [2] * len(occ)
    return (vt, vs), (ot, os_)


def _worklist(v, t2, r2, vt, ot):
    """execute_bufacc's enumeration: admitted output blocks (a,b,i,j) in loop order, and
    per block the admitted reduction tiles (c,d) in sorted-label order."""
    nv, no = len(vt), len(ot)
    c_off, cdims, begin, a_off, b_off, adims, bdims = [], [], [0], [], [], [], []
    for a, b, i, j in itertools.product(range(nv), range(nv), range(no), range(no)):
        oc = r2.locate((a, b, i, j))
        if oc < 0:
            continue
        for c, d in itertools.product(range(nv), range(nv)):
            oa, ob = v.locate((a, b, c, d)), t2.locate((c, d, i, j))
            if oa < 0 or ob < 0:
                continue
            a_off.append(oa)
            b_off.append(ob)
            adims += [vt[a], vt[b], vt[c], vt[d]]
            bdims += [vt[c], vt[d], ot[i], ot[j]]
        c_off.append(oc)
        cdims += [vt[a], vt[b], ot[i], ot[j]]
        begin.append(len(a_off))
    i64 = lambda x: np.asarray(x or [0], dtype=np.int64)  # noqa: E731
    i32 = lambda x: np.asarray(x or [0], dtype=np.int32)  # noqa: E731
    return len(c_off), i64(c_off), i32(cdims), i64(begin), i64(a_off), i64(b_off), i32(adims), i32(bdims)


@pytest.mark.parametrize("mode", [A.TB_MODE_FP64, A.TB_MODE_INT8, A.TB_MODE_BF16X3])
def test_grouped_tier_spin_ladder(mode):
    (vt, vs), (ot, os_) = _spaces([3, 2], [5, 3, 6])
    v = O.BlockTensor([vt] * 4, [vs] * 4, [0, 0, 1, 1])
    t2 = O.BlockTensor([vt, vt, ot, ot], [vs, vs, os_, os_], [0, 0, 1, 1])
    r2 = O.BlockTensor([vt, vt, ot, ot], [vs, vs, os_, os_], [0, 0, 1, 1])
    O.fill_uniform(v.data[:v.total], 11)
    O.fill_normal(t2.data[:t2.total], 12, 0, 0.0, 1e-2)
    O.fill_uniform(r2.data[:r2.total], 13)
    alpha = 0.5
    c0 = r2.data[:r2.total].copy()
    dv = torch.from_numpy(v.data[:v.total].copy()).cuda()
    dt = torch.from_numpy(t2.data[:t2.total].copy()).cuda()
    dr = torch.from_numpy(c0.copy()).cuda()

    ng, c_off, cdims, begin, a_off, b_off, adims, bdims = _worklist(v, t2, r2, vt, ot)
    lab = lambda x: np.asarray(x, dtype=np.int32)  # noqa: E731
    cl, al, bl = lab([1, 2, 5, 6]), lab([1, 2, 3, 4]), lab([3, 4, 5, 6])
    L = A.lib()
    plan, wl = A.vp(), A.vp()
    A.check(L.tb_plan_contraction(cl.ctypes.data_as(A.ip), 4, al.ctypes.data_as(A.ip), 4, bl.ctypes.data_as(A.ip),
                                  4, mode, 1e-11, 0, C.byref(plan)))
    try:
        A.check(L.tb_worklist_build(plan, ng, c_off.ctypes.data_as(A.i64p), cdims.ctypes.data_as(A.i32p),
                                    begin.ctypes.data_as(A.i64p), a_off.ctypes.data_as(A.i64p),
                                    b_off.ctypes.data_as(A.i64p), adims.ctypes.data_as(A.i32p),
                                    bdims.ctypes.data_as(A.i32p), C.byref(wl)))
        ntasks, flops = C.c_int64(), C.c_double()
        A.check(L.tb_worklist_info(wl, C.byref(ntasks), C.byref(flops)))
        want_tasks, want_flops = O.mult_count(r2, [1, 2, 5, 6], v, [1, 2, 3, 4], t2, [3, 4, 5, 6])
        assert ntasks.value == want_tasks and flops.value == want_flops
        stream = torch.cuda.current_stream().cuda_stream
        # the same work list twice: it is reusable, and C accumulates
        for _ in range(2):
            A.check(L.tb_contract(plan, wl, alpha, dv.data_ptr(), dt.data_ptr(), dr.data_ptr(), C.c_void_p(stream)))
        torch.cuda.synchronize()
        st = A.tb_stats()
        A.check(L.tb_plan_stats(plan, C.byref(st)))
        assert st.flops == want_flops and st.flops_run == want_flops
    finally:
        if wl:
            L.tb_worklist_destroy(wl)
        L.tb_plan_destroy(plan)
    O.mult_bufacc(r2, [1, 2, 5, 6], 2 * alpha, v, [1, 2, 3, 4], t2, [3, 4, 5, 6],
                  impl="ref" if O.ref() is not None else "port")
    want = r2.data[:r2.total]
    got = dr.cpu().numpy()
    err = float(np.max(np.abs(got - want))) / float(np.max(np.abs(want - c0)))
    assert err <= TOL[mode], f"mode {mode}: max rel err {err:.3e}"
