"""Triples-style 6-index contraction streamed over occupied pairs, reduced into an
FP64 energy without storing t3:

    W(a,b,c,i,j,k) = sum_d t2(a,d,i,j) v(b,c,d,k) - sum_l t2(a,b,i,l) v(l,c,j,k)
    E = sum W^2 / (e_i + e_j + e_k - e_a - e_b - e_c)

on the spin-blocked MO space of the ladder (v from Cholesky vectors, t2 from the
orbital-energy denominators).  TAMM has no (T) code of its own (it lives in the
applications built on it); the contractions are TAMM MultOps and the reduction is
the denominator-energy op of this library.

Streaming: a t3 block of one tile tuple holds tile^6 values (4e9 at tile 40), so W
is formed one step at a time, a step being one occupied index i and one block of
`jtile` occupied indices j: W(a,b,c,k) for that (i, j-block) is one contraction
over d into a shared buffer (a fused assignment: the kernel stores), minus one over
l, then slot += sum W^2 / D.  With `fused=True` the energy instead runs in the
epilogue of the contraction over d (Scheduler.mult_energy), after W = -t2.v over l:
each element W + t2.v is formed in registers, squared, divided by D and summed, so W
is written once and read once.  Both give the same energy up to summation order;
the separate ops are the default, being the faster on a B200 (both contraction
kernels are bound by their per-tile epilogue here, not by the bytes of W).
The streamed labels need finer occupied tiles (i single, j in blocks of jtile)
while the summed l keeps the uniform tiles, so t2 is held in two tilings
(t2(a,d,i,j) with i single and j blocked; t2(a,b,i,l) with l uniform) and v(l,c,j,k)
with j blocked; both t2 copies come from one dense array, so they hold the same
values.  v(b,c,d,k) is stored as (b,c,k,d) so that the summed d is contiguous, and
the summed d has its own tiling (`dtile`, default one tile per spin block): a task
then contracts over the whole spin block instead of one 40-wide tile.

    python -m tamm_b200.triples [--oa 25 --va 250 --tile 40 --jtile 2 --dtile 250 --seed 4 --steps 8]
"""
from __future__ import annotations

import argparse
import json
import math
from dataclasses import dataclass

import numpy as np

from . import workloads as W
from .tamm import (ExecutionContext, ExecutionHW, IndexSpace, Precision, Scheduler, Tensor, TiledIndexSpace,
                   _device_array, mult_info)

SLOT_E = 2


@dataclass
class TriplesProblem:
    ec: ExecutionContext
    V: TiledIndexSpace     # virtual, uniform tiles
    Ob: TiledIndexSpace    # occupied, uniform tiles (summed l, streamed-in k)
    O1: TiledIndexSpace    # occupied, one index per tile (streamed i)
    Oj: TiledIndexSpace    # occupied, blocks of jtile indices (streamed j)
    Vd: TiledIndexSpace    # virtual, tiling of the summed d
    eps: np.ndarray
    T: dict
    buffer: int            # device address of the W storage, from the context's arena
    most: int

    def release(self):
        """Returns the W storage to the context's arena."""
        if self.buffer:
            self.ec.free(self.buffer)
            self.buffer = 0


def _dense_t2(oa, va, eps, seed):
    """t2(a,b,i,j) ~ N(0, 0.1^2) / (e_a + e_b - e_i - e_j) on the full (virt, virt, occ, occ)
    ranges, zero outside the spin-conserving blocks."""
    no, nv = 2 * oa, 2 * va
    rng = np.random.default_rng(seed + 7)
    eo, ev = eps[:no], eps[no:]
    so = np.array([0] * oa + [1] * oa)
    sv = np.array([0] * va + [1] * va)
    t = rng.normal(0.0, 0.1, size=(nv, nv, no, no))
    t /= ev[:, None, None, None] + ev[None, :, None, None] - eo[None, None, :, None] - eo[None, None, None, :]
    ok = (sv[:, None, None, None] + sv[None, :, None, None]) == (so[None, None, :, None] + so[None, None, None, :])
    return t * ok


def build(oa: int, va: int, tile: int = 40, jtile: int = 2, dtile: int = 0, seed: int = 4, nchol=None,
          ec: ExecutionContext | None = None):
    is_ = W.mo_index_space(oa, va)
    MOb = TiledIndexSpace(is_, tile)
    MO1 = TiledIndexSpace(is_, 1)
    MOj = TiledIndexSpace(is_, jtile)
    MOd = TiledIndexSpace(is_, dtile if dtile > 0 else va)
    V, Ob, O1, Oj, Vd = MOb("virt"), MOb("occ"), MO1("occ"), MOj("occ"), MOd("virt")
    ec = ec or ExecutionContext(0, 0)
    e_occ, e_virt = W.orbital_energies(oa, va, seed)
    eps = np.concatenate([e_occ, e_occ, e_virt, e_virt])
    no = 2 * oa
    Q = nchol if nchol is not None else 5 * (2 * oa + 2 * va)
    CI = TiledIndexSpace(IndexSpace(Q), 1000)
    T = {}

    def new(name, spaces, **kw):
        T[name] = Tensor(spaces, **kw).allocate(ec)
        return T[name]

    def chol(seed_):
        rng = np.random.default_rng(seed_)

        def f(bid, dims, rg):
            ip = np.arange(rg[1][0], rg[1][1])[:, None]
            iq = np.arange(rg[2][0], rg[2][1])[None, :]
            return rng.normal(0.0, 1.0, size=dims) / math.sqrt(Q) * np.exp(-np.abs(ip - iq) / 50.0)[None]
        return f

    for name, (s1, s2), sd in (("L_vv", (V, Vd), 13), ("L_vo", (V, Ob), 11), ("L_oo", (Ob, Oj), 12)):
        t = new(name, [CI, s1, s2], spin_mask=[2, 0, 1])
        t.write(W.fill_blocks(t, chol(seed + sd)))
    dense = _dense_t2(oa, va, eps, seed)
    for name, sp in (("t2x", [V, Vd, O1, Oj]), ("t2y", [V, V, O1, Ob])):
        t = new(name, sp, spin=(2, 2))
        t.write(W.fill_blocks(t, lambda bid, dims, rg: dense[rg[0][0] - no:rg[0][1] - no, rg[1][0] - no:rg[1][1] - no,
                                                            rg[2][0]:rg[2][1], rg[3][0]:rg[3][1]]))
    del dense
    new("vx", [V, V, Ob, Vd], spin=(2, 2))   # v(b,c,d,k) = sum_Q L(Q,b,d) L(Q,c,k), stored (b,c,k,d)
    new("vy", [Ob, V, Oj, Ob], spin=(2, 2))  # v(l,c,j,k) = sum_Q L(Q,l,j) L(Q,c,k)
    q = CI.label()
    b, c = V.labels(2)
    (d,) = Vd.labels(1)
    k, l = Ob.labels(2)
    (j,) = Oj.labels(1)
    sch = Scheduler(ec)
    sch(T["vx"](b, c, k, d).assign(T["L_vv"](q, b, d) * T["L_vo"](q, c, k)))
    sch(T["vy"](l, c, j, k).assign(T["L_oo"](q, l, j) * T["L_vo"](q, c, k)))
    sch.execute(ExecutionHW.GPU)
    # constant through the streamed steps: marked read-only, the exactly-zero spin
    # blocks of the integrals (e.g. vx(b,c,k,d) with spin(b) != spin(d)) are skipped
    for t in T.values():
        t.set_read_only(True)
    most = 0  # the W layout depends on the spin of i and on the j block
    for i in (0, oa):
        for jt in range(Oj.num_tiles):
            most = max(most, _w_tensor(V, O1, Oj, Ob, i, jt).nelems)
    return TriplesProblem(ec, V, Ob, O1, Oj, Vd, eps, T, ec.alloc(most * 8), most)


def _w_tensor(V, O1, Oj, Ob, i, jt):
    return Tensor([V, V, V, O1.sub(i, i + 1), Oj.sub(jt, jt + 1), Ob], spin=(3, 3))


def steps(P: TriplesProblem):
    """All streaming steps: (occupied index i, tile index of the j block)."""
    return [(i, jt) for i in range(P.O1.num_tiles) for jt in range(P.Oj.num_tiles)]


def queue_pair(P: TriplesProblem, sch: Scheduler, i: int, jt: int, fused: bool = False):
    """Queues W(a,b,c,k) for occupied index i and j block jt, and slot SLOT_E +=
    sum W^2 / D (fused: in the epilogue of the contraction over d, W then holding only
    the term over l afterwards).  Returns (W tensor, FP64 FLOPs of the two contractions)."""
    Wt = _w_tensor(P.V, P.O1, P.Oj, P.Ob, i, jt)
    Wt.attach(P.ec, P.buffer, P.most * 8)
    a, b, c = P.V.labels(3)
    (d,) = P.Vd.labels(1)
    k, l = P.Ob.labels(2)
    li, lj = Wt.spaces[3].label(), Wt.spaces[4].label()
    T = P.T
    w = Wt(a, b, c, li, lj, k)
    x = (w, T["vx"](b, c, k, d), T["t2x"](a, d, li, lj))
    y = (w, T["t2y"](a, b, li, l), T["vy"](l, c, lj, k))
    signs = [-1, -1, -1, 1, 1, 1]
    if fused:
        sch(w.assign(-1.0 * y[1] * y[2]))
        sch.mult_energy(SLOT_E, 1.0, w.iadd(x[1] * x[2]), P.eps, signs)
    else:
        sch(w.assign(x[1] * x[2]))
        sch(w.isub(y[1] * y[2]))
        sch.denom_energy(SLOT_E, 1.0, Wt(a, b, c, li, lj, k), P.eps, signs)
    return Wt, mult_info(*x)[2] + mult_info(*y)[2]


def energy(P: TriplesProblem, pairs, sch: Scheduler, release_every: int = 8, fused: bool = False):
    """E summed over the given steps (i, j block); returns (E, FP64 FLOPs, device ms).

    The steps are enqueued back to back (tb_sched_execute_async): the host builds the
    next step's work lists while the device runs the current one, and the device time
    is that of the whole sample, one pair of CUDA events around it.  The cached plans
    and work lists of finished steps (they never recur) are dropped every
    `release_every` steps, after the device has finished them."""
    import torch
    stream = torch.cuda.ExternalStream(P.ec.stream)
    sch.set_scalar(SLOT_E, 0.0).execute()
    flops, keep = 0.0, []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for n, (i, j) in enumerate(pairs):
        Wt, fl = queue_pair(P, sch, i, j, fused)
        keep.append(Wt)
        sch.execute_async()
        flops += fl
        if (n + 1) % release_every == 0 and n + 1 < len(pairs):
            sch.wait()
            sch.release()
            for t in keep:
                t.deallocate()
            keep = []
    e1.record(stream)
    sch.wait()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    sch.release()
    for t in keep:
        t.deallocate()
    return float(sch.scalars(SLOT_E + 1)[SLOT_E]), flops, ms


def main(argv=None):
    """Sampled full-size run: FP64 and split-INT8 energies and times over a seeded
    sample of streaming steps, the full run extrapolated, and the INT8 W of one step
    compared element by element with the FP64 one on the device."""
    import torch
    p = argparse.ArgumentParser()
    p.add_argument("--oa", type=int, default=25)
    p.add_argument("--va", type=int, default=250)
    p.add_argument("--tile", type=int, default=40)
    p.add_argument("--jtile", type=int, default=2)
    p.add_argument("--dtile", type=int, default=0, help="tiling of the summed d (0: one tile per spin block)")
    p.add_argument("--seed", type=int, default=4)
    p.add_argument("--steps", type=int, default=8)
    p.add_argument("--pool-gib", type=int, default=80)
    p.add_argument("--fuse", action="store_true",
                   help="energy fused into the epilogue of the contraction over d (Scheduler.mult_energy)")
    p.add_argument("--digit-cache-gib", type=int, default=16,
                   help="split-INT8 digits of the read-only integrals kept across contractions (0: off)")
    args = p.parse_args(argv)
    ec = ExecutionContext(0, args.pool_gib << 30)
    ec.set_digit_cache(args.digit_cache_gib << 30)
    P = build(args.oa, args.va, tile=args.tile, jtile=args.jtile, dtile=args.dtile, seed=args.seed, ec=ec)
    allsteps = steps(P)
    rng = np.random.default_rng(args.seed + 5)
    sample = [allsteps[int(x)] for x in rng.choice(len(allsteps), size=min(args.steps, len(allsteps)), replace=False)]
    out = {"workload": f"triples_energy_O{2 * args.oa}_V{2 * args.va}_tile{args.tile}_jtile{args.jtile}_dtile{args.dtile}",
           "sampled_steps": sample, "steps_total": len(allsteps), "fused_energy": args.fuse}
    res, wref = {}, None
    for name, mode in (("fp64", Precision.FP64), ("int8", Precision.INT8)):
        ec.set_precision(mode, 1e-11)
        sch = Scheduler(ec)
        energy(P, sample[:1], sch, fused=args.fuse)  # warm-up: kernels, digit layouts
        e, fl, ms = energy(P, sample, sch, fused=args.fuse)
        res[name] = {"energy_sample": e, "flops_sample": fl, "ms": ms, "tflops": fl / ms / 1e9,
                     "full_run_s_extrapolated": ms / len(sample) * len(allsteps) / 1e3}
        # W of the first sampled step (both terms: the unfused ops), kept on the device
        Wt, _ = queue_pair(P, sch, *sample[0], fused=False)
        sch.execute(ExecutionHW.GPU)
        wv = _device_array(P.buffer, Wt.nelems, ec.device)
        if wref is None:
            wref = wv.clone()
        else:  # chunked, to keep temporaries small
            dmax, rmax, ch = 0.0, 0.0, 1 << 27
            for o in range(0, wv.numel(), ch):
                dmax = max(dmax, float((wv[o:o + ch] - wref[o:o + ch]).abs().max()))
                rmax = max(rmax, float(wref[o:o + ch].abs().max()))
            out["int8_vs_fp64_W_max_rel_err"] = dmax / rmax
        Wt.deallocate()
    ec.set_precision(Precision.FP64)
    out.update(res)
    out["int8_vs_fp64_energy_rel_err"] = abs(res["int8"]["energy_sample"] - res["fp64"]["energy_sample"]) / abs(
        res["fp64"]["energy_sample"])
    print(json.dumps(out))


if __name__ == "__main__":
    main()
