"""A coupled-cluster doubles-residual iteration on the device, in one Scheduler op
list that can be captured into a CUDA graph.

The term list follows the structure of the CD-CCSD doubles residual of TAMM's
CCSD test driver (tests/tamm/Test_CCSD.cpp:168-582): Fock-dressed one-body
intermediates, a hole-hole ladder with its quadratic intermediate, ring terms
through an (ov|vo) intermediate with the four P(ab)P(ij) permutations, and the
particle-particle ladder with v(a,b,c,d) built on demand from Cholesky vectors,
as TAMM builds it with a lambda tensor (Test_CCSD.cpp:300-488):

    F_vv(b,c)   = f_vv(b,c) - 1/2 v(c,d,k,l) t2(b,d,k,l)
    F_oo(k,j)   = f_oo(k,j) + 1/2 v(c,d,k,l) t2(c,d,j,l)
    W_oo(k,l,i,j) = 1/2 v_oooo(k,l,i,j) + 1/4 v(c,d,k,l) t2(c,d,i,j)
    W_ov(k,b,c,j) = v_ovvo(k,b,c,j) + 1/2 v(c,d,k,l) t2(d,b,l,j)
    r2(a,b,i,j) = v(a,b,i,j) + F_vv(b,c) t2(a,c,i,j) - F_vv(a,c) t2(b,c,i,j)
                - F_oo(k,j) t2(a,b,i,k) + F_oo(k,i) t2(a,b,j,k) + W_oo(k,l,i,j) t2(a,b,k,l)
                + P(ab) P(ij) [t2(a,c,i,k) W_ov(k,b,c,j)]
                + 1/2 sum_cd [sum_Q L(Q,a,c) L(Q,b,d)] t2(c,d,i,j)
    E = 1/4 v(a,b,i,j) t2(a,b,i,j),  |r2|,  t2 -= r2 / (e_a + e_b - e_i - e_j)

with v(a,b,i,j) = sum_Q L(Q,a,i) L(Q,b,j) (and v(c,d,k,l) the same tensor read as
(oo|vv)), v_oooo and v_ovvo likewise from the Cholesky vectors.  Every tensor is
spin-blocked with TAMM's sum rule.  v(a,b,c,d) is a lambda tensor built on demand
(tb_tensor_create_built): the ladder is one op, r2 += 1/2 v(a,b,c,d) t2(c,d,i,j), and
the scheduler runs it in batches of the virtual tiles of a, each batch
v(a',b,c,d) = L(Q,a',c) L(Q,b,d) materialised into scratch, contracted and released,
so v is never stored whole.

    python -m tamm_b200.ccsd [--oa 30 --va 240 --seed 2 --tile-lo 20 --tile-hi 64]
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from .tamm import (ExecutionContext, ExecutionHW, IndexSpace, Precision, Scheduler, Tensor, TiledIndexSpace,
                   mult_info)

SLOT_ENERGY, SLOT_NORM = 0, 1


@dataclass
class CCSDProblem:
    ec: ExecutionContext
    MO: TiledIndexSpace
    O: TiledIndexSpace
    V: TiledIndexSpace
    CI: TiledIndexSpace
    eps: np.ndarray                     # orbital energies over the MO space
    T: dict                             # name -> Tensor (v_vvvv: the lambda tensor)
    ladder_batches: int                 # batches the particle ladder runs in
    flops: dict = field(default_factory=dict)


def _fill(t: Tensor, fn, seed: int):
    rng = np.random.default_rng(seed)
    t.write(W.fill_blocks(t, lambda bid, dims, rg: fn(rng, bid, dims, rg)))


def build(oa: int, va: int, seed: int = 2, tile_lo: int = 20, tile_hi: int = 64, nchol=None,
          ec: ExecutionContext | None = None, batch_tiles: int = 1) -> CCSDProblem:
    """Allocates and fills everything one iteration needs (integrals from Cholesky
    vectors, Fock matrices with small off-diagonal couplings, MP2 amplitudes)."""
    import torch
    rng = np.random.default_rng(seed)
    occ_t = W.random_tiles(oa, tile_lo, tile_hi, rng)
    virt_t = W.random_tiles(va, tile_lo, tile_hi, rng)
    MO = W.mo_tiled(oa, va, occ_t, virt_t)
    O, V = MO("occ"), MO("virt")
    ec = ec or ExecutionContext(0, 0)
    sch = Scheduler(ec)
    e_occ, e_virt = W.orbital_energies(oa, va, seed)
    eps = np.concatenate([e_occ, e_occ, e_virt, e_virt])
    Q = nchol if nchol is not None else 5 * (2 * oa + 2 * va)
    CI = TiledIndexSpace(IndexSpace(Q), 1000)
    T = {}

    def new(name, spaces, **kw):
        T[name] = Tensor(spaces, **kw).allocate(ec)
        return T[name]

    # Cholesky vectors L(Q,p,q) ~ N(0,1)/sqrt(Q) exp(-|p-q|/50), nonzero for spin(p) == spin(q)
    def chol(bid, dims, rg, rng):
        ip = np.arange(rg[1][0], rg[1][1])[:, None]
        iq = np.arange(rg[2][0], rg[2][1])[None, :]
        return rng.normal(0.0, 1.0, size=dims) / math.sqrt(Q) * np.exp(-np.abs(ip - iq) / 50.0)[None]

    for name, (s1, s2), sd in (("L_vo", (V, O), 11), ("L_oo", (O, O), 12), ("L_vv", (V, V), 13)):
        _fill(new(name, [CI, s1, s2], spin_mask=[2, 0, 1]), lambda r, b, d, g: chol(b, d, g, r), seed + sd)

    # Fock matrices: orbital energies on the diagonal, 1e-3 couplings between same-spin orbitals
    def fock(rng, bid, dims, rg):
        ip = np.arange(rg[0][0], rg[0][1])[:, None]
        iq = np.arange(rg[1][0], rg[1][1])[None, :]
        off = 1e-3 * rng.normal(0.0, 1.0, size=dims)
        return np.where(ip == iq, eps[np.clip(ip, 0, len(eps) - 1)] + 0 * iq, off)

    _fill(new("f_oo", [O, O], spin=(1, 1)), fock, seed + 21)
    _fill(new("f_vv", [V, V], spin=(1, 1)), fock, seed + 22)
    for name, sp in (("v_vvoo", [V, V, O, O]), ("t2", [V, V, O, O]), ("r2", [V, V, O, O]), ("X", [V, V, O, O]),
                     ("v_oooo", [O, O, O, O]), ("W_oo", [O, O, O, O]), ("v_ovvo", [O, V, V, O]),
                     ("W_ov", [O, V, V, O])):
        new(name, sp, spin=(2, 2))
    new("F_vv", [V, V], spin=(1, 1))
    new("F_oo", [O, O], spin=(1, 1))
    q = CI.label()
    a, b, c, d = V.labels(4)
    i, j, k, l = O.labels(4)
    Lvo, Loo = T["L_vo"], T["L_oo"]
    sch(T["v_vvoo"](a, b, i, j).assign(Lvo(q, a, i) * Lvo(q, b, j)))
    sch(T["v_oooo"](k, l, i, j).assign(Loo(q, k, i) * Loo(q, l, j)))
    sch(T["v_ovvo"](k, b, c, j).assign(Lvo(q, c, k) * Lvo(q, b, j)))
    # MP2 amplitudes: t2 = -v / (e_a + e_b - e_i - e_j)
    sch(T["t2"]().assign(0.0))
    sch.denom(T["t2"](a, b, i, j), -1.0, T["v_vvoo"](a, b, i, j), eps, [1, 1, -1, -1])
    sch.execute(ExecutionHW.GPU)
    # v(a,b,c,d) built on demand in batches of the virtual tiles of a, `batch_tiles`
    # tiles' worth of blocks per batch
    q2 = CI.label()

    def build_batch(batch, first, last, bsch):
        ap = batch.spaces[0].label()
        b2, c2, d2 = V.labels(3)
        bsch(batch(ap, b2, c2, d2).assign(T["L_vv"](q2, ap, c2) * T["L_vv"](q2, b2, d2)))

    shape = Tensor([V, V, V, V], spin=(2, 2))  # host-only: the block table of v
    keys, offs = shape.block_table()
    stride = V.num_tiles ** 3
    per_tile = np.zeros(V.num_tiles, dtype=np.int64)
    ends = np.append(offs[1:], shape.nelems)
    for k, o, e in zip(keys.tolist(), offs.tolist(), ends.tolist()):
        per_tile[k // stride] += e - o
    batch_bytes = 8 * int(max(per_tile[x:x + batch_tiles].sum() for x in range(V.num_tiles)))
    T["v_vvvv"] = Tensor.built([V, V, V, V], build_batch, spin=(2, 2), batch_bytes=batch_bytes)
    nb, acc = 0, None
    for x in range(V.num_tiles):  # the scheduler's greedy cut of the first mode's tiles
        if acc is None or acc + 8 * per_tile[x] > batch_bytes:
            nb, acc = nb + 1, 8 * int(per_tile[x])
        else:
            acc += 8 * int(per_tile[x])
    # the integrals and Fock matrices stay constant through the iterations: marked
    # read-only, their exactly-zero spin blocks (e.g. v(a,b,i,j) with spin(a) != spin(i))
    # are skipped by the contractions that read them
    for name in ("L_vo", "L_oo", "L_vv", "f_oo", "f_vv", "v_vvoo", "v_oooo", "v_ovvo"):
        T[name].set_read_only(True)
    P = CCSDProblem(ec, MO, O, V, CI, eps, T, nb)
    P.flops = iteration_flops(P)
    return P


def _ops(P: CCSDProblem):
    """The iteration as (kind, lhs, alpha, factors, is_assign) entries."""
    T, (a, b, c, d), (i, j, k, l) = P.T, P.V.labels(4), P.O.labels(4)
    q = P.CI.label()
    t2, v, r2, X = T["t2"], T["v_vvoo"], T["r2"], T["X"]
    ops = [
        (T["F_vv"](b, c), 1.0, [T["f_vv"](b, c)], True),
        (T["F_vv"](b, c), -0.5, [v(c, d, k, l), t2(b, d, k, l)], False),
        (T["F_oo"](k, j), 1.0, [T["f_oo"](k, j)], True),
        (T["F_oo"](k, j), 0.5, [v(c, d, k, l), t2(c, d, j, l)], False),
        (T["W_oo"](k, l, i, j), 0.5, [T["v_oooo"](k, l, i, j)], True),
        (T["W_oo"](k, l, i, j), 0.25, [v(c, d, k, l), t2(c, d, i, j)], False),
        (T["W_ov"](k, b, c, j), 1.0, [T["v_ovvo"](k, b, c, j)], True),
        (T["W_ov"](k, b, c, j), 0.5, [v(c, d, k, l), t2(d, b, l, j)], False),
        (r2(a, b, i, j), 1.0, [v(a, b, i, j)], True),
        (r2(a, b, i, j), 1.0, [T["F_vv"](b, c), t2(a, c, i, j)], False),
        (r2(a, b, i, j), -1.0, [T["F_vv"](a, c), t2(b, c, i, j)], False),
        (r2(a, b, i, j), -1.0, [T["F_oo"](k, j), t2(a, b, i, k)], False),
        (r2(a, b, i, j), 1.0, [T["F_oo"](k, i), t2(a, b, j, k)], False),
        (r2(a, b, i, j), 1.0, [T["W_oo"](k, l, i, j), t2(a, b, k, l)], False),
        (X(a, b, i, j), 1.0, [t2(a, c, i, k), T["W_ov"](k, b, c, j)], True),
        (r2(a, b, i, j), 1.0, [X(a, b, i, j)], False),
        (r2(a, b, i, j), -1.0, [X(b, a, i, j)], False),
        (r2(a, b, i, j), -1.0, [X(a, b, j, i)], False),
        (r2(a, b, i, j), 1.0, [X(b, a, j, i)], False),
    ]
    ops.append((r2(a, b, i, j), 0.5, [T["v_vvvv"](a, b, c, d), t2(c, d, i, j)], False))
    return ops


def iteration_flops(P: CCSDProblem) -> dict:
    """Admitted FP64 FLOPs of the iteration's contractions, with the particle ladder and
    the on-demand build of its integrals v(a,b,c,d) = L(Q,a,c) L(Q,b,d) listed apart."""
    total, ladder = 0.0, 0.0
    ops = _ops(P)
    for n, (lhs, _, f, _) in enumerate(ops):
        if len(f) == 2:
            fl = mult_info(lhs, f[0], f[1])[2]
            total += fl
            if n == len(ops) - 1:
                ladder = fl
    a, b, c, d = P.V.labels(4)
    q = P.CI.label()
    shape = Tensor([P.V, P.V, P.V, P.V], spin=(2, 2))
    build = mult_info(shape(a, b, c, d), P.T["L_vv"](q, a, c), P.T["L_vv"](q, b, d))[2]
    return {"contractions": total + build, "ladder": ladder, "v_build": build}


def queue_iteration(P: CCSDProblem, sch: Scheduler):
    """Queues one iteration: residual, energy (slot 0), residual norm (slot 1) and the
    denominator update of t2."""
    for lhs, alpha, f, assign in _ops(P):
        rhs = alpha * f[0] if len(f) == 1 else alpha * f[0] * f[1]
        sch(lhs.assign(rhs) if assign else lhs.iadd(rhs))
    T = P.T
    a, b = P.V.labels(2)
    i, j = P.O.labels(2)
    sch.dot(SLOT_ENERGY, T["v_vvoo"](a, b, i, j), T["t2"](a, b, i, j), 0.25)
    sch.norm(SLOT_NORM, T["r2"](a, b, i, j))
    sch.denom(T["t2"](a, b, i, j), -1.0, T["r2"](a, b, i, j), P.eps, [1, 1, -1, -1])
    return sch


def tune_report(sch: Scheduler) -> list:
    """Autotuner choices (or None) of every op of the scheduler's last execute."""
    from ._capi import TambError
    out, x = [], 0
    while True:
        try:
            out.append(sch.tune_info(x))
        except TambError:
            return out
        x += 1


def measure(P: CCSDProblem, iters: int = 3, modes=("fp64", "int8")) -> dict:
    """Eager and graph-replayed iterations in the plain FP64 and split-INT8 (autotuned)
    modes, timed by CUDA events on the context's stream; t2 is restored before each
    mode so every mode iterates from the same amplitudes."""
    import torch
    ec = P.ec
    t2_0 = P.T["t2"].read().copy()
    stream = torch.cuda.ExternalStream(ec.stream)
    results, r2s = {}, {}
    table = {"fp64": (Precision.FP64, False), "int8": (Precision.INT8, True), "bf16x3": (Precision.BF16X3, False)}
    for name in modes:
        mode, tune = table[name]
        ec.set_precision(mode, 1e-11)
        P.T["t2"].write(t2_0)
        sch = Scheduler(ec)
        if tune:
            sch.autotune(True)
        queue_iteration(P, sch)
        t0 = time.perf_counter()
        sch.execute(ExecutionHW.GPU)  # first iteration: plans, work lists, autotuning
        first_s = time.perf_counter() - t0
        e_first, n_first = sch.scalars(2)
        # eager iteration (host-driven op launches), profiled per op
        P.T["t2"].write(t2_0)
        queue_iteration(P, sch)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sch.execute(ExecutionHW.GPU)
        e1.record(stream)
        e1.synchronize()
        eager_ms = e0.elapsed_time(e1)
        # graph: capture once, replay
        P.T["t2"].write(t2_0)
        queue_iteration(P, sch)
        g = sch.graph()  # runs the iteration once, then captures it
        P.T["t2"].write(t2_0)
        g.launch().sync()
        e_graph, n_graph = sch.scalars(2)
        r2s[name] = P.T["r2"].read().copy()
        e0.record(stream)
        for _ in range(iters):
            g.launch()
        e1.record(stream)
        g.sync()
        graph_ms = e0.elapsed_time(e1) / iters
        results[name] = {"energy_first": e_first, "residual_norm_first": n_first, "energy_graph": e_graph,
                         "first_iteration_s": first_s, "eager_ms": eager_ms, "graph_ms": graph_ms,
                         "graph_replays": iters, "tflops_graph": P.flops["contractions"] / graph_ms / 1e9}
        if tune:
            choices = {}
            for ti in tune_report(sch):
                if ti:
                    key = "fp64" if ti["mode"] == Precision.FP64 else f"int8_nt{ti['tile_n']}"
                    choices[key] = choices.get(key, 0) + 1
            results[name]["autotune_choices"] = choices
        del g
    ec.set_precision(Precision.FP64)
    P.T["t2"].write(t2_0)
    if "fp64" in r2s:
        scale = max(float(np.max(np.abs(r2s["fp64"]))), 1e-300)
        for name in r2s:
            if name != "fp64":
                results[name]["r2_max_rel_err_vs_fp64"] = float(np.max(np.abs(r2s[name] - r2s["fp64"]))) / scale
                results[name]["speedup_vs_fp64"] = results["fp64"]["graph_ms"] / results[name]["graph_ms"]
    return results


def main(argv=None):
    """Config of the full doubles iteration: eager and graph-replayed iterations in the
    plain FP64 and split-INT8 (autotuned) modes; prints one JSON line."""
    p = argparse.ArgumentParser()
    p.add_argument("--oa", type=int, default=30)
    p.add_argument("--va", type=int, default=240)
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--tile-lo", type=int, default=20)
    p.add_argument("--tile-hi", type=int, default=64)
    p.add_argument("--iters", type=int, default=3)
    p.add_argument("--pool-gib", type=int, default=150)
    p.add_argument("--modes", default="fp64,int8")
    args = p.parse_args(argv)
    ec = ExecutionContext(0, args.pool_gib << 30)
    P = build(args.oa, args.va, seed=args.seed, tile_lo=args.tile_lo, tile_hi=args.tile_hi, ec=ec)
    out = {"workload": f"ccsd_doubles_iteration_O{2 * args.oa}_V{2 * args.va}", "flops": P.flops,
           "ops_per_iteration": len(_ops(P)) + 3, "ladder_batches": P.ladder_batches}
    out.update(measure(P, args.iters, tuple(args.modes.split(","))))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
