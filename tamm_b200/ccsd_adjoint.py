"""Gradient of a coupled-cluster energy functional with respect to the amplitudes,
at full size, on one GPU:

    E(t2) = sum w(i,j,a,b) t2(a,b,i,j) + 1/4 sum t2(a,b,i,j) [v(a,b,c,d) t2(c,d,i,j)]
    dE/dt2 = w(i,j,a,b) + 1/4 v.t2 + 1/4 sum_ab v(a,b,c,d) t2(a,b,i,j)

O = 2*oa, V = 2*va spin-blocked (default O=30, V=240), v from Cholesky vectors and t2
from orbital-energy denominators as in the ladder, w ~ N(0,1)/sqrt(O*V).  For the
FP64 and split-INT8 modes it reports E, the wall time of one energy + gradient
evaluation through the tape (forward contraction, two dots, backward
swapped-operand contraction and adds), its FP64-equivalent TFLOP/s (2 contractions
of admitted FLOPs), the INT8 gradient's max relative difference from the FP64 one,
and central finite differences (step 1e-5) of E at random amplitudes against the
gradient.  Prints one JSON line.

    python -m tamm_b200.ccsd_adjoint [--oa 15] [--va 120] [--seed 3] [--fd 64]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads as W
from .tamm import ExecutionContext, Precision


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--oa", type=int, default=15)
    p.add_argument("--va", type=int, default=120)
    p.add_argument("--seed", type=int, default=3)
    p.add_argument("--fd", type=int, default=64)
    p.add_argument("--h", type=float, default=1e-5)
    p.add_argument("--budget-bytes", type=int, default=1 << 62)
    p.add_argument("--pool-gib", type=int, default=60)
    p.add_argument("--digit-cache-gib", type=int, default=16,
                   help="split-INT8 digits of the read-only integrals kept across contractions (0: off)")
    args = p.parse_args(argv)
    ec = ExecutionContext(0, args.pool_gib << 30)
    ec.set_digit_cache(args.digit_cache_gib << 30)
    P = W.energy_problem(args.oa, args.va, seed=args.seed, ec=ec, budget_bytes=args.budget_bytes)
    amps = W.fd_amplitudes(P.lad.t2, args.fd, seed=args.seed + 101)
    offs = [o for _, _, o in amps]
    flops = 2.0 * P.lad.flops  # forward v.t2 and the swapped-operand contraction
    out = {"workload": f"ccsd_energy_gradient_O{2 * args.oa}_V{2 * args.va}", "admitted_flops_per_gradient": flops,
           "fd_step": args.h, "fd_amplitudes": args.fd}
    grads = {}
    for name, mode in (("fp64", Precision.FP64), ("int8", Precision.INT8)):
        ec.set_precision(mode, 1e-11)
        W.energy(P, gradient=True)  # warm-up: plans, work lists, digit layouts
        ec.synchronize()
        t0 = time.perf_counter()
        e = W.energy(P, gradient=True)
        ec.synchronize()
        dt = time.perf_counter() - t0
        g = P.g.read().copy()
        grads[name] = g
        fd = W.finite_difference(P, amps, h=args.h)
        gs = g[offs]
        out[name] = {"energy": e, "gradient_ms": 1e3 * dt, "tflops": flops / dt / 1e12,
                     "fd_max_rel_err": float(np.max(np.abs(fd - gs)) / np.max(np.abs(gs))),
                     "recomputed": P.tape.info()["recomputed"]}
    ec.set_precision(Precision.FP64)
    out["int8_vs_fp64_gradient_max_rel_err"] = float(
        np.max(np.abs(grads["int8"] - grads["fp64"])) / np.max(np.abs(grads["fp64"])))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
