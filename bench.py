"""Benchmark: FP64-accurate TFLOP/s of the block-sparse CCSD particle-particle ladder
r2(a,b,i,j) += v(a,b,c,d) * t2(c,d,i,j) at O=40, V=360 (spin-blocked, virtual tiles
U{24..48}), split-INT8 vs plain FP64, one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--mode int8|fp64|bf16x3]
                    [--impl ours|reference] [--oa 20 --va 180]

One "step" is one execution of the contraction over every admitted tile triple
through the Scheduler API.  `value` is the device-timed throughput with inputs
resident in HBM (v is 50 GB, far beyond L2, so no flush is needed between steps);
`e2e` repeats the step through the same public API with the step's input t2 copied
from pinned host memory and the result r2 read back inside the timed region.
The integral tensor v is marked read-only (it is constant through a coupled-cluster
run), so both the FP64 and the split-INT8 path skip the admitted tasks over its
exactly-zero spin blocks; the metric still counts every admitted FLOP, and the line
also reports the FLOPs that ran and the throughput on that basis.
Under torchrun (N > 1) the ladder is sharded by output block (TAMM's owner-computes
rule with a FLOP-balanced assignment every rank derives alone): each rank zeroes r2,
computes the blocks it owns, and one NCCL all-reduce on the context's stream
assembles r2 on every rank inside the step; inputs are replicated, the total work is
fixed ("scaling": "strong"), timing is the max over ranks.  --shard runs the same
path on one GPU (a one-rank NCCL group).

After the ladder, the full doubles-residual iteration (O=60, V=480, tiles U{20..64},
seed 2; one CUDA graph per mode) is timed in FP64, autotuned split-INT8 and BF16x3 and
reported under "ccsd_iteration" with a sampled reference-CPU baseline (--no-ccsd skips
it); on one GPU the energy gradient (O=30, V=240) and sampled steps of the streamed
triples energy (O=50, V=500; each step timed as a CUDA graph replay, the streamed
run's window beside it) follow under "adjoint" and "triples" (--no-adjoint,
--no-triples skip them).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64-accurate TFLOP/s, block-sparse CC contractions: split-INT8 vs plain FP64"

# k_contract_i8<6, 80> on the ladder: DRAM bytes (read + write) per INT8 tensor op from one
# ncu launch of the O=40/V=160 ladder (1.883e9 B read + 0.167e9 B written for 4.571e12
# ops incl. tile padding)
I8_DRAM_BYTES_PER_OP = (1.883e9 + 0.167e9) / 4.571e12
I8_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_contract_i8<6,80> launch of the "
                     "O=40/V=160 ladder (2.05 GB for 4.57e12 INT8 ops), scaled by this launch's INT8 ops")


def gemm_bytes_alg(lad, v_zero_elems, S):
    """Algorithmic DRAM bytes of one ladder GEMM launch: every digit of the nonzero v
    blocks and of t2 read once, r2 read and written once."""
    return S * (lad.v.nelems - v_zero_elems + lad.t2.nelems) + 16.0 * lad.r2.nelems


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", default=None, choices=["int8", "fp64", "bf16x3"])
    p.add_argument("--oa", type=int, default=20)
    p.add_argument("--va", type=int, default=180)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--cpu-seconds", type=float, default=20.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-ccsd", action="store_true", help="skip the doubles-iteration measurement")
    p.add_argument("--ccsd-steps", type=int, default=3, help="graph replays timed per mode")
    p.add_argument("--ccsd-oa", type=int, default=30)
    p.add_argument("--ccsd-va", type=int, default=240)
    p.add_argument("--shard", action="store_true", help="owner-computes path with an all-reduce even at N=1")
    p.add_argument("--adjoint", action="store_true",
                   help="time the energy gradient (O=30, V=240) also with several ranks (default: one rank only)")
    p.add_argument("--triples", action="store_true",
                   help="time sampled triples-energy steps (O=50, V=500) also with several ranks (default: one rank only)")
    p.add_argument("--no-adjoint", action="store_true", help="skip the energy-gradient measurement")
    p.add_argument("--no-triples", action="store_true", help="skip the triples-energy measurement")
    p.add_argument("--triples-steps", type=int, default=4)
    p.add_argument("--pool-gib", type=float, default=150.0,
                   help="device arena of the ladder workloads (small cases: a few GiB)")
    p.add_argument("--workload", default="ladder", choices=["ladder", "blockops"],
                   help="blockops: the HBM-bound block kernels on the ladder's r2 (one JSON line, GB/s)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 6:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[2 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peak(torch, kind):
    """Live cuBLAS throughput on this GPU, the denominator for kernels without a
    driver-measured peak: FP64 DGEMM (torch.matmul float64), BF16 (torch.matmul bfloat16)
    or INT8 (torch._int_mm)."""
    n = 8192
    if kind in ("fp64", "bf16"):
        a = torch.randn(n, n, dtype=torch.float64 if kind == "fp64" else torch.bfloat16, device="cuda")
        f = lambda: torch.matmul(a, a)  # noqa: E731
    else:
        a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device="cuda")
        f = lambda: torch._int_mm(a, a)  # noqa: E731
    for _ in range(2):
        f()
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        f()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def cpu_baseline_sample(wl_triples, seconds, threads, what="the O=40/V=360 ladder"):
    """The reference's own kernels::block_multiply (oracle/_ref, OpenBLAS GEMM) timed on
    host buffers with the shapes of a fixed-seed sample of the workload's tile triples."""
    from oracle import oracle as O
    ref = O.ref()
    kind = "reference"
    if ref is None:
        kind = "port"
    else:
        ref.ref_set_blas_threads(threads)
    rng = np.random.default_rng(0)
    order = rng.permutation(len(wl_triples))
    lab = {c: -ord(c) for c in "abcdij"}
    done_flops, t_used, n = 0.0, 0.0, 0
    bufs = {}
    for idx in order:
        (ad, bd, cd) = wl_triples[idx]
        key = (ad, bd)
        if key not in bufs:
            A = np.zeros(ad)
            B = np.zeros(bd)
            O.fill_uniform(A.reshape(-1), 1)
            O.fill_uniform(B.reshape(-1), 2)
            bufs = {key: (A, B, np.zeros(cd))}
        A, B, Cb = bufs[key]
        t0 = time.perf_counter()
        rc = O.block_multiply(1.0, A, [lab[c] for c in "abcd"], B, [lab[c] for c in "cdij"], 1.0, Cb,
                              [lab[c] for c in "abij"], 0, impl="ref" if kind == "reference" else "port")
        t_used += time.perf_counter() - t0
        assert rc == 0
        done_flops += 2.0 * np.prod(cd) * ad[2] * ad[3]
        n += 1
        if t_used >= seconds:
            break
    return {"value": done_flops / t_used / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": kind,
            "sample": f"{n} tile triples of {what} (fixed-seed random order), "
                      f"{done_flops:.3e} FLOP in {t_used:.1f} s through kernels::block_multiply "
                      f"(CPU branch, OpenBLAS GEMM, {threads} threads)"}


def ladder_triples(oa, va, seed, lo=24, hi=48):
    """Block shapes (A dims, B dims, C dims) of every admitted ladder triple (host only)."""
    import tamm_b200 as tb
    from tamm_b200 import workloads as W
    rng = np.random.default_rng(seed)
    occ_t = W.random_tiles(oa, lo, hi, rng)
    virt_t = W.random_tiles(va, lo, hi, rng)
    vs = [1] * len(virt_t) + [2] * len(virt_t)
    vt = virt_t + virt_t
    os_ = [1] * len(occ_t) + [2] * len(occ_t)
    ot = occ_t + occ_t
    out = []
    for a in range(len(vt)):
        for b in range(len(vt)):
            for i in range(len(ot)):
                for j in range(len(ot)):
                    if vs[a] + vs[b] != os_[i] + os_[j]:
                        continue
                    for c in range(len(vt)):
                        for d in range(len(vt)):
                            if vs[c] + vs[d] != vs[a] + vs[b]:
                                continue
                            out.append(((vt[a], vt[b], vt[c], vt[d]), (vt[c], vt[d], ot[i], ot[j]),
                                        (vt[a], vt[b], ot[i], ot[j])))
    del tb
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    triples = ladder_triples(args.oa, args.va, args.seed)
    total_flops = sum(2.0 * np.prod(c) * a[2] * a[3] for a, _, c in triples)
    per_step = max(2.0, args.cpu_seconds / max(args.steps, 1))
    cb = None
    vals = []
    for s in range(args.warmup + args.steps):
        r = cpu_baseline_sample(triples, per_step if s >= args.warmup else 1.0, threads)
        if s >= args.warmup:
            vals.append(r["value"])
            cb = r
    value = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_flops / (value * 1e12) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": f"ccsd_ladder_O{2*args.oa}_V{2*args.va}",
                                            "admitted_flops": total_flops, "parallelism": "host threads"},
            "cpu_baseline": {**cb, "value": value},
            "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def measure_adjoint(ec, torch):
    """Energy + gradient of E(t2) = w.t2 + 1/4 t2.(v t2) at O=30, V=240 through the tape,
    FP64 and split-INT8 (v read-only; its digits kept under both operand views, the
    forward one with rows (a,b) and the backward one with rows (c,d): 10.7 GB within a
    16 GiB cache): device time of one evaluation after a warm-up (median of `reps`),
    FP64-equivalent TFLOP/s of its two contractions."""
    import tamm_b200 as tb
    from tamm_b200 import workloads as W
    P = W.energy_problem(15, 120, seed=3, ec=ec)
    stream = torch.cuda.ExternalStream(ec.stream)
    flops = 2.0 * P.lad.flops
    out, grads = {"workload": "ccsd_energy_gradient_O30_V240", "admitted_flops_per_gradient": flops}, {}
    ec.set_digit_cache(int(16 * 2 ** 30))
    reps = 3
    for name, mode in (("fp64", tb.Precision.FP64), ("int8", tb.Precision.INT8)):
        ec.set_precision(mode, 1e-11)
        W.energy(P, gradient=True)
        ec.synchronize()
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            W.energy(P, gradient=True)
            e1.record(stream)
            ec.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = float(np.median(times))
        grads[name] = P.g.read()
        out[name] = {"gradient_ms": ms, "tflops": flops / ms / 1e9, "evaluations_timed": reps}
    out["int8"]["digit_cache_bytes"] = ec.digit_cache_info()[0]
    ec.set_precision(tb.Precision.FP64)
    ec.set_digit_cache(0)
    out["speedup_int8_vs_fp64"] = out["fp64"]["gradient_ms"] / out["int8"]["gradient_ms"]
    out["int8_vs_fp64_gradient_max_rel_err"] = float(np.max(np.abs(grads["int8"] - grads["fp64"])) /
                                                     np.max(np.abs(grads["fp64"])))
    P.lad.v.set_read_only(False)
    P.lad.sch.deallocate(P.lad.v, P.lad.t2, P.lad.r2, P.w, P.X, P.g)
    return out


def measure_triples(ec, torch, nsteps):
    """Sampled steps of the streamed triples energy at O=50, V=500, tile 40 (j blocks of
    2, the summed d one tile per spin block), FP64 and split-INT8 (integrals read-only,
    their digits kept): device time of the sample (each step's ops captured as one CUDA
    graph and replayed, as the doubles iteration is timed), FP64-equivalent TFLOP/s; the
    streamed run's window (steps enqueued back to back, each step's host work - new W
    tensor, work lists, denominator tables - overlapping the previous step's device
    work) beside it as stream_ms."""
    import tamm_b200 as tb
    from tamm_b200 import triples as T3
    P = T3.build(25, 250, tile=40, jtile=2, dtile=0, seed=4, ec=ec)
    allsteps = T3.steps(P)
    rng = np.random.default_rng(9)
    sample = [allsteps[int(x)] for x in rng.choice(len(allsteps), size=nsteps, replace=False)]
    out, es = {"workload": "triples_energy_O50_V500_tile40", "sampled_steps": sample, "steps_total": len(allsteps),
               "energy": "W = t2.v over d (stored), W -= t2.v over l, then sum W^2 / D (k_denom)"}, {}
    out["digit_cache_bytes_before"] = ec.digit_cache_info()[0]
    ec.set_digit_cache(int(24 * 2 ** 30))
    for name, mode in (("fp64", tb.Precision.FP64), ("int8", tb.Precision.INT8)):
        ec.set_precision(mode, 1e-11)
        sch = tb.Scheduler(ec)
        T3.energy(P, sample[:1], sch)  # warm-up
        e, fl, ms = T3.energy(P, sample, sch)
        es[name] = e
        stream = torch.cuda.ExternalStream(ec.stream)
        gms = 0.0
        for (i, j) in sample:  # device time per step: its ops as one graph, replayed twice
            sg = tb.Scheduler(ec)
            Wt, _ = T3.queue_pair(P, sg, i, j)
            g = sg.graph()  # runs the step once, then captures it
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(2):
                g.launch()
            e1.record(stream)
            g.sync()
            gms += e0.elapsed_time(e1) / 2
            del g
            sg.release()
            Wt.deallocate()
        out[name] = {"energy_sample": e, "flops_sample": fl, "ms": gms, "tflops": fl / gms / 1e9,
                     "stream_ms": ms, "stream_tflops": fl / ms / 1e9,
                     "digit_cache_bytes": ec.digit_cache_info()[0]}
    ec.set_precision(tb.Precision.FP64)
    ec.set_digit_cache(0)
    out["speedup_int8_vs_fp64"] = out["fp64"]["ms"] / out["int8"]["ms"]
    out["speedup_int8_vs_fp64_stream"] = out["fp64"]["stream_ms"] / out["int8"]["stream_ms"]
    out["int8_vs_fp64_energy_rel_err"] = abs(es["int8"] - es["fp64"]) / abs(es["fp64"])
    for t in P.T.values():
        t.set_read_only(False)
        t.deallocate()
    P.release()
    return out


def run_blockops(args, torch, tb, W, local):
    """The HBM-bound block kernels at the ladder's sizes (r2, t2: O=40, V=360 spin-blocked,
    7.8e7 elements, 0.62 GB each, beyond L2): permuted add r2(a,b,i,j) += X(b,a,j,i)
    (k_assign_blocks, 24 B/element; also X(a,b,j,i) and the streamed X(b,a,i,j), the other
    adds of the P(ab)P(ij) symmetrisation), flat add r2 += X (k_axpby, 24), dot r2.t2 and norm
    (k_dot_partial, 16 and 8), denominator update t2 += r2 / D (k_denom, 24) and an
    in-place map r2 = 2 r2 (k_map_blocks, 16).  Each timed over `steps` launches after
    `warmup` with CUDA events on the context's stream; GB/s of algorithmic bytes."""
    # r2, t2 and X only (v is not needed): 1.9 GB at O=40, V=360
    lad = W.ladder(args.oa, args.va, seed=args.seed, ec=tb.ExecutionContext(local, int(4 * 2 ** 30)),
                   build_v=False, alloc_v=False)
    ec = lad.ec
    a, b, c, d, i, j = lad.labels
    X = tb.Tensor([lad.V, lad.V, lad.O, lad.O], spin=(2, 2)).allocate(ec)
    X.write(np.random.default_rng(3).normal(size=X.nelems))
    lad.r2.write(np.random.default_rng(4).normal(size=lad.r2.nelems))
    n = lad.r2.nelems
    eps = np.concatenate([np.full(2 * args.oa, -1.0), np.full(2 * args.va, 1.0)]) * \
        np.random.default_rng(5).uniform(0.3, 2.0, size=2 * (args.oa + args.va))
    stream = torch.cuda.ExternalStream(ec.stream)
    peaks = load_peaks()
    hbm = peaks.get("hbm_gbs")
    cases = {
        "permuted_add k_assign_blocks": (24, lambda s: s(lad.r2(a, b, i, j).iadd(X(b, a, j, i)))),
        "permuted_add_abji k_assign_blocks": (24, lambda s: s(lad.r2(a, b, i, j).iadd(X(a, b, j, i)))),
        "permuted_add_baij k_assign_blocks (streamed rows)": (24, lambda s: s(lad.r2(a, b, i, j).iadd(X(b, a, i, j)))),
        "flat_add k_axpby": (24, lambda s: s(lad.r2(a, b, i, j).iadd(X(a, b, i, j)))),
        "dot k_dot_partial": (16, lambda s: s.dot(0, lad.r2(a, b, i, j), lad.t2(a, b, i, j))),
        "norm k_dot_partial": (8, lambda s: s.norm(1, lad.r2(a, b, i, j))),
        "denominator_update k_denom": (24, lambda s: s.denom(lad.t2(a, b, i, j), -1e-3, lad.r2(a, b, i, j), eps,
                                                                [1, 1, -1, -1])),
        "map_scale k_map_blocks": (16, lambda s: s.map(lad.r2(a, b, i, j), lad.r2(a, b, i, j), tb.Map.SCALE, 1.0)),
    }
    out = {}
    for name, (bpe, q) in cases.items():
        sch = tb.Scheduler(ec)
        q(sch)
        g = sch.graph()  # one captured launch per step: no host work in the timed region
        for _ in range(args.warmup):
            g.launch()
        g.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            g.launch()
        e1.record(stream)
        g.sync()
        ms = e0.elapsed_time(e1) / args.steps
        del g
        gbs = bpe * n / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "GB/s": gbs, "frac_of_measured_hbm": (gbs / hbm) if hbm else None,
                     "bytes_per_element": bpe}
    print(json.dumps({"workload": f"blockops_ladder_O{2 * args.oa}_V{2 * args.va}", "elements": n,
                      "hbm_peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured copy)",
                      "kernels": out}), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import ctypes as C

    import torch
    import torch.distributed as dist
    shard = world > 1 or args.shard
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    elif shard:  # one-rank group: the sharded path's collective on a single GPU
        import datetime
        dist.init_process_group("nccl", init_method="tcp://127.0.0.1:29533", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=600))
    import tamm_b200 as tb
    from tamm_b200 import _capi as A
    from tamm_b200 import workloads as W

    if args.workload == "blockops":
        run_blockops(args, torch, tb, W, local)
        return
    headline = args.mode or "int8"
    modes = {"fp64": tb.Precision.FP64, "int8": tb.Precision.INT8, "bf16x3": tb.Precision.BF16X3}
    ec = tb.ExecutionContext(local, int(args.pool_gib * 2 ** 30))
    lad = W.ladder(args.oa, args.va, seed=args.seed, ec=ec)
    lad.v.set_read_only(True)  # constant integrals: tasks over exactly-zero blocks are skipped
    _, v_zero_blocks, v_zero_elems = lad.v.read_only_info()
    a, b, c, d, i, j = lad.labels
    stream = torch.cuda.ExternalStream(ec.stream)
    if shard:
        lad.sch.set_owner(rank, world)  # Mult ops compute this rank's output blocks only

    def allreduce(t):
        """Sum of the ranks' shares of t, in place, on the context's stream."""
        with torch.cuda.stream(stream):
            dist.all_reduce(t.device_view())
        t.record_use()

    def step(profile=False):
        if shard:  # blocks of other ranks stay zero here; the all-reduce adds the shares
            lad.sch(lad.r2().assign(0.0))
        lad.sch(lad.r2(a, b, i, j).iadd(lad.v(a, b, c, d) * lad.t2(c, d, i, j))).execute(
            tb.ExecutionHW.GPU, profile)
        if shard:
            allreduce(lad.r2)

    def reset():
        lad.sch(lad.r2().assign(0.0)).execute()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def sum_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t)
        return float(t.item())

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    # plain FP64 path: reference result + throughput
    ec.set_precision(tb.Precision.FP64)
    reset()
    step()
    r2_fp64 = lad.r2.read().copy()
    fp64_ms = timed(step, max(1, min(args.steps, 3))) if headline != "fp64" else None

    # headline mode: accuracy against the FP64 path, then the timed steps
    ec.set_precision(modes[headline], 1e-11)
    reset()
    step()
    r2_h = lad.r2.read()
    scale = float(np.max(np.abs(r2_fp64)))
    max_rel_err = float(np.max(np.abs(r2_h - r2_fp64)) / scale) if headline != "fp64" else 0.0
    clk = ClockSampler(local)
    clk.start()
    ms = timed(step, args.steps)
    clocks = clk.stop()
    if fp64_ms is None:
        fp64_ms = ms
    jobs = 1 if shard else world  # copies of the workload the job computes
    # separately reported: the read-only v's digits split once and kept across steps
    # (tb_ctx_set_digit_cache); the headline above splits v in every step
    cached = None
    if headline == "int8":
        ec.set_digit_cache(int(48 * 2 ** 30))
        reset()
        step()  # splits v into the cache
        cms = timed(step, args.steps)
        cached = {"value": (1 if shard else world) * lad.flops / (cms * 1e-3) / 1e12, "unit": "TFLOP/s",
                  "ms_per_step": cms, "cache_bytes": ec.digit_cache_info()[0],
                  "note": "v's split digits kept across steps (constant integrals); not the headline"}
        ec.set_digit_cache(0)
        lad.v.set_read_only(False)  # drops the kept digits
        lad.v.set_read_only(True)
    value = jobs * lad.flops / (ms * 1e-3) / 1e12

    # e2e through the public API: every step copies its t2 in from pinned host memory
    # and reads its r2 back, with two device buffer sets used in turn so that a step's
    # transfers (copy streams) overlap the neighbouring steps' contractions
    t2_pin = torch.from_numpy(lad.t2_host).pin_memory()
    r2_pin = [torch.empty(lad.r2.nelems, dtype=torch.float64).pin_memory() for _ in range(2)]
    t2b = tb.Tensor([lad.V, lad.V, lad.O, lad.O], spin=(2, 2)).allocate(ec)
    r2b = tb.Tensor([lad.V, lad.V, lad.O, lad.O], spin=(2, 2)).allocate(ec)
    lad.sch(r2b().assign(0.0)).execute()
    bufs = [(lad.t2, lad.r2), (t2b, r2b)]

    def e2e_step(k):
        t2x, r2x = bufs[k % 2]
        t2x.write_async(t2_pin.data_ptr())
        if shard:
            lad.sch(r2x().assign(0.0))
        lad.sch(r2x(a, b, i, j).iadd(lad.v(a, b, c, d) * t2x(c, d, i, j))).execute_async()
        if shard:
            allreduce(r2x)
        r2x.read_async(r2_pin[k % 2].data_ptr())

    n_e2e = args.steps
    for k in range(args.warmup):
        e2e_step(k)
    lad.sch.wait()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(n_e2e):
        e2e_step(k)
    ec.join()  # the last read-back is inside the timed region
    e1.record(stream)
    lad.sch.wait()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / n_e2e)
    e2e_val = jobs * lad.flops / (e2e_ms * 1e-3) / 1e12
    lad.t2.write(lad.t2_host)

    # roofline of the dominant kernel from a profiled step (CUDA events on the stream)
    step(profile=True)
    st = lad.sch.op_stats(-1)
    flops_run = sum_over_ranks(st["flops_run"]) if shard else st["flops_run"]
    peaks = load_peaks()
    if headline in ("int8", "bf16x3"):
        S = st["slices_max"]
        achieved = st["int8_ops"] / (st["gemm_ms"] * 1e-3) / 1e12
        if headline == "int8":
            peak = measured_peak(torch, "int8")
            kernel, src = f"k_contract_i8<S={S}> (tcgen05 kind::i8)", (
                "measured live: cuBLASLt INT8 GEMM (torch._int_mm) 8192^3 on this GPU; "
                "MEASURED_PEAKS.json has no INT8 figure")
            ops = "INT8 tensor ops (2 per multiply-add) incl. padding to 128x80x32 tiles"
        else:
            peak = peaks.get("bf16_tflops") or measured_peak(torch, "bf16")
            kernel, src = "k_contract_i8<S=2, bf16> (tcgen05 kind::f16, bf16 A/B, f32 accumulate)", (
                "MEASURED_PEAKS.json bf16_tflops (measured burst cuBLAS bf16 GEMM)")
            ops = "BF16 tensor FLOPs (2 per multiply-add, 3 piece products) incl. padding to 128x80x16 tiles"
        achieved_alg = st["int8_ops_alg"] / (st["gemm_ms"] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "kernel": kernel, "ops": ops, "peak_source": src,
                "achieved_algorithmic": achieved_alg, "frac_algorithmic": achieved_alg / peak,
                "algorithmic": "the same slice products without tile padding",
                "gemm_ms": st["gemm_ms"], "split_ms": st["split_ms"]}
        # the split pass is HBM-bound: FP64 read + S digit bytes (bf16 pieces: 2 bytes
        # each) written per operand element
        nsplit = lad.v.nelems - v_zero_elems + lad.t2.nelems  # blocks of v that take part
        split_bytes = nsplit * (8 + S * (2 if headline == "bf16x3" else 1)) + 0.0
        hbm = peaks.get("hbm_gbs")
        if headline == "int8":
            # DRAM traffic per launch from ncu: one launch of the O=40/V=160 ladder (same
            # output width N = 400, so the same re-reads of A digits per op), scaled by
            # the INT8 ops of this launch
            roof["traffic"] = st["int8_ops"] * I8_DRAM_BYTES_PER_OP
            roof["traffic_source"] = I8_TRAFFIC_SOURCE
            roof["traffic_algorithmic"] = gemm_bytes_alg(lad, v_zero_elems, S)
        roof["split"] = {"bound": "hbm", "achieved": split_bytes / (st["split_ms"] * 1e-3) / 1e9,
                         "peak": hbm, "unit": "GB/s",
                         "frac": (split_bytes / (st["split_ms"] * 1e-3) / 1e9 / hbm) if hbm else None,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)"}
    else:
        peak = measured_peak(torch, "fp64")
        achieved = flops_run / (st["gemm_ms"] * 1e-3) / 1e12  # the FLOPs the kernel ran
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "kernel": "k_contract_fp64 (DMMA m16n8k8)",
                "peak_source": "measured live: cuBLAS DGEMM 8192^3 on this GPU; "
                               "MEASURED_PEAKS.json has no FP64 figure"}
    # the doubles-residual iteration (config of the CCSD-shaped residual), after the
    # ladder's tensors are released
    ccsd_line = None
    if not args.no_ccsd:
        lad.v.set_read_only(False)
        lad.sch.deallocate(lad.v, lad.t2, lad.r2, t2b, r2b)
        del t2_pin, r2_pin
        from tamm_b200 import ccsd as CC
        P = CC.build(args.ccsd_oa, args.ccsd_va, seed=2, tile_lo=20, tile_hi=64, ec=ec)
        res = CC.measure(P, max(1, args.ccsd_steps), ("fp64", "int8", "bf16x3"))
        for m in res.values():  # max over ranks of the replay time
            m["graph_ms"] = max_over_ranks(m["graph_ms"])
            m["tflops_graph"] = world * P.flops["contractions"] / m["graph_ms"] / 1e9
        for m in ("int8", "bf16x3"):
            res[m]["speedup_vs_fp64"] = res["fp64"]["graph_ms"] / res[m]["graph_ms"]
        ccsd_line = {"workload": f"ccsd_doubles_iteration_O{2 * args.ccsd_oa}_V{2 * args.ccsd_va}",
                     "unit": "TFLOP/s (admitted FP64 FLOPs of the iteration's contractions / graph replay time)",
                     "flops": P.flops, "ops_per_iteration": len(CC._ops(P)) + 3,
                     "ladder_batches": P.ladder_batches, **res, "cpu_baseline": None}
        for t in P.T.values():  # the iteration's arena memory goes back before the next workload
            if getattr(t, "ec", None) is not None:
                t.set_read_only(False)
                t.deallocate()
        del P
        import gc
        gc.collect()
    # configs 4 and 5 beside the ladder on one GPU (several ranks: only when asked for;
    # the triples problem stages 5 GB of dense amplitudes on the host per rank)
    do_adjoint = not args.no_adjoint and (world == 1 or args.adjoint)
    do_triples = not args.no_triples and (world == 1 or args.triples)
    adjoint_line = measure_adjoint(ec, torch) if do_adjoint else None
    triples_line = measure_triples(ec, torch, args.triples_steps) if do_triples else None
    if world > 1:
        dist.barrier()
    if rank == 0:
        # the reference's CPU path, after every GPU measurement (its BLAS threads on all
        # host cores would otherwise slow the host side of the GPU runs that follow)
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cpu = cpu_baseline_sample(ladder_triples(args.oa, args.va, args.seed), args.cpu_seconds,
                                      os.cpu_count() or 1)
            if ccsd_line is not None:
                # the reference's block_multiply on a fixed-seed sample of the iteration's
                # particle-ladder triples (its largest contraction), extrapolated
                cpu3 = cpu_baseline_sample(ladder_triples(args.ccsd_oa, args.ccsd_va, 2, 20, 64),
                                           args.cpu_seconds / 2, os.cpu_count() or 1,
                                           f"the O={2 * args.ccsd_oa}/V={2 * args.ccsd_va} particle ladder "
                                           f"(tiles U{{20..64}}, seed 2)")
                cpu3["iteration_s_extrapolated"] = ccsd_line["flops"]["contractions"] / (cpu3["value"] * 1e12)
                cpu3["speedup_int8_graph_vs_cpu"] = cpu3["iteration_s_extrapolated"] / (
                    ccsd_line["int8"]["graph_ms"] * 1e-3)
                ccsd_line["cpu_baseline"] = cpu3
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong" if shard else "weak",
            "vs_baseline": None, "dtype": {"fp64": "f64", "int8": "s8 balanced digits, s32 accumulate, f64 recombination",
                                           "bf16x3": "bf16 hi+lo pieces, f32 accumulate, f64 recombination"}[headline],
            "data": "synthetic (seeded; no dataset)",
            "config": {"workload": f"ccsd_ladder_O{2*args.oa}_V{2*args.va}", "mode": headline,
                       "contraction": "r2(a,b,i,j) += v(a,b,c,d) * t2(c,d,i,j), spin-blocked, virt tiles U{24..48}",
                       "admitted_flops": lad.flops, "nonzero_flops": flops_run,
                       "v_read_only": {"zero_blocks": v_zero_blocks, "zero_elements": v_zero_elems},
                       "slices": st.get("slices_max"),
                       "l2": f"inputs larger than L2 (v = {8*lad.v.nelems/1e9:.1f} GB), no flush",
                       "parallelism": (f"owner-computes x{world} (output blocks FLOP-balanced, NCCL all-reduce of "
                                       f"r2 in every step)") if shard else f"replicas x{world}"},
            "fp64_path": {"value": jobs * lad.flops / (fp64_ms * 1e-3) / 1e12, "unit": "TFLOP/s", "ms_per_step": fp64_ms},
            "value_nonzero": {"value": jobs * flops_run / (ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                              "basis": "FLOPs of the tasks that ran (exactly-zero blocks of v skipped)"},
            "speedup_vs_fp64_path": fp64_ms / ms,
            "int8_cached_digits": cached,
            "max_rel_err_vs_fp64": max_rel_err,
            "e2e": {"value": e2e_val, "unit": "TFLOP/s", "h2d_bytes_per_step": 8 * lad.t2.nelems,
                    "d2h_bytes_per_step": 8 * lad.r2.nelems, "ms_per_step": e2e_ms},
            # our kernels per step: INT8 = split A, split B, k_task_slices, GEMM; BF16x3 =
            # split A, split B, GEMM (its digit counts come from a memset); FP64 = one kernel
            "gpu_launches": args.steps * {"int8": 4, "bf16x3": 3, "fp64": 1}[headline],
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "ccsd_iteration": ccsd_line,
            "adjoint": adjoint_line,
            "triples": triples_line,
        }
        print(json.dumps(line), flush=True)
    if shard:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
