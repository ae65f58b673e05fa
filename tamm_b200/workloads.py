"""Synthetic coupled-cluster workloads built through the public API.

The molecular-orbital space follows the closed-shell CCSD layout of TAMM's
tests/tamm/Test_CCSD.cpp:639-668: indices [occ_alpha, occ_beta, virt_alpha, virt_beta],
Spin{1} = alpha, Spin{2} = beta, named subspaces occ/virt (+ _alpha/_beta), and a
tile list that splits at every spin/named boundary.  Inputs are seeded synthetic
data with the distributions of the benchmark configurations (there is no dataset).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .tamm import ExecutionContext, IndexSpace, Scheduler, Tape, Tensor, TiledIndexSpace, mult_info


def mo_index_space(oa: int, va: int) -> IndexSpace:
    """IndexSpace of 2*(oa+va) spin orbitals, CCSD layout (Test_CCSD.cpp:639-648)."""
    nocc, n = 2 * oa, 2 * (oa + va)
    return IndexSpace(n, named={
        "occ": [(0, nocc)], "occ_alpha": [(0, oa)], "occ_beta": [(oa, nocc)],
        "virt": [(nocc, n)], "virt_alpha": [(nocc, nocc + va)], "virt_beta": [(nocc + va, n)]},
        spin={1: [(0, oa), (nocc, nocc + va)], 2: [(oa, nocc), (nocc + va, n)]})


def even_tiles(n: int, tile: int) -> list:
    """Test_CCSD.cpp:650-668: ceil(n/tile) near-equal tiles."""
    nt = max(1, math.ceil(n / tile))
    return [n // nt + (1 if x < n % nt else 0) for x in range(nt)]


def random_tiles(n: int, lo: int, hi: int, rng: np.random.Generator) -> list:
    """Tile sizes drawn uniformly from [lo, hi], the last one truncated so they sum to n;
    a block smaller than lo is a single tile."""
    if n <= lo:
        return [n]
    out, s = [], 0
    while s < n:
        t = int(rng.integers(lo, hi + 1))
        t = min(t, n - s)
        out.append(t)
        s += t
    return out


def mo_tiled(oa: int, va: int, occ_tiles: list, virt_tiles: list) -> TiledIndexSpace:
    """TiledIndexSpace over the MO space: occ_alpha, occ_beta, virt_alpha, virt_beta tile
    lists (alpha and beta share the per-spin tile list)."""
    is_ = mo_index_space(oa, va)
    return TiledIndexSpace(is_, list(occ_tiles) + list(occ_tiles) + list(virt_tiles) + list(virt_tiles))


def fill_blocks(t: Tensor, fn) -> np.ndarray:
    """Packed host buffer of t: fn(blockid, dims, index ranges per mode) -> block array,
    called for every admitted block in storage order.  Ranges are absolute positions
    in the root index space (e.g. MO orbital indices)."""
    keys, offs = t.block_table()
    out = np.empty(max(t.nelems, 1), dtype=np.float64)
    nts = [s.num_tiles for s in t.spaces]
    starts = [s.tile_offsets for s in t.spaces]
    for key, off in zip(keys, offs):
        bid, k = [], int(key)
        for n in reversed(nts):
            bid.append(k % n)
            k //= n
        bid = bid[::-1]
        dims = tuple(int(s.tile_sizes[b]) for s, b in zip(t.spaces, bid))
        rng = [(int(starts[m][b]), int(starts[m][b]) + dims[m]) for m, b in enumerate(bid)]
        blk = np.asarray(fn(bid, dims, rng), dtype=np.float64)
        out[off:off + blk.size] = blk.ravel()
    return out[:t.nelems]


@dataclass
class Ladder:
    """r2(a,b,i,j) += v(a,b,c,d) * t2(c,d,i,j) on a spin-blocked MO space."""
    ec: ExecutionContext
    sch: Scheduler
    MO: TiledIndexSpace
    O: TiledIndexSpace
    V: TiledIndexSpace
    v: Tensor
    t2: Tensor
    r2: Tensor
    labels: tuple
    flops: float
    t2_host: np.ndarray


def orbital_energies(oa: int, va: int, seed: int):
    rng = np.random.default_rng(seed + 1000)
    e_occ = rng.uniform(-2.0, -0.3, size=oa)
    e_virt = rng.uniform(0.1, 5.0, size=va)
    return e_occ, e_virt


def ladder(oa: int, va: int, seed: int = 1, tile_lo: int = 24, tile_hi: int = 48, nchol=None,
           ec: ExecutionContext | None = None, pool_bytes: int = 0, build_v: bool = True,
           chol_tile: int = 1000, alloc_v: bool = True) -> Ladder:
    """Config of the CCSD particle-particle ladder: O = 2*oa, V = 2*va, virtual tiles
    U{tile_lo..tile_hi}, v from Cholesky vectors L(Q,a,c), Q = 5*(O+V),
    L ~ N(0,1)/sqrt(Q) * exp(-|a-c|/50) for same-spin (a,c), t2 ~ N(0, 0.1^2) /
    (e_a + e_b - e_i - e_j).  alloc_v=False (with build_v=False) leaves v unallocated."""
    rng = np.random.default_rng(seed)
    occ_t = random_tiles(oa, tile_lo, tile_hi, rng)
    virt_t = random_tiles(va, tile_lo, tile_hi, rng)
    MO = mo_tiled(oa, va, occ_t, virt_t)
    O, V = MO("occ"), MO("virt")
    ec = ec or ExecutionContext(0, pool_bytes)
    sch = Scheduler(ec)
    a, b, c, d = V.labels(4)
    i, j = O.labels(2)
    v = Tensor([V, V, V, V], spin=(2, 2))
    t2 = Tensor([V, V, O, O], spin=(2, 2))
    r2 = Tensor([V, V, O, O], spin=(2, 2))
    if build_v and not alloc_v:
        raise ValueError("building v needs it allocated")
    if alloc_v:
        sch.allocate(v)
    sch.allocate(t2, r2)
    nocc = 2 * oa
    e_occ, e_virt = orbital_energies(oa, va, seed)
    eps = np.concatenate([e_occ, e_occ, e_virt, e_virt])
    trng = np.random.default_rng(seed + 7)

    def t2_block(bid, dims, rg):
        ea = eps[rg[0][0]:rg[0][1]][:, None, None, None]
        eb = eps[rg[1][0]:rg[1][1]][None, :, None, None]
        ei = eps[rg[2][0]:rg[2][1]][None, None, :, None]
        ej = eps[rg[3][0]:rg[3][1]][None, None, None, :]
        return trng.normal(0.0, 0.1, size=dims) / (ea + eb - ei - ej)

    t2_host = fill_blocks(t2, t2_block)
    t2.write(t2_host)
    sch(r2("a,b,i,j").assign(0.0)).execute()
    if build_v:
        Q = nchol if nchol is not None else 5 * (2 * oa + 2 * va)
        CI = TiledIndexSpace(IndexSpace(Q), chol_tile)
        q = CI.label()
        L = Tensor([CI, V, V], spin_mask=[2, 0, 1])  # nonzero for spin(a) == spin(c)
        L.allocate(ec)
        lrng = np.random.default_rng(seed + 11)

        def l_block(bid, dims, rg):
            ia = np.arange(rg[1][0], rg[1][1])[:, None]
            ic = np.arange(rg[2][0], rg[2][1])[None, :]
            damp = np.exp(-np.abs(ia - ic) / 50.0)
            return lrng.normal(0.0, 1.0, size=dims) / math.sqrt(Q) * damp[None, :, :]

        L.write(fill_blocks(L, l_block))
        b2, d2 = V.labels(2)
        a2, c2 = V.labels(2)
        sch(v(a2, b2, c2, d2).assign(L(q, a2, c2) * L(q, b2, d2))).execute()
        L.deallocate()
        del L
    flops = mult_flops(r2(a, b, i, j), v(a, b, c, d), t2(c, d, i, j))
    return Ladder(ec, sch, MO, O, V, v, t2, r2, (a, b, c, d, i, j), flops, t2_host)


def mult_flops(lhs, a, b):
    """Admitted FP64 FLOPs of lhs += a * b (no GPU needed)."""
    return mult_info(lhs, a, b)[2]


@dataclass
class EnergyProblem:
    """E(t2) = sum w(i,j,a,b) t2(a,b,i,j) + 1/4 sum t2(a,b,i,j) X(a,b,i,j),
    X(a,b,i,j) = v(a,b,c,d) t2(c,d,i,j), on the ladder's spin-blocked spaces, with its
    gradient dE/dt2 = w(i,j,a,b) + 1/4 X + 1/4 sum_ab v(a,b,c,d) t2(a,b,i,j)."""
    lad: Ladder
    w: Tensor
    X: Tensor
    g: Tensor
    tape: Tape
    w_host: np.ndarray


def energy_problem(oa: int, va: int, seed: int = 3, tile_lo: int = 24, tile_hi: int = 48,
                   ec: ExecutionContext | None = None, build_v: bool = True,
                   budget_bytes: int = 1 << 62) -> EnergyProblem:
    """Config of the adjoint check: ladder inputs (v from Cholesky vectors, t2 from
    the orbital-energy denominators) and w ~ N(0, 1) / sqrt(O * V)."""
    lad = ladder(oa, va, seed=seed, tile_lo=tile_lo, tile_hi=tile_hi, ec=ec, build_v=build_v)
    if build_v:  # the integrals stay constant: tasks over their exactly-zero blocks are skipped
        lad.v.set_read_only(True)
    O, V = lad.O, lad.V
    w = Tensor([O, O, V, V], spin=(2, 2)).allocate(lad.ec)
    rng = np.random.default_rng(seed + 29)
    w_host = rng.normal(0.0, 1.0, size=w.nelems) / math.sqrt((2 * oa) * (2 * va))
    w.write(w_host)
    X = Tensor([V, V, O, O], spin=(2, 2)).allocate(lad.ec)
    g = Tensor([V, V, O, O], spin=(2, 2)).allocate(lad.ec)
    return EnergyProblem(lad, w, X, g, Tape(lad.ec, budget_bytes), w_host)


def energy(P: EnergyProblem, gradient: bool = False) -> float:
    """E(t2) through the tape; with gradient=True, P.g = dE/dt2 afterwards."""
    a, b, c, d, i, j = P.lad.labels
    t2, v = P.lad.t2, P.lad.v
    tape = P.tape.reset()
    if gradient:
        P.lad.sch(P.g().assign(0.0)).execute()
        tape.leaf(t2, P.g)
    tape.contract(P.X(a, b, i, j), v(a, b, c, d) * t2(c, d, i, j))
    e = tape.dot(P.w(i, j, a, b), t2(a, b, i, j))
    e += tape.dot(t2(a, b, i, j), P.X(a, b, i, j), 0.25)
    if gradient:
        tape.backward()
    return e


def fd_amplitudes(t: Tensor, count: int, seed: int):
    """`count` distinct stored amplitudes of t, chosen at random: (block id, element
    index within the block, packed offset)."""
    rng = np.random.default_rng(seed)
    keys, offs = t.block_table()
    nts = [s.num_tiles for s in t.spaces]
    out, seen = [], set()
    while len(out) < count:
        bi = int(rng.integers(len(keys)))
        key, bid = int(keys[bi]), []
        for n in reversed(nts):
            bid.append(key % n)
            key //= n
        bid = bid[::-1]
        size = int(np.prod(t.block_dims(bid)))
        e = int(rng.integers(size))
        if (bi, e) in seen:
            continue
        seen.add((bi, e))
        out.append((bid, e, int(offs[bi]) + e))
    return out


def finite_difference(P: EnergyProblem, amps, h: float = 1e-5):
    """Central differences (E(t2 + h e_k) - E(t2 - h e_k)) / 2h at the given amplitudes."""
    t2 = P.lad.t2
    out = []
    for bid, e, _ in amps:
        blk = t2.get(bid)
        x0 = float(blk.reshape(-1)[e])
        vals = []
        for s in (+1.0, -1.0):
            b2 = blk.copy().reshape(-1)
            b2[e] = x0 + s * h
            t2.put(bid, b2)
            vals.append(energy(P))
        t2.put(bid, blk)
        out.append((vals[0] - vals[1]) / (2.0 * h))
    return np.array(out)
