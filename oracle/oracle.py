"""TEST INFRASTRUCTURE ONLY — Python access to the oracle libraries.

Loads ``oracle/liboracle_port.so`` (the C restatement, tamm_oracle.c) and, when it
was built, ``oracle/_ref/libtamm_ref.so`` (TAMM's own kernels::block_multiply /
kernels::assign compiled from the TAMM sources).  Only tests/, the smoke check and
bench.py's CPU-baseline leg import this module; the tamm_b200 package never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle_port.so")
REF_SO = os.path.join(HERE, "_ref", "libtamm_ref.so")
MAXR = 8

_i64p = C.POINTER(C.c_int64)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


def build():
    """Compile the oracle libraries (reference only where the TAMM tree exists)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(path):
    if not os.path.exists(path):
        return None
    return C.CDLL(path)


_port = None
_ref = None


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            build()
        _port = C.CDLL(PORT_SO)
        _setup(_port, "or_")
        _port.or_tile_offsets_uniform.restype = C.c_int64
        _port.or_tile_offsets_uniform.argtypes = [C.c_int64, _i64p, C.c_int, C.c_int64, _i64p, C.c_int64]
        _port.or_tile_offsets_list.restype = C.c_int64
        _port.or_tile_offsets_list.argtypes = [C.c_int64, _i64p, C.c_int, _i64p, C.c_int64, _i64p]
        _port.or_is_non_zero.restype = C.c_int
        _port.or_is_non_zero.argtypes = [C.c_int, _ip, _ip, C.c_int]
        _port.or_nw_pack.restype = C.c_int64
        _port.or_nw_pack.argtypes = [C.c_void_p, _i64p, _i64p, _i64p]
        _port.or_nw_locate.restype = C.c_int64
        _port.or_nw_locate.argtypes = [C.c_void_p, _i64p]
        _port.or_mult_bufacc.restype = C.c_int
        _port.or_mult_bufacc.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
        _port.or_mult_bufacc_fn.restype = C.c_int
        _port.or_mult_bufacc_fn.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        _port.or_mult_count.restype = C.c_int
        _port.or_mult_count.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _i64p, _dp]
        _port.or_set.restype = None
        _port.or_set.argtypes = [C.c_void_p, C.c_double, C.c_int]
        _port.or_norm.restype = C.c_double
        _port.or_norm.argtypes = [C.c_void_p]
        _port.or_fill_uniform.restype = None
        _port.or_fill_uniform.argtypes = [_dp, C.c_int64, C.c_uint64, C.c_uint64, C.c_double, C.c_double]
        _port.or_fill_normal.restype = None
        _port.or_fill_normal.argtypes = [_dp, C.c_int64, C.c_uint64, C.c_uint64, C.c_double, C.c_double]
    return _port


def ref():
    """The compiled reference, or None when oracle/_ref was not built."""
    global _ref
    if _ref is None:
        lib = _load(REF_SO)
        if lib is None:
            return None
        _setup(lib, "ref_")
        lib.ref_set_blas_threads.restype = None
        lib.ref_set_blas_threads.argtypes = [C.c_int]
        _ref = lib
    return _ref


def _setup(lib, pfx):
    bm = getattr(lib, pfx + "block_multiply")
    bm.restype = C.c_int
    bm.argtypes = [C.c_double, _dp, _i64p, _ip, C.c_int, _dp, _i64p, _ip, C.c_int,
                   C.c_double, _dp, _i64p, _ip, C.c_int, C.c_int]
    asg = getattr(lib, pfx + "assign")
    asg.restype = C.c_int
    asg.argtypes = [_dp, _i64p, _ip, C.c_int, C.c_double, _dp, _i64p, _ip, C.c_int, C.c_int]


def _dptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _i64(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int64))
    if a.size == 0:
        a = np.zeros(1, dtype=np.int64)
    return a


def _i32(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int32))
    if a.size == 0:
        a = np.zeros(1, dtype=np.int32)
    return a


def block_multiply(alpha, A, alabels, B, blabels, beta, Cbuf, clabels, is_assign, impl="port"):
    """kernels::block_multiply on host buffers; ``impl`` is "port" or "ref".
    Arrays carry their block dims as shapes; C is updated in place."""
    lib = port() if impl == "port" else ref()
    fn = lib.or_block_multiply if impl == "port" else lib.ref_block_multiply
    ad, bd, cd = _i64(A.shape), _i64(B.shape), _i64(Cbuf.shape)
    al, bl, cl = _i32(alabels), _i32(blabels), _i32(clabels)
    rc = fn(alpha, _dptr(A), ad.ctypes.data_as(_i64p), al.ctypes.data_as(_ip), A.ndim,
            _dptr(B), bd.ctypes.data_as(_i64p), bl.ctypes.data_as(_ip), B.ndim,
            beta, _dptr(Cbuf), cd.ctypes.data_as(_i64p), cl.ctypes.data_as(_ip), Cbuf.ndim,
            int(bool(is_assign)))
    return rc


def assign(dst, dlabels, scale, src, slabels, is_assign, impl="port"):
    lib = port() if impl == "port" else ref()
    fn = lib.or_assign if impl == "port" else lib.ref_assign
    dd, sd = _i64(dst.shape), _i64(src.shape)
    dl, sl = _i32(dlabels), _i32(slabels)
    return fn(_dptr(dst), dd.ctypes.data_as(_i64p), dl.ctypes.data_as(_ip), dst.ndim, scale,
              _dptr(src), sd.ctypes.data_as(_i64p), sl.ctypes.data_as(_ip), src.ndim,
              int(bool(is_assign)))


def tile_offsets_uniform(n, bounds, tile):
    b = _i64(bounds)
    out = np.zeros(n + 2, dtype=np.int64)
    cnt = port().or_tile_offsets_uniform(n, b.ctypes.data_as(_i64p), len(bounds), tile,
                                         out.ctypes.data_as(_i64p), out.size)
    if cnt < 0:
        raise ValueError("tiling failed")
    return out[:cnt]


def tile_offsets_list(n, bounds, tiles):
    b = _i64(bounds)
    t = _i64(tiles)
    out = np.zeros(len(tiles) + 2, dtype=np.int64)
    cnt = port().or_tile_offsets_list(n, b.ctypes.data_as(_i64p), len(bounds), t.ctypes.data_as(_i64p),
                                      len(tiles), out.ctypes.data_as(_i64p))
    if cnt < 0:
        raise ValueError("tile list does not match the index space boundaries")
    return out[:cnt]


def is_non_zero(spins, mask, has_spin=True):
    s, m = _i32(spins), _i32(mask)
    return bool(port().or_is_non_zero(len(spins), s.ctypes.data_as(_ip), m.ctypes.data_as(_ip),
                                      int(has_spin)))


# ----------------------------------------------------------------------------- tensors

class _OrTensor(C.Structure):
    _fields_ = [("nmodes", C.c_int), ("has_spin", C.c_int), ("spin_mask", C.c_int * MAXR),
                ("ntiles", C.c_int64 * MAXR), ("tile_size", _i64p * MAXR),
                ("tile_spin", _ip * MAXR), ("nblocks", C.c_int64), ("keys", _i64p),
                ("offsets", _i64p), ("data", _dp)]


class _OrOperand(C.Structure):
    _fields_ = [("t", C.c_void_p), ("labels", C.c_int * MAXR), ("tmap", _i64p * MAXR),
                ("lntiles", C.c_int64 * MAXR)]


@dataclass
class BlockTensor:
    """Distribution_NW-packed block-sparse tensor on the host.

    ``tiles[i]``: tile sizes of mode i; ``spins[i]``: spin of each tile of mode i;
    ``mask``: per-mode 0 upper / 1 lower / 2 ignore, or None for no spin symmetry."""
    tiles: list
    spins: list | None = None
    mask: list | None = None
    keys: np.ndarray = field(init=False)
    offsets: np.ndarray = field(init=False)
    data: np.ndarray = field(init=False)

    def __post_init__(self):
        self.tiles = [np.ascontiguousarray(np.asarray(t, dtype=np.int64)) for t in self.tiles]
        if self.spins is None:
            self.spins = [np.zeros(len(t), dtype=np.int32) for t in self.tiles]
        self.spins = [np.ascontiguousarray(np.asarray(s, dtype=np.int32)) for s in self.spins]
        self._s = _OrTensor()
        s = self._s
        s.nmodes = len(self.tiles)
        s.has_spin = int(self.mask is not None)
        for i in range(s.nmodes):
            s.spin_mask[i] = int(self.mask[i]) if self.mask is not None else 2
            s.ntiles[i] = len(self.tiles[i])
            s.tile_size[i] = self.tiles[i].ctypes.data_as(_i64p)
            s.tile_spin[i] = self.spins[i].ctypes.data_as(_ip)
        nall = int(np.prod([len(t) for t in self.tiles])) if self.tiles else 1
        keys = np.zeros(max(nall, 1), dtype=np.int64)
        offs = np.zeros(max(nall, 1), dtype=np.int64)
        total = C.c_int64(0)
        nb = port().or_nw_pack(C.byref(s), keys.ctypes.data_as(_i64p), offs.ctypes.data_as(_i64p),
                               C.byref(total))
        self.keys = keys[:nb].copy()
        self.offsets = offs[:nb].copy()
        self.data = np.zeros(max(int(total.value), 1), dtype=np.float64)
        self.total = int(total.value)
        s.nblocks = nb
        s.keys = self.keys.ctypes.data_as(_i64p)
        s.offsets = self.offsets.ctypes.data_as(_i64p)
        s.data = self.data.ctypes.data_as(_dp)

    @property
    def nmodes(self):
        return len(self.tiles)

    def struct(self):
        return self._s

    def locate(self, blockid):
        b = _i64(blockid)
        return int(port().or_nw_locate(C.byref(self._s), b.ctypes.data_as(_i64p)))

    def block_dims(self, blockid):
        return tuple(int(self.tiles[i][b]) for i, b in enumerate(blockid))

    def block(self, blockid):
        off = self.locate(blockid)
        if off < 0:
            return None
        dims = self.block_dims(blockid)
        n = int(np.prod(dims)) if dims else 1
        return self.data[off:off + n].reshape(dims)

    def blockids(self):
        """Admitted block ids in storage (key) order."""
        out = []
        nt = [len(t) for t in self.tiles]
        for k in self.keys:
            bid = []
            kk = int(k)
            for n in reversed(nt):
                bid.append(kk % n)
                kk //= n
            out.append(tuple(reversed(bid)))
        return out

    def set(self, value, is_assign=True):
        port().or_set(C.byref(self._s), value, int(is_assign))

    def norm(self):
        return float(port().or_norm(C.byref(self._s)))


def _operand(t: BlockTensor, labels, tmaps=None, lntiles=None):
    op = _OrOperand()
    op.t = C.cast(C.pointer(t.struct()), C.c_void_p)
    keep = []
    for i in range(t.nmodes):
        op.labels[i] = int(labels[i])
        if tmaps is not None and tmaps[i] is not None:
            m = np.ascontiguousarray(np.asarray(tmaps[i], dtype=np.int64))
            keep.append(m)
            op.tmap[i] = m.ctypes.data_as(_i64p)
            op.lntiles[i] = len(m)
        else:
            op.tmap[i] = _i64p()
            op.lntiles[i] = len(t.tiles[i]) if lntiles is None else int(lntiles[i])
    op._keep = keep
    return op


def mult_bufacc(Ct, clabels, alpha, At, alabels, Bt, blabels, tmaps=(None, None, None), impl="port"):
    """MultOp::execute_bufacc: Ct(clabels) += alpha * At(alabels) * Bt(blabels).
    impl "ref" runs every block triple through the reference's compiled block_multiply."""
    c = _operand(Ct, clabels, tmaps[0])
    a = _operand(At, alabels, tmaps[1])
    b = _operand(Bt, blabels, tmaps[2])
    fn = None
    if impl == "ref":
        r = ref()
        if r is None:
            raise RuntimeError("oracle/_ref was not built")
        fn = C.cast(r.ref_block_multiply, C.c_void_p)
    rc = port().or_mult_bufacc_fn(C.byref(c), alpha, C.byref(a), C.byref(b), fn)
    if rc != 0:
        raise RuntimeError(f"or_mult_bufacc failed ({rc})")


def mult_count(Ct, clabels, At, alabels, Bt, blabels, tmaps=(None, None, None)):
    c = _operand(Ct, clabels, tmaps[0])
    a = _operand(At, alabels, tmaps[1])
    b = _operand(Bt, blabels, tmaps[2])
    nt = C.c_int64(0)
    fl = C.c_double(0)
    rc = port().or_mult_count(C.byref(c), C.byref(a), C.byref(b), C.byref(nt), C.byref(fl))
    if rc != 0:
        raise RuntimeError("or_mult_count failed")
    return int(nt.value), float(fl.value)


def fill_uniform(x, seed, first=0, lo=-1.0, hi=1.0):
    port().or_fill_uniform(_dptr(x), x.size, seed, first, lo, hi)


def fill_normal(x, seed, first=0, mean=0.0, sd=1.0):
    port().or_fill_normal(_dptr(x), x.size, seed, first, mean, sd)


# ----------------------------------------------------------------------------- OpMin

def _snoob(sub, full):
    """Next larger subset of `full` with the same number of bits (the enumeration of
    src/tamm/opmin.hpp:60-81); smaller than `sub` when the subsets of that size are
    exhausted."""
    low = sub & -sub
    ripple = sub + low
    if ripple > full:
        return 0
    ones = ((sub ^ ripple) >> 2) // low
    return ripple | ones


def opmin_order(factor_labels, lhs_labels, extent):
    """opmin::Optimizer::optimize (src/tamm/opmin.hpp:438-477 with the callbacks at
    :506-533): subsets of the n factors visited by size, then by value; available
    labels of unions, required labels (available & (available of the rest | lhs)),
    and the cheapest split of each subset, cost = product of the extents of
    required(x) | required(y) plus the parts' costs, first strict improvement kept.
    Returns ([(child1, child2) of each binary step, post order], total cost)."""
    n = len(factor_labels)
    full = (1 << n) - 1
    visit = []
    for k in range(1, n + 1):
        x = (1 << k) - 1
        while x and x <= full:
            visit.append(x)
            x = _snoob(x, full)
    avail = {1 << i: frozenset(f) for i, f in enumerate(factor_labels)}
    seen = []
    for x in visit:
        for y in seen:
            avail[x | y] = avail[x] | avail[y]
        seen.append(x)
    lhs = frozenset(lhs_labels)
    req = {x: avail[x] & (avail.get(full & ~x, frozenset()) | lhs) for x in visit}
    cost = {x: (0.0 if bin(x).count("1") == 1 else float("inf")) for x in visit}
    kids = {}
    seen = []
    for x in visit:
        for y in seen:
            if x & y:
                continue
            c = float(np.prod([extent[l] for l in req[x] | req[y]])) + cost[x] + cost[y]
            if c < cost[x | y]:
                cost[x | y] = c
                kids[x | y] = (x, y)
        seen.append(x)
    steps = []

    def walk(x):
        if x in kids:
            walk(kids[x][0])
            walk(kids[x][1])
            steps.append(kids[x])
    walk(full)
    return steps, (cost[full] if n > 1 else 0.0)
