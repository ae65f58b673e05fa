"""Python front-end mirroring TAMM's LabeledTensor / Scheduler API over the C ABI.

    is_  = IndexSpace(range(100), named={"occ": [(0, 20)], "virt": [(20, 100)]},
                      spin={1: [(0, 10), (20, 60)], 2: [(10, 20), (60, 100)]})
    MO   = TiledIndexSpace(is_, tiles)             # TiledIndexSpace{is, tiles}
    O, V = MO("occ"), MO("virt")
    a, b, c, d = V.labels(4)
    i, j = O.labels(2)
    t2 = Tensor([V, V, O, O], spin=(2, 2))          # Tensor<T>{{V,V,O,O},{2,2}}
    sch = Scheduler(ec)
    sch.allocate(t2, r2, v)
    sch(r2(a, b, i, j).iadd(v(a, b, c, d) * t2(c, d, i, j))).execute(ExecutionHW.GPU)

C++ `C(...) += expr` / `-=` / `=` are `.iadd(expr)` / `.isub(expr)` / `.assign(expr)`
here (Python has no augmented assignment on a call).  Everything executes on the
GPU through libtamm_b200.so; there is no host execution path.
"""
from __future__ import annotations

import ctypes as C
import itertools
from typing import Sequence

import numpy as np

from . import _capi as A
from ._capi import call


class ExecutionHW:
    DEFAULT = 0
    CPU = 1
    GPU = 2


class Precision:
    FP64 = A.TB_MODE_FP64
    INT8 = A.TB_MODE_INT8
    BF16X3 = A.TB_MODE_BF16X3


class Map:
    """Element functions of Scheduler.map (TAMM's apply_ewise wrappers)."""
    COPY, SCALE, SET, SQUARE, SQRT = A.TB_MAP_COPY, A.TB_MAP_SCALE, A.TB_MAP_SET, A.TB_MAP_SQUARE, A.TB_MAP_SQRT
    LOG, LOG10, INVERSE, POW, ABS = A.TB_MAP_LOG, A.TB_MAP_LOG10, A.TB_MAP_INVERSE, A.TB_MAP_POW, A.TB_MAP_ABS


def _i64arr(v):
    a = np.ascontiguousarray(np.asarray(list(v) if not isinstance(v, np.ndarray) else v, dtype=np.int64))
    return a if a.size else np.zeros(1, dtype=np.int64)


class ExecutionContext:
    """ExecutionContext on one GPU: stream + stream-ordered device arena."""

    def __init__(self, device: int = 0, pool_bytes: int = 0):
        self.h = A.h()
        call("tb_ctx_create", device, int(pool_bytes), C.byref(self.h))
        self.device = device

    def set_precision(self, mode=Precision.FP64, err_target=1e-11, nslices=0):
        call("tb_ctx_set_precision", self.h, int(mode), float(err_target), int(nslices))

    def set_digit_cache(self, nbytes: int):
        """Keep up to nbytes of split-INT8 digits of read-only tensors across contractions."""
        call("tb_ctx_set_digit_cache", self.h, int(nbytes))
        return self

    def digit_cache_info(self):
        """(bytes kept, limit) of the digit cache."""
        u, l = C.c_int64(), C.c_int64()
        call("tb_ctx_digit_cache_info", self.h, C.byref(u), C.byref(l))
        return u.value, l.value

    @property
    def stream(self):
        s = A.vp()
        call("tb_ctx_stream", self.h, C.byref(s))
        return s.value

    def alloc(self, nbytes: int) -> int:
        """Device memory from the context's arena (256-byte aligned); returns the address."""
        p = A.vp()
        call("tb_ctx_alloc", self.h, int(nbytes), C.byref(p))
        return p.value

    def free(self, ptr: int):
        call("tb_ctx_free", self.h, C.c_void_p(ptr))
        return self

    def join(self):
        """Later compute-stream work waits for the copy streams (tb_ctx_join)."""
        call("tb_ctx_join", self.h)
        return self

    def synchronize(self):
        call("tb_ctx_synchronize", self.h)

    def arena_info(self):
        u, p, c = C.c_int64(), C.c_int64(), C.c_int64()
        call("tb_ctx_arena_info", self.h, C.byref(u), C.byref(p), C.byref(c))
        return u.value, p.value, c.value

    def close(self):
        if self.h:
            A.lib().tb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ranges(rs):
    out = []
    for r in rs:
        if isinstance(r, range):
            assert r.step == 1
            out.append((r.start, r.stop))
        else:
            out.append((int(r[0]), int(r[1])))
    return out


class IndexSpace:
    """IndexSpace{range(n), {{name, {ranges}}...}, {{Spin{s}, {ranges}}...}}."""

    def __init__(self, n, named: dict | None = None, spin: dict | None = None):
        if isinstance(n, range):
            assert n.start == 0 and n.step == 1
            n = n.stop
        self.n = int(n)
        named = named or {}
        spin = spin or {}
        names = list(named.keys())
        cnames = (C.c_char_p * max(len(names), 1))(*[s.encode() for s in names])
        nn = (C.c_int * max(len(names), 1))(*[len(_ranges(named[s])) for s in names])
        nr = _i64arr([x for s in names for r in _ranges(named[s]) for x in r])
        svals = list(spin.keys())
        sv = (C.c_int * max(len(svals), 1))(*[int(s) for s in svals])
        sn = (C.c_int * max(len(svals), 1))(*[len(_ranges(spin[s])) for s in svals])
        sr = _i64arr([x for s in svals for r in _ranges(spin[s]) for x in r])
        self.h = A.h()
        call("tb_is_create", self.n, len(names), cnames, nn, nr.ctypes.data_as(A.i64p), len(svals),
             sv, sn, sr.ctypes.data_as(A.i64p), C.byref(self.h))

    def __del__(self):
        try:
            A.lib().tb_is_destroy(self.h)
        except Exception:
            pass


_label_ids = itertools.count(1)


class TiledIndexLabel:
    def __init__(self, tis: "TiledIndexSpace", name: str = ""):
        self.tis = tis
        self.id = next(_label_ids)
        self.name = name

    def __repr__(self):
        return f"TiledIndexLabel({self.name or self.id})"

    def __call__(self, *deps: "TiledIndexLabel") -> "_DepLabel":
        """a(i, j): a label over a dependent space, with the labels its tiles depend on."""
        return _DepLabel(self, list(deps))


class _DepLabel:
    def __init__(self, label: TiledIndexLabel, deps: list):
        self.label, self.deps = label, deps


class TiledIndexSpace:
    """TiledIndexSpace{is, tile} or TiledIndexSpace{is, tile_list}."""

    def __init__(self, is_: IndexSpace | None = None, tile=None, _handle=None, _parent=None):
        self.parent = _parent
        self.is_ = is_ if is_ is not None else (_parent.is_ if _parent else None)
        if _handle is not None:
            self.h = _handle
        else:
            self.h = A.h()
            if isinstance(tile, (list, tuple, np.ndarray)):
                t = _i64arr(tile)
                call("tb_tis_create", is_.h, 0, t.ctypes.data_as(A.i64p), len(tile), C.byref(self.h))
            else:
                call("tb_tis_create", is_.h, int(tile), None, 0, C.byref(self.h))
        n = C.c_int64()
        call("tb_tis_num_tiles", self.h, C.byref(n))
        nt = n.value
        sizes = np.zeros(max(nt, 1), dtype=np.int64)
        spins = np.zeros(max(nt, 1), dtype=np.int32)
        roots = np.zeros(max(nt, 1), dtype=np.int64)
        call("tb_tis_tiles", self.h, sizes.ctypes.data_as(A.i64p), spins.ctypes.data_as(A.ip),
             roots.ctypes.data_as(A.i64p))
        self.tile_sizes = sizes[:nt].copy()
        self.tile_spins = spins[:nt].copy()
        self.root_tiles = roots[:nt].copy()

    def __call__(self, name: str = "all") -> "TiledIndexSpace":
        h = A.h()
        call("tb_tis_named", self.h, name.encode(), C.byref(h))
        return TiledIndexSpace(_handle=h, _parent=self)

    def sub(self, first: int, last: int) -> "TiledIndexSpace":
        """TiledIndexSpace{tis, range(first, last)} (a range of tiles)."""
        h = A.h()
        call("tb_tis_subrange", self.h, int(first), int(last), C.byref(h))
        return TiledIndexSpace(_handle=h, _parent=self)

    @property
    def num_tiles(self):
        return len(self.tile_sizes)

    @property
    def tile_offsets(self):
        """Index-space offset of the first index of each tile."""
        root = self
        while root.parent is not None:
            root = root.parent
        starts = np.zeros(root.num_tiles + 1, dtype=np.int64)
        starts[1:] = np.cumsum(root.tile_sizes)
        return starts[self.root_tiles]

    def tile_size(self, i):
        return int(self.tile_sizes[i])

    def spin(self, i):
        return int(self.tile_spins[i])

    def label(self, name=""):
        return TiledIndexLabel(self, name)

    @classmethod
    def dependent(cls, reference: "TiledIndexSpace", on: Sequence, dep: dict) -> "TiledIndexSpace":
        """TiledIndexSpace{reference, {on...}, dep_map}: dep maps a tuple of tile indices
        of the `on` spaces to the sub-space of `reference` whose tiles exist for it."""
        keys = np.asarray([list(k) for k in dep.keys()] or [[0] * len(on)], dtype=np.int64).reshape(-1)
        vals = (A.h * max(len(dep), 1))(*[v.h for v in dep.values()])
        ons = (A.h * len(on))(*[o.h for o in on])
        h = A.h()
        call("tb_tis_create_dependent", reference.h, len(on), ons, len(dep), keys.ctypes.data_as(A.i64p), vals,
             C.byref(h))
        t = cls(_handle=h, _parent=reference)
        t._deps = (list(on), dict(dep))  # keep the spaces alive
        return t

    def labels(self, n, name="all"):
        sp = self if name == "all" else self(name)
        return tuple(TiledIndexLabel(sp) for _ in range(n))

    def __del__(self):
        try:
            A.lib().tb_tis_destroy(self.h)
        except Exception:
            pass


class Tensor:
    """Tensor<double>{tis...}, with `spin=(nupper, nlower)` or `spin_mask=[...]` for
    spin-blocked sparsity."""

    def __init__(self, spaces: Sequence, spin=None, spin_mask=None):
        dep = [s for s in spaces if isinstance(s, _DepLabel)]
        plain = [s.label if isinstance(s, _DepLabel) else s for s in spaces]
        self.spaces = [s.tis if isinstance(s, TiledIndexLabel) else s for s in plain]
        self.default_labels = [s if isinstance(s, TiledIndexLabel) else None for s in plain]
        n = len(self.spaces)
        hs = (A.h * max(n, 1))(*[s.h for s in self.spaces])
        self.h = A.h()
        if dep:  # Tensor{i, j, a(i, j), e(i, j)}: modes over dependent spaces
            dm = (C.c_int * (4 * n))(*([-1] * (4 * n)))
            for m, s in enumerate(spaces):
                if isinstance(s, _DepLabel):
                    for k, d in enumerate(s.deps):
                        dm[4 * m + k] = [x is d for x in plain].index(True)
            if spin is not None:
                spin_mask = [0] * int(spin[0]) + [1] * int(spin[1]) + [2] * (n - int(spin[0]) - int(spin[1]))
            mk = (C.c_int * n)(*spin_mask) if spin_mask is not None else None
            call("tb_tensor_create_dependent", n, hs, mk, dm, C.byref(self.h))
        elif spin is not None:
            call("tb_tensor_create_spin_sizes", n, hs, int(spin[0]), int(spin[1]), C.byref(self.h))
        elif spin_mask is not None:
            m = (C.c_int * n)(*spin_mask)
            call("tb_tensor_create", n, hs, m, C.byref(self.h))
        else:
            call("tb_tensor_create", n, hs, None, C.byref(self.h))
        nm, nb, ne = C.c_int(), C.c_int64(), C.c_int64()
        call("tb_tensor_info", self.h, C.byref(nm), C.byref(nb), C.byref(ne))
        self.nmodes, self.nblocks, self.nelems = nm.value, nb.value, ne.value
        self.ec = None

    # --- lambda tensors (blocks on demand) ---
    @classmethod
    def lambda_(cls, spaces: Sequence, fn, spin=None, spin_mask=None, batch_bytes: int = 0):
        """Tensor<T>(tis, Func): fn(blockid, dims) -> array of the block's values, called
        when a contraction reads the block (tb_tensor_create_lambda; the values are
        copied to the device on the stream the library gives)."""
        import torch

        def cb(bid_p, nm, dims_p, dst, n, stream, user):
            try:
                bid = [bid_p[k] for k in range(nm)]
                dims = [dims_p[k] for k in range(nm)]
                arr = np.ascontiguousarray(fn(bid, dims), dtype=np.float64).reshape(-1)
                if arr.size != n:
                    return 2
                view = _device_array(dst, n, torch.cuda.current_device())
                with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                    view.copy_(torch.from_numpy(arr))
                return 0
            except Exception:  # a failing callback fails the op, not the process
                import traceback
                traceback.print_exc()
                return 1
        return cls._on_demand(spaces, spin, spin_mask, "tb_tensor_create_lambda", A.BLOCK_FN(cb), batch_bytes)

    @classmethod
    def built(cls, spaces: Sequence, builder, spin=None, spin_mask=None, batch_bytes: int = 0):
        """A tensor built batch by batch when a contraction reads it
        (tb_tensor_create_built): builder(batch, first_tile, last_tile, sch) queues ops
        on the scheduler `sch` that write the allocated tensor `batch` (the tiles
        [first_tile, last_tile) of the first mode's label space, the other modes whole)."""
        holder = {}

        def cb(batch_h, first, last, sch_h, user):
            try:
                me = holder["t"]
                spaces_b = []
                for m in range(me.nmodes):
                    th = A.h()
                    call("tb_tensor_space", batch_h, m, C.byref(th))
                    spaces_b.append(TiledIndexSpace(_handle=th, _parent=me.spaces[m]))
                builder(_BorrowedTensor(batch_h, spaces_b), int(first), int(last), _BorrowedScheduler(sch_h))
                return 0
            except Exception:
                import traceback
                traceback.print_exc()
                return 1
        t = cls._on_demand(spaces, spin, spin_mask, "tb_tensor_create_built", A.BATCH_FN(cb), batch_bytes)
        holder["t"] = t
        return t

    @classmethod
    def _on_demand(cls, spaces, spin, spin_mask, ctor, cfn, batch_bytes):
        self = cls.__new__(cls)
        self.spaces = [s.tis if isinstance(s, TiledIndexLabel) else s for s in spaces]
        self.default_labels = [s if isinstance(s, TiledIndexLabel) else None for s in spaces]
        n = len(self.spaces)
        hs = (A.h * max(n, 1))(*[s.h for s in self.spaces])
        if spin is not None:
            mask = [0] * int(spin[0]) + [1] * int(spin[1]) + [2] * (n - int(spin[0]) - int(spin[1]))
        else:
            mask = spin_mask
        m = (C.c_int * n)(*mask) if mask is not None else None
        self.h = A.h()
        self._fn = cfn  # the C callback must outlive the tensor
        call(ctor, n, hs, m, C.cast(cfn, C.c_void_p), None, C.byref(self.h))
        if batch_bytes:
            call("tb_tensor_set_batch_bytes", self.h, int(batch_bytes))
        nm, nb, ne = C.c_int(), C.c_int64(), C.c_int64()
        call("tb_tensor_info", self.h, C.byref(nm), C.byref(nb), C.byref(ne))
        self.nmodes, self.nblocks, self.nelems = nm.value, nb.value, ne.value
        self.ec = None
        return self

    def set_batch_bytes(self, nbytes: int):
        call("tb_tensor_set_batch_bytes", self.h, int(nbytes))
        return self

    # --- storage ---
    def allocate(self, ec: ExecutionContext):
        call("tb_tensor_allocate", self.h, ec.h)
        self.ec = ec
        return self

    def deallocate(self):
        call("tb_tensor_deallocate", self.h)
        self.ec = None

    def write_async(self, host_ptr: int):
        """Asynchronous copy of the packed store from pinned host memory at host_ptr."""
        call("tb_tensor_write_async", self.h, C.cast(host_ptr, A.dp), self.nelems)
        return self

    def read_async(self, host_ptr: int):
        """Asynchronous copy of the packed store into pinned host memory at host_ptr."""
        call("tb_tensor_read_async", self.h, C.cast(host_ptr, A.dp), self.nelems)
        return self

    def save(self, path: str):
        """Checkpoint (TAMM's write_to_disk element order, raw file)."""
        call("tb_tensor_save", self.h, str(path).encode())
        return self

    def load(self, path: str):
        """Restart from a checkpoint of a tensor with the same spaces and spin mask."""
        call("tb_tensor_load", self.h, str(path).encode())
        return self

    def attach(self, ec: ExecutionContext, device_ptr: int, nbytes: int):
        """Caller-owned device storage (>= 8 * nelems bytes, 16-byte aligned), e.g. one
        buffer shared by tensors used one after another in stream order."""
        call("tb_tensor_attach", self.h, ec.h, C.c_void_p(device_ptr), int(nbytes))
        self.ec = ec
        return self

    def record_use(self):
        """Order later asynchronous transfers after work the caller enqueued on the
        context's stream (e.g. a collective over this tensor's storage)."""
        call("tb_tensor_record_use", self.h)
        return self

    def device_view(self):
        """A torch tensor sharing this tensor's packed device storage (no copy), for
        collectives and checks; valid while the tensor stays allocated."""
        return _device_array(self.data_ptr(), self.nelems, self.ec.device)

    def set_read_only(self, on: bool = True):
        """Declare the contents constant (writes through the library then fail) and let
        contractions skip tasks over its exactly-zero blocks (tb_tensor_set_read_only)."""
        call("tb_tensor_set_read_only", self.h, int(bool(on)))
        return self

    def read_only_info(self):
        """(marked, zero blocks, zero elements) found by the read-only scan."""
        on, nb, ne = C.c_int(), C.c_int64(), C.c_int64()
        call("tb_tensor_read_only_info", self.h, C.byref(on), C.byref(nb), C.byref(ne))
        return bool(on.value), nb.value, ne.value

    def data_ptr(self):
        p = A.vp()
        call("tb_tensor_data", self.h, C.byref(p))
        return p.value

    def block_table(self):
        k = np.zeros(max(self.nblocks, 1), dtype=np.int64)
        o = np.zeros(max(self.nblocks, 1), dtype=np.int64)
        call("tb_tensor_block_table", self.h, k.ctypes.data_as(A.i64p), o.ctypes.data_as(A.i64p))
        return k[:self.nblocks].copy(), o[:self.nblocks].copy()

    def is_non_zero(self, blockid):
        b = _i64arr(blockid)
        r = C.c_int()
        call("tb_tensor_is_non_zero", self.h, b.ctypes.data_as(A.i64p), C.byref(r))
        return bool(r.value)

    def block_dims(self, blockid):
        b = _i64arr(blockid)
        d = np.zeros(max(self.nmodes, 1), dtype=np.int64)
        call("tb_tensor_block_dims", self.h, b.ctypes.data_as(A.i64p), d.ctypes.data_as(A.i64p))
        return tuple(int(x) for x in d[:self.nmodes])

    def locate(self, blockid):
        b = _i64arr(blockid)
        o = C.c_int64()
        call("tb_tensor_locate", self.h, b.ctypes.data_as(A.i64p), C.byref(o))
        return o.value

    def get(self, blockid) -> np.ndarray:
        dims = self.block_dims(blockid)
        buf = np.zeros(int(np.prod(dims)) if dims else 1, dtype=np.float64)
        b = _i64arr(blockid)
        call("tb_tensor_get", self.h, b.ctypes.data_as(A.i64p), buf.ctypes.data_as(A.dp), buf.size)
        return buf.reshape(dims)

    def put(self, blockid, values):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        b = _i64arr(blockid)
        call("tb_tensor_put", self.h, b.ctypes.data_as(A.i64p), v.ctypes.data_as(A.dp), v.size)

    def add(self, blockid, values):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        b = _i64arr(blockid)
        call("tb_tensor_add", self.h, b.ctypes.data_as(A.i64p), v.ctypes.data_as(A.dp), v.size)

    def write(self, packed: np.ndarray):
        v = np.ascontiguousarray(packed, dtype=np.float64).ravel()
        call("tb_tensor_write", self.h, v.ctypes.data_as(A.dp), v.size)

    def read(self) -> np.ndarray:
        v = np.zeros(max(self.nelems, 1), dtype=np.float64)
        call("tb_tensor_read", self.h, v.ctypes.data_as(A.dp), self.nelems)
        return v[:self.nelems]

    def norm(self) -> float:
        r = C.c_double()
        call("tb_tensor_norm", self.h, C.byref(r))
        return r.value

    def fill_random(self, seed, dist=0, p0=-1.0, p1=1.0, first=0):
        call("tb_fill_random", self.data_ptr(), self.nelems, int(seed), int(first), int(dist),
             float(p0), float(p1), A.vp(self.ec.stream))
        self.ec.synchronize()

    # --- labelling ---
    def __call__(self, *labels) -> "LabeledTensor":
        if len(labels) == 1 and isinstance(labels[0], str):
            names = [s.strip() for s in labels[0].split(",")] if labels[0] else []
            return LabeledTensor(self, names)
        if not labels:
            # T(): the tensor's own labels; labels of equal (space, position) coincide
            return LabeledTensor(self, [f"__mode{i}" for i in range(self.nmodes)])
        return LabeledTensor(self, list(labels))

    def __del__(self):
        try:
            A.lib().tb_tensor_destroy(self.h)
        except Exception:
            pass


class _BorrowedTensor(Tensor):
    """A library-owned tensor handed to a callback (not destroyed from Python)."""

    def __init__(self, h, spaces):
        self.h = C.c_void_p(h) if not isinstance(h, C.c_void_p) else h
        self.spaces = spaces
        self.default_labels = [None] * len(spaces)
        nm, nb, ne = C.c_int(), C.c_int64(), C.c_int64()
        call("tb_tensor_info", self.h, C.byref(nm), C.byref(nb), C.byref(ne))
        self.nmodes, self.nblocks, self.nelems = nm.value, nb.value, ne.value
        self.ec = None

    def __del__(self):
        pass


def _device_array(ptr: int, n: int, device: int):
    """A torch view of n doubles of device memory at ptr (no copy)."""
    import torch

    class _Dev:
        pass
    d = _Dev()
    d.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False), "version": 3,
                                  "strides": None}
    return torch.as_tensor(d, device=f"cuda:{device}")


class _Product:
    def __init__(self, alpha, factors):
        self.alpha = alpha
        self.factors = factors

    def __mul__(self, other):
        if isinstance(other, LabeledTensor):
            return _Product(self.alpha, self.factors + [other])
        return _Product(self.alpha * float(other), self.factors)

    __rmul__ = __mul__

    def __neg__(self):
        return _Product(-self.alpha, self.factors)


class LabeledTensor:
    def __init__(self, tensor: Tensor, labels: list):
        if len(labels) != tensor.nmodes:
            raise ValueError(f"{len(labels)} labels for a {tensor.nmodes}-mode tensor")
        self.tensor = tensor
        self.labels = labels

    def __mul__(self, other):
        return _Product(1.0, [self]) * other

    __rmul__ = __mul__

    def __neg__(self):
        return _Product(-1.0, [self])

    # C++ `=`, `+=`, `-=`
    def assign(self, rhs):
        return _OpSpec(self, rhs, is_assign=True, sign=1.0)

    def iadd(self, rhs):
        return _OpSpec(self, rhs, is_assign=False, sign=1.0)

    def isub(self, rhs):
        return _OpSpec(self, rhs, is_assign=False, sign=-1.0)


class _OpSpec:
    def __init__(self, lhs, rhs, is_assign, sign):
        self.lhs, self.rhs, self.is_assign, self.sign = lhs, rhs, is_assign, sign


def _to_c_labeled(lt: LabeledTensor, ids: dict, keep: list):
    """tb_labeled for one operand; labels equal within one op get equal int ids
    (the per-op int labels of MultOp::fillin_int_labels, multop.hpp:955-970)."""
    n = lt.tensor.nmodes
    lab = (C.c_int * max(n, 1))()
    sp = (A.h * max(n, 1))()
    for k, l in enumerate(lt.labels):
        if isinstance(l, TiledIndexLabel):
            key = ("L", l.id)
            sp[k] = l.tis.h
        else:
            key = ("S", l)
            sp[k] = None
        if key not in ids:
            ids[key] = -(len(ids) + 1)
        lab[k] = ids[key]
    keep += [lab, sp]
    return A.tb_labeled(lt.tensor.h, C.cast(lab, A.ip), C.cast(sp, C.POINTER(A.h)))


def apply_ewise_ip(lt: LabeledTensor, fn: int, p: float = 0.0):
    """apply_ewise_ip (tamm_utils.hpp:866): lt = fn(lt) in place, run now on lt's context."""
    Scheduler(lt.tensor.ec).map(lt, lt, fn, p).execute()


def mult_info(lhs: LabeledTensor, a: LabeledTensor, b: LabeledTensor):
    """(admitted output blocks, admitted block triples, FP64 FLOPs) of lhs += a * b,
    computed on the host without running anything."""
    ids: dict = {}
    keep: list = []
    l, x, y = (_to_c_labeled(t, ids, keep) for t in (lhs, a, b))
    ng, nt, fl = C.c_int64(), C.c_int64(), C.c_double()
    call("tb_mult_info", l, x, y, C.byref(ng), C.byref(nt), C.byref(fl))
    return ng.value, nt.value, fl.value


def opmin_order(lhs: LabeledTensor, *factors: LabeledTensor):
    """The binary steps lhs = prod(factors) runs as: [(mask, mask), ...] of factor bits in
    execution order, and the OpMin model's total cost (host only)."""
    ids: dict = {}
    keep: list = []
    l = _to_c_labeled(lhs, ids, keep)
    fs = (A.tb_labeled * len(factors))(*[_to_c_labeled(f, ids, keep) for f in factors])
    pairs = np.zeros(max(2 * (len(factors) - 1), 1), dtype=np.int64)
    cost = C.c_double()
    call("tb_opmin_order", l, fs, len(factors), pairs.ctypes.data_as(A.i64p), C.byref(cost))
    return [(int(pairs[2 * k]), int(pairs[2 * k + 1])) for k in range(len(factors) - 1)], cost.value


def mult_owned(lhs: LabeledTensor, a: LabeledTensor, b: LabeledTensor, rank: int, nranks: int):
    """Output blocks of lhs += a * b that `rank` of `nranks` computes under the
    FLOP-balanced owner rule: (packed offsets in lhs, FP64 FLOPs).  Host-only."""
    ids: dict = {}
    keep: list = []
    l, x, y = (_to_c_labeled(t, ids, keep) for t in (lhs, a, b))
    ng, fl = C.c_int64(), C.c_double()
    call("tb_mult_owned", l, x, y, int(rank), int(nranks), C.byref(ng), C.byref(fl), None, 0)
    offs = np.zeros(max(ng.value, 1), dtype=np.int64)
    call("tb_mult_owned", l, x, y, int(rank), int(nranks), C.byref(ng), C.byref(fl),
         offs.ctypes.data_as(A.i64p), ng.value)
    return offs[:ng.value].copy(), fl.value


class Scheduler:
    """Scheduler{ec}: sch(op)...execute(hw, profile)."""

    def __init__(self, ec: ExecutionContext):
        self.ec = ec
        self.h = A.h()
        call("tb_sched_create", ec.h, C.byref(self.h))
        self._keep = []

    def allocate(self, *tensors):
        for t in tensors:
            t.allocate(self.ec)
        return self

    def deallocate(self, *tensors):
        for t in tensors:
            t.deallocate()
        return self

    def _labeled(self, lt: LabeledTensor, ids: dict):
        return _to_c_labeled(lt, ids, self._keep)

    def __call__(self, spec: _OpSpec, opstr: str = "", hw=ExecutionHW.DEFAULT):
        ids: dict = {}
        lhs = self._labeled(spec.lhs, ids)
        rhs = spec.rhs
        if isinstance(rhs, (int, float)):
            call("tb_sched_set", self.h, lhs, spec.sign * float(rhs), int(spec.is_assign))
            return self
        if isinstance(rhs, LabeledTensor):
            rhs = _Product(1.0, [rhs])
        if not isinstance(rhs, _Product):
            raise TypeError("right-hand side must be a scalar, a labelled tensor or a product")
        alpha = spec.sign * rhs.alpha
        if len(rhs.factors) == 1:
            a = self._labeled(rhs.factors[0], ids)
            call("tb_sched_add", self.h, lhs, alpha, a, int(spec.is_assign))
        elif len(rhs.factors) == 2:
            a = self._labeled(rhs.factors[0], ids)
            b = self._labeled(rhs.factors[1], ids)
            call("tb_sched_mult", self.h, lhs, alpha, a, b, int(spec.is_assign))
        else:  # OpMin: the cheapest binary contraction tree, run through intermediates
            fs = (A.tb_labeled * len(rhs.factors))(*[self._labeled(f, ids) for f in rhs.factors])
            self._keep.append(fs)
            call("tb_sched_mult_n", self.h, lhs, alpha, fs, len(rhs.factors), int(spec.is_assign))
        return self

    def execute(self, hw=ExecutionHW.DEFAULT, profile=False):
        call("tb_sched_execute", self.h, int(hw), int(bool(profile)))
        return self

    def execute_async(self):
        """Enqueue the queued ops without waiting (see tb_sched_execute_async)."""
        call("tb_sched_execute_async", self.h)
        return self

    def wait(self):
        call("tb_sched_wait", self.h)
        return self

    def profile(self):
        n = C.c_int64()
        call("tb_sched_profile", self.h, C.byref(n), None, None, 0)
        ms = np.zeros(max(n.value, 1))
        fl = np.zeros(max(n.value, 1))
        call("tb_sched_profile", self.h, C.byref(n), ms.ctypes.data_as(A.dp), fl.ctypes.data_as(A.dp), n.value)
        return ms[:n.value], fl[:n.value]

    # --- device scalars, denominator update, autotuner, CUDA graphs ---
    def dot(self, slot: int, a: LabeledTensor, b: LabeledTensor, alpha: float = 1.0):
        """Queue scalar slot = alpha * sum a * b (same labels and block layout)."""
        ids: dict = {}
        call("tb_sched_dot", self.h, int(slot), float(alpha), self._labeled(a, ids), self._labeled(b, ids))
        return self

    def norm(self, slot: int, a: LabeledTensor, alpha: float = 1.0):
        """Queue scalar slot = alpha * sqrt(sum a * a)."""
        call("tb_sched_norm", self.h, int(slot), float(alpha), self._labeled(a, {}))
        return self

    def scalars(self, n: int = 64) -> np.ndarray:
        out = np.zeros(n)
        call("tb_sched_scalars", self.h, out.ctypes.data_as(A.dp), int(n))
        return out

    def denom(self, t: LabeledTensor, alpha: float, r: LabeledTensor, eps, signs):
        """Queue t += alpha * r / D, D = sum_m signs[m] * eps[orbital index of mode m]."""
        ids: dict = {}
        e = np.ascontiguousarray(np.asarray(eps, dtype=np.float64))
        sg = np.ascontiguousarray(np.asarray(list(signs) + [0.0] * (8 - len(signs)), dtype=np.float64))
        self._keep += [e, sg]
        call("tb_sched_denom", self.h, self._labeled(t, ids), float(alpha), self._labeled(r, ids),
             e.ctypes.data_as(A.dp), int(e.size), sg.ctypes.data_as(A.dp))
        return self

    def map(self, lhs: LabeledTensor, rhs: LabeledTensor, fn: int, p: float = 0.0):
        """Queue lhs = fn(rhs) element by element over lhs's admitted blocks (MapOp; rhs has
        lhs's labels in the same order and may be lhs itself)."""
        ids: dict = {}
        call("tb_sched_map", self.h, self._labeled(lhs, ids), self._labeled(rhs, ids), int(fn), float(p))
        return self

    def exact_copy(self, lhs: LabeledTensor, rhs: LabeledTensor):
        """Scheduler::exact_copy: lhs's blocks = rhs's blocks with the same tile ids."""
        return self.map(lhs, rhs, Map.COPY)

    def clear(self):
        """Drop the queued ops without running them (e.g. after an execute failed)."""
        call("tb_sched_clear", self.h)
        return self

    def release(self):
        """Free the cached plans and work lists of executed ops (see tb_sched_release)."""
        call("tb_sched_release", self.h)
        return self

    def set_owner(self, rank: int, nranks: int):
        """Mult ops compute only the output blocks `rank` owns (of `nranks`)."""
        call("tb_sched_set_owner", self.h, int(rank), int(nranks))
        return self

    def denom_energy(self, slot: int, alpha: float, w: LabeledTensor, eps, signs):
        """Queue slot += alpha * sum w^2 / D, D = sum_m signs[m] * eps[orbital index of mode m]."""
        e = np.ascontiguousarray(np.asarray(eps, dtype=np.float64))
        sg = np.ascontiguousarray(np.asarray(list(signs) + [0.0] * (8 - len(signs)), dtype=np.float64))
        self._keep += [e, sg]
        call("tb_sched_denom_energy", self.h, int(slot), float(alpha), self._labeled(w, {}),
             e.ctypes.data_as(A.dp), int(e.size), sg.ctypes.data_as(A.dp))
        return self

    def mult_energy(self, slot: int, scale: float, spec: _OpSpec, eps, signs):
        """Queue slot += scale * sum (lhs + alpha * a * b)^2 / D for spec = lhs.iadd(alpha * a * b)
        (or lhs.isub(...)), D = sum_m signs[m] * eps[orbital index of lhs mode m]: the
        contraction with the denominator energy fused into its epilogue; lhs is read, not
        written."""
        if spec.is_assign:
            raise ValueError("the energy epilogue adds to lhs's values; an assignment has none")
        rhs = spec.rhs
        if not isinstance(rhs, _Product) or len(rhs.factors) != 2:
            raise TypeError("right-hand side must be a product of two labelled tensors")
        ids: dict = {}
        lhs = self._labeled(spec.lhs, ids)
        a = self._labeled(rhs.factors[0], ids)
        b = self._labeled(rhs.factors[1], ids)
        e = np.ascontiguousarray(np.asarray(eps, dtype=np.float64))
        sg = np.ascontiguousarray(np.asarray(list(signs) + [0.0] * (8 - len(signs)), dtype=np.float64))
        self._keep += [e, sg]
        call("tb_sched_mult_energy", self.h, int(slot), float(scale), lhs, spec.sign * rhs.alpha, a, b,
             e.ctypes.data_as(A.dp), int(e.size), sg.ctypes.data_as(A.dp))
        return self

    def set_scalar(self, slot: int, value: float = 0.0):
        call("tb_sched_set_scalar", self.h, int(slot), float(value))
        return self

    def autotune(self, enable: bool = True):
        call("tb_sched_autotune", self.h, int(bool(enable)))
        return self

    def tune_info(self, index: int):
        """Autotuner choice for op `index` of the last execute: None if not tuned, else
        dict(mode, tile_n, candidates=[(mode, tile_n, ms), ...])."""
        mode, tile, nc = C.c_int(), C.c_int(), C.c_int()
        cm = (C.c_int * 8)()
        ct = (C.c_int * 8)()
        ms = (C.c_double * 8)()
        call("tb_sched_tune_info", self.h, int(index), C.byref(mode), C.byref(tile), C.byref(nc),
             C.cast(cm, A.ip), C.cast(ct, A.ip), C.cast(ms, A.dp), 8)
        if nc.value == 0:
            return None
        return {"mode": mode.value, "tile_n": tile.value,
                "candidates": [(cm[i], ct[i], ms[i]) for i in range(min(nc.value, 8))]}

    def graph(self) -> "Graph":
        """Run the queued ops once, then capture them into a CUDA graph."""
        g = A.h()
        call("tb_sched_graph_create", self.h, C.byref(g))
        return Graph(g, self)

    def op_stats(self, index=-1):
        """Kernel statistics (dict) of one op of the last profiled execute."""
        n = C.c_int64()
        call("tb_sched_profile", self.h, C.byref(n), None, None, 0)
        if index < 0:
            index += n.value
        st = A.tb_stats()
        call("tb_sched_op_stats", self.h, int(index), C.byref(st))
        return {k: getattr(st, k) for k, _ in A.tb_stats._fields_}

    def __del__(self):
        try:
            A.lib().tb_sched_destroy(self.h)
        except Exception:
            pass


class _BorrowedScheduler(Scheduler):
    """A library-owned scheduler handed to a batch builder (not destroyed from Python)."""

    def __init__(self, h):
        self.ec = None
        self.h = C.c_void_p(h) if not isinstance(h, C.c_void_p) else h
        self._keep = []

    def __del__(self):
        pass


class Graph:
    """A captured sequence of scheduler ops; launch() enqueues one replay on the
    context's stream, sync() waits and checks the device error words."""

    def __init__(self, handle, sched):
        self.h = handle
        self._sched = sched  # keeps the ops' tensors and the scheduler alive

    def launch(self):
        call("tb_graph_launch", self.h)
        return self

    def sync(self):
        call("tb_graph_sync", self.h)
        return self

    def __del__(self):
        try:
            A.lib().tb_graph_destroy(self.h)
        except Exception:
            pass


class Tape:
    """Differentiation of a contraction sequence (no counterpart in TAMM): a tape of
    Functions run eagerly on their own Scheduler, in the context's precision mode.

        tape = Tape(ec, budget_bytes)
        tape.leaf(t2, g)                                  # g accumulates dE/dt2
        tape.contract(X(a, b, i, j), v(a, b, c, d) * t2(c, d, i, j))
        e1 = tape.dot(w(i, j, a, b), t2(a, b, i, j))
        e2 = tape.dot(t2(a, b, i, j), X(a, b, i, j), 0.25)
        tape.backward()                                   # g += dE/dt2, E = e1 + e2

    Contract's backward is the pair of swapped-operand contractions dA += alpha *
    dC * B, dB += alpha * A * dC; Dot's is a pair of permuted adds.  Contract outputs
    beyond `budget_bytes` (in recording order) are freed at the start of the backward
    sweep and recomputed when needed.  Call reset() before the next evaluation."""

    def __init__(self, ec: ExecutionContext, budget_bytes: int = 1 << 62):
        self.ec = ec
        self.h = A.h()
        call("tb_tape_create", ec.h, int(budget_bytes), C.byref(self.h))
        self._keep = []

    def leaf(self, x: Tensor, grad: Tensor | None = None):
        call("tb_tape_leaf", self.h, x.h, grad.h if grad is not None else None)
        return self

    def contract(self, y: LabeledTensor, product):
        if isinstance(product, LabeledTensor) or not isinstance(product, _Product) or len(product.factors) != 2:
            raise ValueError("contract takes y(labels) and a product of two labelled tensors")
        ids: dict = {}
        l, a, b = (_to_c_labeled(t, ids, self._keep) for t in (y, product.factors[0], product.factors[1]))
        call("tb_tape_contract", self.h, l, float(product.alpha), a, b)
        return self

    def dot(self, p: LabeledTensor, q: LabeledTensor, alpha: float = 1.0) -> float:
        ids: dict = {}
        x, y = (_to_c_labeled(t, ids, self._keep) for t in (p, q))
        v = C.c_double()
        call("tb_tape_dot", self.h, float(alpha), x, y, C.byref(v))
        return v.value

    def backward(self):
        call("tb_tape_backward", self.h)
        return self

    def info(self):
        n, kept, rec = C.c_int64(), C.c_int64(), C.c_int64()
        obj = C.c_double()
        call("tb_tape_info", self.h, C.byref(n), C.byref(obj), C.byref(kept), C.byref(rec))
        return {"nodes": n.value, "objective": obj.value, "kept_bytes": kept.value, "recomputed": rec.value}

    def reset(self):
        call("tb_tape_reset", self.h)
        self._keep = []
        return self

    def __del__(self):
        try:
            A.lib().tb_tape_destroy(self.h)
        except Exception:
            pass
