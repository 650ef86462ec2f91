"""Field build on the GPU: analytic recipes and dense sampled fields into the block-sparse layout.

Drop-in surfaces with the reference's signatures:

* ``klassificera_och_evaluera_testfalt(meta, hx, hy, hz, r, corrupt_index=False, device=...)`` --
  src/field_engine/faltkarna_v1.py:258-299 (box minus unbounded z cylinder) -> SparseField.
* ``klassificera_och_evaluera_fran_tatt_falt(wp, dense, pitch, block, device)`` --
  src/field_engine/faltkarna_v1_mesh_to_sdf.py:660-692 -> dict (``wp`` accepted and ignored).
* ``rekonstruera_tat(sf)`` / ``rekonstruera_tat_gpu(sf, device=...)`` -- faltkarna_v1.py:302-350.
* ``volym_via_gpu_reduktion``-style int64 checksum: ``checksum_i64(tiles)`` (faltkarna_v1.py:250-255).

General recipes: ``build_field(node, meta) -> SparseField`` (the reference has no general builder;
the node format is src/field_engine/ikarus_v1/expr.py).  ``FieldBuilder`` keeps the compiled
recipe, scratch and outputs resident on the device for repeated / graph-captured builds.
"""
from __future__ import annotations

import ctypes as ct
import math

import weakref

import numpy as np

from . import _lib
from .expr import compile_recipe, Compiled
from .grid import BIG, FIXPT_SCALE, GridMeta, SparseField, stats_of
from . import expr as X


class FbGeom(ct.Structure):
    """C layout of fb_geom (include/field_b200.h)."""
    _fields_ = [("x0", ct.c_double), ("y0", ct.c_double), ("z0", ct.c_double), ("pitch", ct.c_double),
                ("nx", ct.c_int32), ("ny", ct.c_int32), ("nz", ct.c_int32), ("block", ct.c_int32),
                ("margin", ct.c_float), ("guard", ct.c_float), ("reserved", ct.c_int32 * 2)]


def _large_tori(c: Compiled, meta: GridMeta) -> bool:
    """A torus whose ring radius exceeds four leaf extents (block * pitch) in its own frame, the
    frame's stretch taken as the root-mean-square of its linear part (localise's rule)."""
    tori = c.prims[c.prims["type"] == X.P_TORUS]
    if not len(tori):
        return False
    a = tori["A"].reshape(-1, 3, 4)[:, :, :3]
    scale = np.sqrt((a * a).sum(axis=(1, 2)) / 3.0)
    return bool(np.any(tori["p"][:, 0] > 4.0 * meta.block * meta.pitch * scale))


def geom_of(meta: GridMeta, guard=None) -> FbGeom:
    if meta.block not in (4, 8, 16):
        raise ValueError("block must be 4, 8 or 16")
    return FbGeom(meta.x0, meta.y0, meta.z0, meta.pitch, meta.nx, meta.ny, meta.nz, meta.block,
                  float(np.float32(meta.margin_mm)), float(meta.guard() if guard is None else guard))


class DeviceField:
    """A field resident in HBM: torch tensors with the SparseField layout."""

    def __init__(self, meta, kind, cma, active, count, tiles, n_active):
        self.meta = meta
        self.kind = kind
        self.corner_min_abs = cma
        self.active = active
        self.count = count
        self.tiles = tiles
        self.n_active = n_active

    def to_host(self) -> SparseField:
        """The field as host arrays.  They land in page-locked memory from torch's caching host
        allocator (copies at full link speed; blocks return to the cache when the arrays are
        dropped, so repeated calls allocate no new pinned memory), one synchronisation for all."""
        import torch
        n = int(self.n_active)
        b = self.meta.block

        def pinned(t):
            h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            h.copy_(t, non_blocking=True)
            return h
        parts = [pinned(self.kind), pinned(self.active[:n]), pinned(self.tiles[:n].reshape(n, b, b, b)),
                 pinned(self.corner_min_abs)]
        torch.cuda.current_stream(self.kind.device).synchronize()
        kind, active, tiles, cma = (p.numpy() for p in parts)
        return SparseField(meta=self.meta, kind=kind, active_ids=active, tiles=tiles, corner_min_abs=cma,
                           stats=stats_of(self.meta, kind, n))


def device_tables(comp: Compiled, device, stream, *, alloc=None, pinned=None):
    """(primitive table, instruction table) of a compiled recipe as uint8 device tensors, validated
    and uploaded once per device and kept on the Compiled object; `stream` is made to wait for the
    upload, so builds on any stream may share the tables (the kernels only read them).

    alloc(nbytes) -> uint8 device tensor places the tables in the caller's device pool (the
    returned blocks are kept with the tables); pinned (a serve.PinnedPool) supplies the host
    staging, whose blocks go back to it through release_staging once the upload has completed
    (at the latest when the Compiled object goes away)."""
    import torch
    cache = comp.__dict__.setdefault("_device_tables", {})
    key = str(device)
    if key not in cache:
        mode = 1 if comp.chain is not None else 0
        insns = comp.chain if mode == 1 else comp.program
        if len(comp.prims) < 1:
            raise ValueError("recipe has no primitive")
        _validate_program(comp.prims, insns, mode, len(comp.tables))
        prims = comp.with_table_addresses(device_table_addresses(comp, device, stream)) if comp.tables else comp.prims
        host = [np.ascontiguousarray(prims).view(np.uint8).reshape(-1),
                np.ascontiguousarray(insns).view(np.uint8).reshape(-1)]
        handles = []
        with torch.cuda.stream(stream):
            staged, out = [], []
            for h in host:
                if pinned is not None:
                    view, handle = pinned.take(h.nbytes)
                    view.numpy()[:] = h
                    handles.append(handle)
                else:
                    view = torch.from_numpy(h.copy()).pin_memory()
                staged.append(view)
                if alloc is not None:
                    d = alloc(h.nbytes)
                    d.copy_(view, non_blocking=True)
                else:
                    d = view.to(device, non_blocking=True)
                out.append(d)
            done = torch.cuda.Event()
            done.record(stream)
        if handles:
            weakref.finalize(comp, _give_back_all, pinned, handles)
        cache[key] = (out[0], out[1], done, tuple(staged), handles)
    dprims, dchain, done = cache[key][:3]
    stream.wait_event(done)
    return dprims, dchain


def device_table_addresses(comp: Compiled, device, stream):
    """Device addresses of comp's leaf tables (float32, 256-byte aligned in one buffer), uploaded once
    per device and kept on the Compiled object; `stream` is made to wait for the upload."""
    import torch
    cache = comp.__dict__.setdefault("_device_table_data", {})
    key = str(device)
    if key not in cache:
        sizes = [(t.nbytes + 255) // 256 * 256 for t in comp.tables]
        buf = torch.empty(max(sum(sizes), 256), dtype=torch.uint8, device=device)
        addrs, at = [], 0
        with torch.cuda.stream(stream):
            for t, size in zip(comp.tables, sizes):
                buf[at:at + t.nbytes].copy_(torch.from_numpy(t.view(np.uint8).reshape(-1)))
                addrs.append(buf.data_ptr() + at)
                at += size
        cache[key] = (buf, addrs)
    return cache[key][1]


def _give_back_all(pinned, handles):
    while handles:
        pinned.give_back(handles.pop())


def release_staging(comp: Compiled, device, pinned):
    """Return the pinned staging blocks of comp's table upload to `pinned`; call it once that
    upload has completed (after an event recorded on the upload stream behind it)."""
    entry = comp.__dict__.get("_device_tables", {}).get(str(device))
    if entry is not None and entry[4]:
        _give_back_all(pinned, entry[4])


class FieldBuilder:
    """Compiled recipe + scratch + outputs for one grid, resident on one device.

    ``build()`` returns a DeviceField sized exactly (one 4-byte count read between the classify and
    leaf launches); ``enqueue(capacity_tiles)`` runs the whole build stream-ordered into a fixed
    tile buffer (CUDA-graph capturable).  ``alloc`` (optional) supplies the one device allocation
    the builder makes (outputs + scratch), e.g. from a server's memory pool, and -- with
    ``pinned`` -- the recipe's tables when they are first uploaded (see device_tables).  ``tables``
    (a pair of uint8 device tensors: primitive records, chain or program records) uses tables the
    caller placed on the device instead, e.g. a batch's table arena."""

    def __init__(self, recipe, meta: GridMeta, *, device="cuda", guard=None, library=None, alloc=None,
                 pinned=None, tables=None):
        import torch
        self.lib = _lib.lib(library)
        self.meta = meta
        self.device = torch.device(device)
        self.compiled: Compiled = recipe if isinstance(recipe, Compiled) else compile_recipe(recipe)
        c = self.compiled
        self.mode = 1 if c.chain is not None else 0
        insns = c.chain if self.mode == 1 else c.program
        self.n_prims = len(c.prims)
        self.n_chain = len(insns)
        if self.n_prims < 1:
            raise ValueError("recipe has no primitive")
        if guard is None and c.tables:  # float32 table samples carry more error than the default band
            guard = max(meta.guard(), c.sampling_guard())
        self.geom = geom_of(meta, guard)
        # fb_geom.reserved[0] bit 0: sampled-grid leaves present (the kernels then mark the voxels at
        # a table's boundary for the float64 recheck); bit 1: a torus whose ring radius exceeds four
        # leaf extents in its frame (the leaf evaluates it in its ring frame, float32 within 1e-5
        # pitch there)
        self.geom.reserved[0] = int(bool(np.any(c.prims["type"] == X.P_GRID))) | (2 * int(_large_tori(c, meta)))
        if tables is not None:
            # the caller placed the tables on the device (e.g. a batch's table arena); still checked
            _validate_program(c.prims, insns, self.mode, len(c.tables))
            self.prims, self.chain = tables
            if self.prims.numel() != c.prims.nbytes or self.chain.numel() != insns.nbytes:
                raise ValueError("device tables do not match the compiled recipe")
        else:
            self.prims, self.chain = device_tables(c, self.device, torch.cuda.current_stream(self.device),
                                                   alloc=alloc, pinned=pinned)
        nbytes = self.lib.fb_field_scratch_bytes(ct.addressof(self.geom), self.n_prims, self.n_chain)
        if nbytes < 0:
            raise ValueError("grid outside the build contract")
        # one device allocation carved into the outputs and the scratch (256-byte aligned parts);
        # count[0] is written by every classification, so nothing needs clearing here
        nb = meta.n_blocks
        part = lambda n: (n + 255) // 256 * 256
        sizes = (part(nb * 4), part(nb * 4), part(nb * 4), 256, part(int(nbytes)))
        # `alloc(nbytes) -> uint8 device tensor` lets a caller place the slab in its own memory pool
        self.slab = (alloc(sum(sizes)) if alloc is not None
                     else torch.empty(sum(sizes), dtype=torch.uint8, device=self.device))
        views, at = [], 0
        for size in sizes:
            views.append(self.slab[at:at + size])
            at += size
        self.kind = views[0][:nb * 4].view(torch.int32)
        self.cma = views[1][:nb * 4].view(torch.float32)
        self.active = views[2][:nb * 4].view(torch.int32)
        self.count = views[3][:4].view(torch.int32)
        self.scratch = views[4][:int(nbytes)]

    def _args(self):
        return (ct.addressof(self.geom), self.prims.data_ptr(), self.n_prims, self.chain.data_ptr(), self.n_chain,
                self.mode)

    def classify(self, stream=None):
        st = self.lib.fb_field_classify_device(*self._args(), self.kind.data_ptr(), self.cma.data_ptr(),
                                               self.active.data_ptr(), self.count.data_ptr(), self.scratch.data_ptr(),
                                               self.scratch.numel(), _lib.stream_handle(stream))
        _lib.check(st, "field classify")

    def leaf(self, tiles, capacity, active=None, stream=None):
        act = self.active if active is None else active
        st = self.lib.fb_field_leaf_device(*self._args(), self.kind.data_ptr(), act.data_ptr(), self.count.data_ptr(),
                                           tiles.data_ptr(),
                                           int(capacity), self.scratch.data_ptr(), self.scratch.numel(),
                                           _lib.stream_handle(stream))
        _lib.check(st, "field leaf")

    def enqueue(self, tiles, capacity, stream=None):
        """Whole build into `tiles` (>= capacity * B^3 floats), no host synchronisation."""
        st = self.lib.fb_field_build_device(*self._args(), self.kind.data_ptr(), self.cma.data_ptr(),
                                            self.active.data_ptr(), self.count.data_ptr(), tiles.data_ptr(),
                                            int(capacity), self.scratch.data_ptr(), self.scratch.numel(),
                                            _lib.stream_handle(stream))
        _lib.check(st, "field build")

    def compact_error(self, stream=None) -> int:
        return self.lib.fb_field_compact_error(ct.addressof(self.geom), self.n_prims, self.n_chain,
                                               self.scratch.data_ptr(), _lib.stream_handle(stream))

    def build(self, stream=None, corrupt_index=False) -> DeviceField:
        import torch
        self.classify(stream)
        n = int(self.count.item())
        b3 = self.meta.block ** 3
        tiles = torch.empty((max(n, 1), b3), dtype=torch.float32, device=self.device)
        if n:
            active = self.active
            if corrupt_index:
                # planted fault (faltkarna_v1.py:177-180): evaluate every tile one block further on
                active = self.active.clone()
                active[:n] += 1
            self.leaf(tiles, n, active=active, stream=stream)
        if self.compact_error(stream):
            raise RuntimeError("compaction wait timed out")
        return DeviceField(self.meta, self.kind, self.cma, self.active, self.count, tiles, n)


def _validate_program(prims, insns, mode, n_tables=0):
    """Every instruction names a valid operation and, where it reads one, an existing primitive;
    the device kernels index the primitive table with these arguments unchecked.  Primitive kinds
    are known ones and every table-backed record names an existing table."""
    n = len(prims)
    if len(prims) and ((prims["type"] < X.P_SPHERE) | (prims["type"] > X.P_XBORE)).any():
        raise ValueError("unknown primitive kind")
    tab = np.isin(prims["type"], X.TABLE_KINDS)
    if tab.any():
        idx = prims["p"][tab, 9]
        if ((idx < 0) | (idx >= n_tables) | (idx != np.floor(idx))).any():
            raise ValueError("table-backed primitive names no table")
    ops = insns["op"]
    args = insns["arg"]
    if mode == 1:
        if len(insns) == 0 or ops[0] not in (X.CH_SET, X.CH_SETNEG):
            raise ValueError("chain must start with a set")
        reads = ops != X.CH_OFFSET
        if ((ops < X.CH_SET) | (ops > X.CH_OFFSET)).any():
            raise ValueError("unknown chain operation")
    else:
        reads = ops == X.OP_PUSH
        if ((ops < X.OP_PUSH) | (ops > X.OP_OFFSET)).any():
            raise ValueError("unknown program operation")
        depth = np.cumsum(np.where(ops == X.OP_PUSH, 1, np.where(ops == X.OP_OFFSET, 0, -1)))
        if depth.min() < 1 or depth[-1] != 1 or depth.max() > 32:
            raise ValueError("malformed postfix program")
    if reads.any() and ((args[reads] < 0) | (args[reads] >= n)).any():
        raise ValueError("instruction names a primitive outside the table")
    if not np.isfinite(insns["k"]).all() or not np.isfinite(prims["p"]).all() or not np.isfinite(prims["A"]).all():
        raise ValueError("non-finite recipe parameter")


def build_field(recipe, meta: GridMeta, *, device="cuda", guard=None, corrupt_index=False) -> SparseField:
    """Classify, compact and evaluate an analytic recipe into a SparseField on the host."""
    fb = FieldBuilder(recipe, meta, device=device, guard=guard)
    return fb.build(corrupt_index=corrupt_index).to_host()


def testfalt(hx, hy, hz, r):
    """Box (half extents hx, hy, hz at the origin) minus the unbounded z cylinder of radius r
    (src/field_engine/faltkarna_v1.py:121-126)."""
    return X.subtract(X.box((hx, hy, hz), (0.0, 0.0, 0.0)), X.cylinder_z_infinite(r, (0.0, 0.0)))


def klassificera_och_evaluera_testfalt(meta: GridMeta, hx, hy, hz, r, corrupt_index=False,
                                       device="cuda:0") -> SparseField:
    """Rasterise the test field (box minus cylinder) into a SparseField (faltkarna_v1.py:258-299).
    ``corrupt_index=True`` plants the block-index fault of the reference's self-test."""
    return build_field(testfalt(hx, hy, hz, r), meta, device=device, corrupt_index=corrupt_index)


def klassificera_och_evaluera_fran_tatt_falt(wp, dense: np.ndarray, pitch: float, block: int, device="cuda:0"):
    """Sparse classification of a dense float32 SDF by the 8-corner rule
    (src/field_engine/faltkarna_v1_mesh_to_sdf.py:660-692).  ``wp`` is accepted and ignored."""
    import torch
    lib = _lib.lib()
    d = np.ascontiguousarray(dense, dtype=np.float32)
    if d.ndim != 3:
        raise ValueError("dense field must be 3-D")
    nx, ny, nz = d.shape
    n_bx, n_by, n_bz = -(-nx // block), -(-ny // block), -(-nz // block)
    n_blocks = n_bx * n_by * n_bz
    margin = math.sqrt(3.0) * block * pitch
    dev = torch.device(device)
    dd = torch.from_numpy(d).to(dev)
    kind = torch.empty(n_blocks, dtype=torch.int32, device=dev)
    active = torch.empty(n_blocks, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    b3 = block ** 3
    tiles = torch.empty((n_blocks, b3), dtype=torch.float32, device=dev)
    scratch = torch.empty(int(lib.fb_dense_scratch_bytes(nx, ny, nz, block)), dtype=torch.uint8, device=dev)
    st = lib.fb_dense_classify_device(dd.data_ptr(), nx, ny, nz, block, float(np.float32(margin)), kind.data_ptr(),
                                      None, active.data_ptr(), count.data_ptr(), tiles.data_ptr(), n_blocks,
                                      scratch.data_ptr(), scratch.numel(), _lib.stream_handle())
    _lib.check(st, "dense classify")
    n = int(count.item())
    return dict(kind=kind.cpu().numpy(), active_ids=active[:n].cpu().numpy().astype(np.int32),
                tiles=tiles[:n].reshape(n, block, block, block).cpu().numpy(), n_bx=n_bx, n_by=n_by, n_bz=n_bz,
                n_blocks=int(n_blocks), n_active=int(n), margin_mm=margin)


def reconstruct_device(kind, active, n_active, tiles, meta: GridMeta):
    """Dense (nx, ny, nz) float32 CUDA tensor from device-resident sparse arrays."""
    import torch
    lib = _lib.lib()
    dev = kind.device
    slot = torch.empty(meta.n_blocks, dtype=torch.int32, device=dev)
    out = torch.empty((meta.nx, meta.ny, meta.nz), dtype=torch.float32, device=dev)
    st = lib.fb_field_reconstruct_device(kind.data_ptr(), active.data_ptr() if n_active else None, int(n_active),
                                         tiles.data_ptr() if n_active else None, meta.nx, meta.ny, meta.nz, meta.block,
                                         float(BIG), slot.data_ptr(), out.data_ptr(), _lib.stream_handle())
    _lib.check(st, "reconstruct")
    return out


def rekonstruera_tat_gpu(sf: SparseField, device="cuda:0") -> np.ndarray:
    """Dense (nx, ny, nz) float32 array: tiles in active blocks, -BIG / +BIG elsewhere
    (faltkarna_v1.py:328-350)."""
    import torch
    dev = torch.device(device)
    kind = torch.from_numpy(np.ascontiguousarray(sf.kind, dtype=np.int32)).to(dev)
    n = len(sf.active_ids)
    active = torch.from_numpy(np.ascontiguousarray(sf.active_ids, dtype=np.int32)).to(dev)
    tiles = torch.from_numpy(np.ascontiguousarray(sf.tiles, dtype=np.float32).reshape(max(n, 0), -1)).to(dev)
    return reconstruct_device(kind, active, n, tiles, sf.meta).cpu().numpy()


def rekonstruera_tat(sf: SparseField) -> np.ndarray:
    """Same result as rekonstruera_tat_gpu (faltkarna_v1.py:302-325); computed on the device."""
    return rekonstruera_tat_gpu(sf)


def checksum_i64(values, scale=FIXPT_SCALE) -> int:
    """Deterministic int64 fixed-point sum of the negative values (faltkarna_v1.py:250-255)."""
    import torch
    lib = _lib.lib()
    v = values if hasattr(values, "data_ptr") else torch.from_numpy(np.ascontiguousarray(values, np.float32)).cuda()
    v = v.reshape(-1).contiguous()
    out = torch.zeros(1, dtype=torch.int64, device=v.device)
    _lib.check(lib.fb_checksum_i64_device(v.data_ptr(), v.numel(), float(scale), out.data_ptr(),
                                          _lib.stream_handle()), "checksum")
    return int(out.item())
