"""Batched builds of many independent recipes: device work-lists, one launch per phase, a tuner.

``BatchBuilder(recipes)`` keeps every recipe's compiled tables, culling scratch and outputs resident
(one FieldBuilder slab each) and builds them all with ``fb_batch_build_device``: each phase -- the
float32 mirror of the tables, two culling levels, classification (a thread per block culling its
superblock's list; the active blocks keep their lists), compaction, the leaf tiles -- is one
launch over a work-list spanning every recipe, so the small recipes fill the GPU beside the large
ones.  The active counts, each recipe's place in the tile arena and the active-block work-lists
are formed on the device: a build has no host synchronisation and allocates nothing, and the ~10
launches can be captured into one CUDA graph.  With ``edt=True``
every build is followed by each recipe's occupancy rasterisation (batched) and the squared EDT of
that occupancy (distance to the solid), spread over side streams.

``plain_build(...)`` is the same work recipe by recipe through the public single-build path
(classification, a host read of the active count, leaf evaluation, then occupancy and EDT when
asked), the reference's own orchestration (src/field_engine/faltkarna_v1_g7_fix.py:56-112:
classify, host read of the kinds, compaction, tile evaluation).

``Autotuner`` chooses the leaf size (4, 8 or 16) per recipe: it times the three sizes on one
representative recipe of each (grid size, primitive-count octave) bucket and keeps the fastest
build per bucket in a JSON table; ``BatchBuilder.tune_schedule`` then times the batch's grid
sizing of the active-block passes (CTAs per SM).  The reference's nearest counterpart is its
two-term cost model cached per kernel shape (src/field_engine/ikarus_v1/cost_model_v1_2.py:1-112).
"""
from __future__ import annotations

import ctypes as ct
import json
import math
from pathlib import Path

import numpy as np

from . import _lib
from .build import DeviceField, FieldBuilder, device_table_addresses
from .expr import Compiled, compile_recipe
from .grid import GridMeta

LEAF_SIZES = (4, 8, 16)
SCHEDULES = (8, 16, 32)  # CTAs per SM of the active-block passes


def cube_meta(n, block):
    """Unit-cube grid of n^3 vertex samples at pitch 1/n."""
    return GridMeta(0.0, 0.0, 0.0, 1.0 / n, n, n, n, block)


class Autotuner:
    """Leaf size per (grid edge, primitive-count octave) bucket, by measurement."""

    def __init__(self, path=None, device="cuda"):
        self.path = Path(path) if path else None
        self.device = device
        self.table = {}
        if self.path and self.path.exists():
            self.table = json.loads(self.path.read_text())

    @staticmethod
    def bucket(n, n_prims):
        return f"{int(n)}:{int(math.log2(max(n_prims, 1)))}"

    def _time_build(self, comp, n, block, reps=2):
        import torch
        fb = FieldBuilder(comp, cube_meta(n, block), device=self.device)
        fb.classify()
        cap = max(int(fb.count.item()), 1)
        tiles = torch.empty((cap, block ** 3), dtype=torch.float32, device=fb.device)
        best = float("inf")
        for _ in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fb.enqueue(tiles, cap)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    def tune(self, recipes):
        """recipes: list of (compiled recipe, grid edge n).  Fills the table for every bucket seen
        and returns the leaf size of each recipe."""
        todo = {}
        for comp, n in recipes:
            key = self.bucket(n, len(comp.prims))
            if key not in self.table and key not in todo:
                todo[key] = (comp, n)
        for key, (comp, n) in todo.items():
            times = {b: self._time_build(comp, n, b) for b in LEAF_SIZES}
            self.table[key] = dict(block=min(times, key=times.get), ms={str(b): t for b, t in times.items()})
        if self.path and todo:
            self.path.write_text(json.dumps(self.table, indent=1, sort_keys=True))
        return [int(self.table[self.bucket(n, len(comp.prims))]["block"]) for comp, n in recipes]


class _Item(ct.Structure):
    """C layout of fb_batch_item (include/field_b200.h)."""
    _fields_ = [("geom", ct.c_void_p), ("d_prims", ct.c_void_p), ("d_chain", ct.c_void_p),
                ("n_prims", ct.c_int32), ("n_chain", ct.c_int32), ("d_kind", ct.c_void_p), ("d_cma", ct.c_void_p),
                ("d_active", ct.c_void_p), ("d_count", ct.c_void_p), ("d_scratch", ct.c_void_p),
                ("scratch_len", ct.c_int64), ("d_slot", ct.c_void_p), ("d_mask", ct.c_void_p)]


class BatchBuilder:
    """Many chain recipes built together.  recipes: list of (recipe or Compiled, GridMeta).

    capacity: floats of the tile arena (default 30 % of every recipe's voxels; ``ensure_capacity``
    grows it to the exact need after a build that ran out).  edt: keep per-recipe occupancy masks and
    EDT outputs, filled by ``enqueue(edt=True)``.  streams: side streams of the per-recipe EDTs."""

    def __init__(self, recipes, *, device="cuda", capacity=None, edt=False, streams=8, ctas_per_sm=0):
        import torch
        self.device = torch.device(device)
        self.lib = _lib.lib()
        self.has_edt = bool(edt)
        self.ctas_per_sm = int(ctas_per_sm)
        comps = []
        for r, meta in recipes:
            comp = r if isinstance(r, Compiled) else compile_recipe(r)
            if comp.chain is None:
                raise ValueError("batched builds take chain recipes (hard/smooth booleans reducing to a chain)")
            comps.append(comp)
        # every recipe's primitive and chain tables in one device buffer (256-byte aligned parts), with
        # a pinned host image: upload_tables() refreshes all of them with one copy
        parts, sizes = [], []
        for comp in comps:
            prims = comp.prims
            if comp.tables:  # leaf tables live in their own per-device buffers (see device_table_addresses)
                prims = comp.with_table_addresses(device_table_addresses(comp, self.device,
                                                                         torch.cuda.current_stream(self.device)))
            for arr in (prims, comp.chain):
                b = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
                parts.append(b)
                sizes.append((b.nbytes + 255) // 256 * 256)
        total = int(sum(sizes))
        self.table_host = torch.empty(max(total, 1), dtype=torch.uint8).pin_memory()
        self.table_dev = torch.empty(max(total, 1), dtype=torch.uint8, device=self.device)
        views, at = [], 0
        host = self.table_host.numpy()
        for b, size in zip(parts, sizes):
            host[at:at + b.nbytes] = b
            views.append(self.table_dev[at:at + b.nbytes])
            at += size
        self.upload_tables()
        self.builders = []
        for k, ((_, meta), comp) in enumerate(zip(recipes, comps)):
            self.builders.append(FieldBuilder(comp, meta, device=self.device, tables=(views[2 * k], views[2 * k + 1])))
        self.metas = [fb.meta for fb in self.builders]
        self.slots, self.masks, self.edts = [], [], []
        if self.has_edt:
            for m in self.metas:
                self.slots.append(torch.empty(m.n_blocks, dtype=torch.int32, device=self.device))
                self.masks.append(torch.empty((m.nx, m.ny, m.nz), dtype=torch.uint8, device=self.device))
                self.edts.append(torch.empty((m.nx, m.ny, m.nz), dtype=torch.int32, device=self.device))
        n = len(self.builders)
        self._items = (_Item * n)()
        for i, fb in enumerate(self.builders):
            it = self._items[i]
            it.geom = ct.addressof(fb.geom)
            it.d_prims, it.d_chain = fb.prims.data_ptr(), fb.chain.data_ptr()
            it.n_prims, it.n_chain = fb.n_prims, fb.n_chain
            it.d_kind, it.d_cma, it.d_active, it.d_count = (fb.kind.data_ptr(), fb.cma.data_ptr(),
                                                             fb.active.data_ptr(), fb.count.data_ptr())
            it.d_scratch, it.scratch_len = fb.scratch.data_ptr(), fb.scratch.numel()
            if self.has_edt:
                it.d_slot, it.d_mask = self.slots[i].data_ptr(), self.masks[i].data_ptr()
        self.handle = self.lib.fb_batch_create(self._items, n, _lib.stream_handle())
        if not self.handle:
            raise RuntimeError("fb_batch_create failed")
        self.b3 = np.array([m.block ** 3 for m in self.metas], np.int64)
        if capacity is None:
            capacity = int(0.3 * sum(m.n_blocks * m.block ** 3 for m in self.metas))
        self.tiles = torch.empty(max(int(capacity), 1), dtype=torch.float32, device=self.device)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, streams))] if edt else []
        self.edt_scratch = []
        if self.has_edt:
            edt_max = max(int(self.lib.fb_edt_scratch_bytes(m.nx, m.ny, m.nz, 0)) for m in self.metas)
            self.edt_scratch = [torch.empty(edt_max, dtype=torch.uint8, device=self.device) for _ in self.streams]
        # largest EDT grids first, dealt round-robin: the side streams finish close together
        self.edt_order = sorted(range(n), key=lambda i: -self.metas[i].nx * self.metas[i].ny * self.metas[i].nz)
        self.graphs = {}
        off, cnt = ct.c_void_p(), ct.c_void_p()
        _lib.check(self.lib.fb_batch_outputs(self.handle, ct.byref(off), ct.byref(cnt)), "batch outputs")
        self._tile_off_ptr, self._leaf_count_ptr = off.value, cnt.value

    def __len__(self):
        return len(self.builders)

    def upload_tables(self, stream=None):
        """Copy every recipe's tables from the pinned host image to the device (one transfer)."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.stream(st):
            self.table_dev.copy_(self.table_host, non_blocking=True)

    @property
    def table_bytes(self):
        return int(self.table_host.numel())

    @property
    def launches(self):
        """Launches of one build (and with the EDT form: occupancy + 3 per recipe's EDT)."""
        n = int(self.lib.fb_batch_launches(self.handle))
        if self.has_edt:
            n += 5 + 3 * len(self)
        return n

    def close(self):
        if getattr(self, "handle", None):
            self.lib.fb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _with_edt(self, edt):
        edt = self.has_edt if edt is None else bool(edt)
        if edt and not self.has_edt:
            raise ValueError("this BatchBuilder was made with edt=False")
        return edt

    def enqueue(self, edt=None, stream=None):
        """One build of every recipe on `stream` (default: the current stream), then, with edt,
        occupancy and the squared EDT of each recipe on the side streams, joined back."""
        import torch
        edt = self._with_edt(edt)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        h = _lib.stream_handle(st)
        _lib.check(self.lib.fb_batch_build_device(self.handle, self.tiles.data_ptr(), self.tiles.numel(),
                                                  self.ctas_per_sm, h), "batch build")
        self._after_build(edt, st, h)

    def enqueue_timed(self, events, work=None, stream=None, edt=False):
        """enqueue() recording six torch CUDA events at the phase boundaries (start, culling,
        classification with the active blocks' lists, compaction, an empty phase, leaves); `work`
        (int64[2] device tensor) adds
        the leaf pass's executed evaluations and float32 operations."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        for e in events:
            if not e.cuda_event:  # torch creates the event at its first record
                e.record(st)
        h = _lib.stream_handle(st)
        ev = (ct.c_void_p * 6)(*[e.cuda_event for e in events])
        _lib.check(self.lib.fb_batch_build_timed_device(self.handle, self.tiles.data_ptr(), self.tiles.numel(),
                                                        self.ctas_per_sm, ev,
                                                        work.data_ptr() if work is not None else None, h),
                   "batch build")
        self._after_build(self._with_edt(edt), st, h)

    def _after_build(self, edt, st, h):
        if not edt:
            return
        _lib.check(self.lib.fb_batch_occupancy_device(self.handle, self.tiles.data_ptr(), h), "batch occupancy")
        for s in self.streams:
            s.wait_stream(st)
        for k, i in enumerate(self.edt_order):
            j = k % len(self.streams)
            m = self.metas[i]
            # distance of every voxel to the solid: sites are the nonzero occupancy bytes
            _lib.check(self.lib.fb_edt_squared_device(self.masks[i].data_ptr(), m.nx, m.ny, m.nz, 1,
                                                      self.edts[i].data_ptr(), self.edt_scratch[j].data_ptr(),
                                                      self.edt_scratch[j].numel(), _lib.stream_handle(self.streams[j])),
                       "edt")
        for s in self.streams:
            st.wait_stream(s)

    def capture(self, edt=None):
        """Record one build into a CUDA graph (after one eager build has configured the kernels);
        one graph per form (build only, build + EDT)."""
        import torch
        edt = self._with_edt(edt)
        self.enqueue(edt)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.enqueue(edt)
        torch.cuda.synchronize(self.device)
        self.graphs[edt] = g
        return g

    def replay(self, edt=None):
        edt = self._with_edt(edt)
        if edt not in self.graphs:
            self.capture(edt)
        self.graphs[edt].replay()

    def status(self, stream=None) -> int:
        """0, 6 (a compaction wait gave up) or 8 (the tile arena was too small); synchronises."""
        return int(self.lib.fb_batch_status(self.handle, _lib.stream_handle(stream)))

    def _host_array(self, ptr, n, dtype):
        out = np.empty(n, dtype)
        _lib.check(self.lib.fb_copy_device(out.ctypes.data, ptr, out.nbytes, _lib.stream_handle()), "copy")
        import torch
        torch.cuda.current_stream(self.device).synchronize()
        return out

    def tile_offsets(self):
        """Host copy of each recipe's tile offset (floats into self.tiles) after a build."""
        return self._host_array(self._tile_off_ptr, len(self), np.int64)

    def leaf_counts(self):
        """Host copy of the tiles each recipe got (its active blocks, unless the arena ran out)."""
        return self._host_array(self._leaf_count_ptr, len(self), np.int32)

    def active_counts(self):
        import torch
        return torch.cat([fb.count for fb in self.builders]).cpu().numpy()

    def ensure_capacity(self, edt=None):
        """After a build: when the arena was too small, grow it to the exact need and build again.
        Returns True when it grew (captured graphs are dropped: they hold the old arena)."""
        st = self.status()
        if st == 6:
            raise RuntimeError("batch build: a compaction wait timed out")
        if st != 8:
            return False
        import torch
        need = int((self.active_counts().astype(np.int64) * self.b3).sum())
        self.tiles = torch.empty(max(need, 1), dtype=torch.float32, device=self.device)
        self.graphs = {}
        self.enqueue(edt)
        if self.status() != 0:
            raise RuntimeError("batch build failed after growing the tile arena")
        return True

    @property
    def leaf_voxels(self):
        """Leaf voxels of the last build (host read)."""
        return int((self.leaf_counts().astype(np.int64) * self.b3).sum())

    def field(self, i, offsets=None, counts=None) -> DeviceField:
        """Recipe i's field after a build: its kind / active / count and a view of its tiles."""
        offsets = self.tile_offsets() if offsets is None else offsets
        counts = self.leaf_counts() if counts is None else counts
        fb = self.builders[i]
        b3 = int(self.b3[i])
        n = int(counts[i])
        tiles = self.tiles[int(offsets[i]):int(offsets[i]) + n * b3].view(n, b3)
        return DeviceField(fb.meta, fb.kind, fb.cma, fb.active, fb.count, tiles, n)

    def tune_schedule(self, reps=3):
        """Time the build at each schedule (CTAs per SM of the active-block passes) and keep the
        fastest; returns {schedule: ms}."""
        import torch
        times = {}
        for c in SCHEDULES:
            self.ctas_per_sm = c
            best = float("inf")
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self.enqueue(edt=False)
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            times[c] = best
        self.ctas_per_sm = min(times, key=times.get)
        self.graphs = {}
        return times


class PlainBuffers:
    """Per-recipe tile buffers (and, for the EDT form, occupancy and EDT buffers) of the plain path,
    sized from known active counts."""

    def __init__(self, builders, counts, edt=False):
        import torch
        self.builders = builders
        self.tiles = [torch.empty((max(int(c), 1), fb.meta.block ** 3), dtype=torch.float32, device=fb.device)
                      for fb, c in zip(builders, counts)]
        self.capacity = [max(int(c), 1) for c in counts]
        self.slot = self.mask = self.edt = None
        if edt:
            self.slot = [torch.empty(fb.meta.n_blocks, dtype=torch.int32, device=fb.device) for fb in builders]
            self.mask = [torch.empty((fb.meta.nx, fb.meta.ny, fb.meta.nz), dtype=torch.uint8, device=fb.device)
                         for fb in builders]
            self.edt = [torch.empty((fb.meta.nx, fb.meta.ny, fb.meta.nz), dtype=torch.int32, device=fb.device)
                        for fb in builders]


def plain_build(buf: PlainBuffers, edt_scratch=None):
    """The same work recipe by recipe on the current stream, with the single-build path's host
    synchronisation (the active count is read before each leaf pass); occupancy + EDT per recipe
    when edt_scratch is given."""
    import torch
    lib = _lib.lib()
    for i, fb in enumerate(buf.builders):
        fb.classify()
        n = int(fb.count.item())
        if n:
            fb.leaf(buf.tiles[i], min(n, buf.capacity[i]))
        if edt_scratch is None:
            torch.cuda.current_stream().synchronize()
            continue
        m = fb.meta
        _lib.check(lib.fb_field_occupancy_device(fb.kind.data_ptr(), fb.active.data_ptr(), fb.count.data_ptr(),
                                                 buf.tiles[i].data_ptr(), buf.capacity[i], m.nx, m.ny, m.nz, m.block,
                                                 buf.slot[i].data_ptr(), buf.mask[i].data_ptr(), _lib.stream_handle()),
                   "occupancy")
        _lib.check(lib.fb_edt_squared_device(buf.mask[i].data_ptr(), m.nx, m.ny, m.nz, 1, buf.edt[i].data_ptr(),
                                             edt_scratch.data_ptr(), edt_scratch.numel(), _lib.stream_handle()),
                   "edt")
        torch.cuda.current_stream().synchronize()
