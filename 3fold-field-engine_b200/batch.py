"""Batched builds of many independent recipes: one CUDA graph, several streams, an autotuner.

``BatchBuilder(recipes)`` prepares every recipe once (compiled tables, scratch, fixed-capacity
tile buffers and, with ``edt=True``, occupancy masks and EDT outputs) and records the whole batch
-- per recipe: culling, classification, compaction and fused leaf evaluation (the field build),
optionally followed by occupancy rasterisation and the squared EDT of that occupancy -- into one
CUDA graph whose branches are spread over ``streams`` streams.  A replay launches everything with
one host call and no host synchronisation in between; the recipes' kernels overlap on the device.

``plain_build(...)`` is the same work done recipe by recipe through the public single-build path
(classification, a host read of the active count, leaf evaluation, then occupancy and EDT when
asked), the reference's own orchestration (src/field_engine/faltkarna_v1_g7_fix.py:56-112: classify,
host read of the kinds, compaction, tile evaluation).

``Autotuner`` chooses the leaf size (4, 8 or 16) per recipe: it times the three sizes on one
representative recipe of each (grid size, primitive-count octave) bucket and keeps the fastest
build per bucket in a JSON table; the reference's nearest counterpart is its two-term cost model
cached per kernel shape (src/field_engine/ikarus_v1/cost_model_v1_2.py:1-112).
"""
from __future__ import annotations

import json
import math
import time
from pathlib import Path

import numpy as np

from . import _lib
from .build import FieldBuilder
from .expr import Compiled, compile_recipe
from .grid import GridMeta

LEAF_SIZES = (4, 8, 16)


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


class _Item:
    """One recipe's resident state."""

    def __init__(self, comp, meta, device, edt=True):
        import torch
        self.meta = meta
        self.fb = FieldBuilder(comp, meta, device=device)
        self.fb.classify()
        self.capacity = max(int(self.fb.count.item()), 1)
        self.tiles = torch.empty((self.capacity, meta.block ** 3), dtype=torch.float32, device=self.fb.device)
        self.slot = self.mask = self.edt = None
        if edt:
            self.slot = torch.empty(meta.n_blocks, dtype=torch.int32, device=self.fb.device)
            self.mask = torch.empty((meta.nx, meta.ny, meta.nz), dtype=torch.uint8, device=self.fb.device)
            self.edt = torch.empty((meta.nx, meta.ny, meta.nz), dtype=torch.int32, device=self.fb.device)

    @property
    def leaf_voxels(self):
        return self.capacity * self.meta.block ** 3

    def enqueue(self, edt_scratch, stream=None):
        """The field build; then occupancy and EDT when edt_scratch is given."""
        lib = self.fb.lib
        self.fb.enqueue(self.tiles, self.capacity, stream=stream)
        if edt_scratch is None:
            return
        m = self.meta
        st = lib.fb_field_occupancy_device(self.fb.kind.data_ptr(), self.fb.active.data_ptr(), self.fb.count.data_ptr(),
                                           self.tiles.data_ptr(), self.capacity, m.nx, m.ny, m.nz, m.block,
                                           self.slot.data_ptr(), self.mask.data_ptr(), _lib.stream_handle(stream))
        _lib.check(st, "occupancy")
        # distance of every voxel to the solid: sites are the nonzero occupancy bytes
        st = lib.fb_edt_squared_device(self.mask.data_ptr(), m.nx, m.ny, m.nz, 1, self.edt.data_ptr(),
                                       edt_scratch.data_ptr(), edt_scratch.numel(), _lib.stream_handle(stream))
        _lib.check(st, "edt")


class BatchBuilder:
    """Many recipes, one CUDA graph.  recipes: list of (recipe or Compiled, GridMeta)."""

    def __init__(self, recipes, *, device="cuda", streams=8, edt=True):
        import torch
        self.device = torch.device(device)
        self.has_edt = bool(edt)
        self.items = [_Item(r if isinstance(r, Compiled) else compile_recipe(r), meta, self.device, edt=self.has_edt)
                      for r, meta in recipes]
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, streams))]
        self.edt_scratch = []
        if self.has_edt:
            edt_max = max(int(_lib.lib().fb_edt_scratch_bytes(it.meta.nx, it.meta.ny, it.meta.nz, 0))
                          for it in self.items)
            self.edt_scratch = [torch.empty(edt_max, dtype=torch.uint8, device=self.device) for _ in self.streams]
        self.graphs = {}
        # largest recipes first, dealt round-robin: the streams finish close together
        self.order = sorted(range(len(self.items)), key=lambda i: -self.items[i].meta.n_blocks)

    @property
    def leaf_voxels(self):
        return sum(it.leaf_voxels for it in self.items)

    def _with_edt(self, edt):
        edt = self.has_edt if edt is None else bool(edt)
        if edt and not self.has_edt:
            raise ValueError("this BatchBuilder was made with edt=False")
        return edt

    def enqueue(self, edt=None):
        """All recipes, stream-ordered on the side streams, joined back on the current stream.
        edt: also occupancy + EDT per recipe (default: when the builder holds their buffers)."""
        import torch
        edt = self._with_edt(edt)
        main = torch.cuda.current_stream(self.device)
        for s in self.streams:
            s.wait_stream(main)
        for k, i in enumerate(self.order):
            j = k % len(self.streams)
            with torch.cuda.stream(self.streams[j]):
                self.items[i].enqueue(self.edt_scratch[j] if edt else None, stream=self.streams[j])
        for s in self.streams:
            main.wait_stream(s)

    def capture(self, edt=None):
        """Record the batch into one CUDA graph (after one eager run has configured every kernel);
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

    @property
    def graph(self):
        return self.graphs.get(self.has_edt)

    def replay(self, edt=None):
        edt = self._with_edt(edt)
        if edt not in self.graphs:
            self.capture(edt)
        self.graphs[edt].replay()

    def check_counts(self):
        """True when every recipe still has the active count its tiles were sized for."""
        return all(int(it.fb.count.item()) == it.capacity for it in self.items)


def plain_build(items, edt_scratch=None):
    """The same work recipe by recipe on the current stream, with the single-build path's host
    synchronisation (the active count is read before each leaf pass); occupancy + EDT per recipe
    when edt_scratch is given."""
    import torch
    lib = _lib.lib()
    for it in items:
        fb = it.fb
        fb.classify()
        n = int(fb.count.item())
        if n:
            fb.leaf(it.tiles, min(n, it.capacity))
        if edt_scratch is None:
            torch.cuda.current_stream().synchronize()
            continue
        m = it.meta
        _lib.check(lib.fb_field_occupancy_device(fb.kind.data_ptr(), fb.active.data_ptr(), fb.count.data_ptr(),
                                                 it.tiles.data_ptr(), it.capacity, m.nx, m.ny, m.nz, m.block,
                                                 it.slot.data_ptr(), it.mask.data_ptr(), _lib.stream_handle()),
                   "occupancy")
        _lib.check(lib.fb_edt_squared_device(it.mask.data_ptr(), m.nx, m.ny, m.nz, 1, it.edt.data_ptr(),
                                             edt_scratch.data_ptr(), edt_scratch.numel(), _lib.stream_handle()),
                   "edt")
        torch.cuda.current_stream().synchronize()
