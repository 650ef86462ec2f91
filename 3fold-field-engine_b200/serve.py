"""Serving: a continuous-batching request loop over device-resident fields.

Requests (``submit`` returns a Future):
  * ``build``  (recipe, GridMeta)               -> new resident field id + stats
  * ``edit``   (field id, tools, op)             -> the field rebuilt with tool primitives unioned
                                                   or subtracted (milling / drilling edits)
  * ``query``  (field id, points (N, 3))         -> float32 values and central-difference gradients
  * ``edt``    (field id)                        -> squared EDT of the field's occupancy (device)

Request preparation (compiling a recipe, compiling edit tools to primitive records, copying query
points given as numpy arrays into pinned host memory) runs on the submitting thread; points given as
pinned host or device tensors are used without a host copy.  Query results are numpy arrays over
pooled pinned blocks, which return to the pool when the client drops them.  The scheduler thread admits queued
requests while a stream slot is free and the HBM budget allows their estimated footprint, runs
each request as a generator that enqueues asynchronous GPU work on its slot's stream and yields a
CUDA event, resumes it when the event has completed, and admits the next arrival as soon as a slot
frees -- so requests that arrive while others are on the GPU overlap with them on the device.

Per field, requests take effect in submission order: a request waits while an earlier request on
the same field is still queued or an earlier edit of it is still running, so every result is the
one the same requests give one at a time.  An edit appends the compiled tools to the field's chain
(no recompilation of the recipe) and rebuilds into new buffers; requests already running keep
reading the previous version.  Resident fields are evicted least-recently-used when an admission
would exceed the budget.  The reference's service is one synchronous request at a time over a pipe
(src/field_engine/mesh_field_service_v1.py:44-113); its timeout/close behaviour is kept: a failed or
timed-out request fails its future, the server stays usable.
"""
from __future__ import annotations

import bisect
import collections
import threading
import time
import weakref
from concurrent.futures import Future

import numpy as np

from . import _lib
from . import expr as X
from .build import FieldBuilder, release_staging
from .query import RecipeQueries


class DeviceArena:
    """One device allocation handed out by first fit, so that resident fields do not each cost a
    cudaMalloc (which can stall the whole process for tens of milliseconds on large sizes).

    ``alloc(nbytes)`` returns a uint8 view of the arena, or None when no free range fits.  The range
    returns to the free list when that view object is garbage collected: keep it referenced for as
    long as any tensor derived from it is in use (derived views do not keep it alive).  In the server
    a field's buffers die only after every request that used them has seen its GPU work complete, so
    a returned range is never still being written."""

    ALIGN = 512

    def __init__(self, nbytes, device):
        import torch
        self.nbytes = int(nbytes) // self.ALIGN * self.ALIGN
        self.base = torch.empty(self.nbytes, dtype=torch.uint8, device=device)
        self.free = [(0, self.nbytes)]  # (offset, size), sorted by offset, coalesced
        self.used = 0
        self.lock = threading.Lock()

    def alloc(self, nbytes):
        n = max(self.ALIGN, (int(nbytes) + self.ALIGN - 1) // self.ALIGN * self.ALIGN)
        with self.lock:
            for i, (off, size) in enumerate(self.free):
                if size >= n:
                    if size == n:
                        del self.free[i]
                    else:
                        self.free[i] = (off + n, size - n)
                    self.used += n
                    break
            else:
                return None
        view = self.base[off:off + int(nbytes)]
        weakref.finalize(view, self._release, off, n)
        return view

    def _release(self, off, n):
        with self.lock:
            self.used -= n
            i = bisect.bisect_left(self.free, (off, 0))
            # merge with the following and the preceding free range
            if i < len(self.free) and self.free[i][0] == off + n:
                n += self.free[i][1]
                del self.free[i]
            if i > 0 and self.free[i - 1][0] + self.free[i - 1][1] == off:
                off, n = self.free[i - 1][0], self.free[i - 1][1] + n
                del self.free[i - 1]
                i -= 1
            self.free.insert(i, (off, n))


class PinnedPool:
    """Pinned host blocks handed out by power-of-two size class and recycled, so that a request's
    host staging costs no pinned allocation once the pool has warmed up (a fresh pinned allocation
    is a driver call that can take milliseconds and holds the caller).

    ``take(nbytes)`` returns (uint8 pinned view, handle).  ``bind(obj, handle)`` returns the block
    to the pool when `obj` -- the numpy array handed to a client, say -- is garbage collected;
    ``give_back(handle)`` returns it at once."""

    MIN = 1 << 16

    def __init__(self):
        self.free = collections.defaultdict(list)  # size class -> pinned uint8 tensors
        self.lock = threading.Lock()
        self.allocated = 0

    def _new(self, cls):
        import torch
        return torch.empty(cls, dtype=torch.uint8, pin_memory=True)

    SPAN = 2  # a request may take a free block up to 2^SPAN times its own size class

    @classmethod
    def size_class(cls, nbytes):
        return max(cls.MIN, 1 << max(0, int(nbytes) - 1).bit_length())

    def take(self, nbytes):
        """A free block of nbytes' size class, else of one of the next SPAN classes up (so small
        requests do not drain the blocks kept for large ones); a new block of the class only when
        none of those is free."""
        cls = self.size_class(nbytes)
        blk, got = None, cls
        with self.lock:
            for k in range(self.SPAN + 1):
                lst = self.free.get(cls << k)
                if lst:
                    blk, got = lst.pop(), cls << k
                    break
        if blk is None:
            blk = self._new(cls)
            self.allocated += cls
        return blk[:int(nbytes)], (got, blk)

    def bind(self, obj, handle):
        weakref.finalize(obj, self.give_back, handle)

    def reserve(self, nbytes, count):
        """Make sure at least `count` blocks of nbytes' own size class are free (allocating ahead
        of need)."""
        cls = self.size_class(nbytes)
        with self.lock:
            missing = count - len(self.free[cls])
        for _ in range(max(0, missing)):
            blk = self._new(cls)
            self.allocated += cls
            self.give_back((cls, blk))

    def give_back(self, handle):
        cls, blk = handle
        with self.lock:
            self.free[cls].append(blk)


class _Field:
    def __init__(self, fid, comp, meta, fb, tiles, n_active):
        self.id = fid
        self.comp = comp
        self.meta = meta
        self.fb = fb
        self.tiles = tiles
        self.n_active = n_active
        self.queries = None  # (RecipeQueries, CUDA event marking its tables ready)
        self.edt = None
        self.owners = []  # arena blocks behind tiles / edt (they must outlive those views)
        self.busy = 0
        self.editing = False
        self.last_use = time.perf_counter()
        self.accounted = 0  # bytes of this field in the server's resident total

    @property
    def nbytes(self):
        """Device bytes the field holds: the build's slab (block arrays + scratch), tiles, EDT."""
        t = [self.fb.slab, self.tiles]
        if self.edt is not None:
            t.append(self.edt)
        return int(sum(x.numel() * x.element_size() for x in t))


class _Request:
    def __init__(self, kind, args):
        self.kind = kind
        self.args = args
        self.future = Future()
        self.arrival = time.perf_counter()
        self.start = None
        self.end = None
        self.gen = None
        self.event = None
        self.slot = None
        self.estimate = 0

    @property
    def field(self):
        return self.args.get("field")


def _prepare(kind, args):
    """Caller-thread preparation: compiled recipes and tools, pinned float32 points."""
    import torch
    if kind == "build":
        r = args["recipe"]
        args["recipe"] = r if isinstance(r, X.Compiled) else X.compile_recipe(r)
    elif kind == "edit":
        op = args.get("op", "subtract")
        if op not in ("union", "subtract"):
            raise ValueError("edit op must be union or subtract")
        tools = args["tools"]
        args["tool_prims"] = tools if isinstance(tools, np.ndarray) else X.compile_tools(tools)
        args["op"] = op
    elif kind == "query":
        p = args["points"]
        if isinstance(p, torch.Tensor):
            # taken as given: pinned or device tensors are staged asynchronously; a pageable host
            # tensor is copied synchronously when the request runs
            if p.dim() != 2 or p.shape[1] != 3:
                raise ValueError("points must be an (N, 3) array")
            args["points"] = p.to(torch.float32).contiguous()
        else:
            a = np.ascontiguousarray(p, dtype=np.float32)
            if a.ndim != 2 or a.shape[1] != 3:
                raise ValueError("points must be an (N, 3) array")
            args["points"] = torch.from_numpy(a).pin_memory()


class FieldServer:
    def __init__(self, *, device="cuda", slots=8, budget_bytes=150e9, request_timeout_s=30.0, arena_bytes=0):
        """arena_bytes > 0: resident field buffers come from one DeviceArena of that size (requests
        that do not fit fall back to the caching allocator)."""
        import torch
        dev = torch.device(device)
        # an explicit index: the scheduler thread selects this device with torch.cuda.set_device
        self.device = dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())
        self.arena = DeviceArena(arena_bytes, self.device) if arena_bytes else None
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(slots)]
        # per slot: a pinned word area for the scalars its request reads back (active count, EDT
        # checksum); a slot runs one request at a time, so it is never shared
        self.slot_host = [torch.zeros(8, dtype=torch.int64, pin_memory=True) for _ in range(slots)]
        self.slot_dev = torch.zeros((slots, 8), dtype=torch.int64, device=self.device)
        self.pinned = PinnedPool()
        self.free = collections.deque(range(slots))
        self.budget = float(budget_bytes)
        self.timeout = float(request_timeout_s)
        self.fields = collections.OrderedDict()  # least recently used first
        self.resident = 0  # sum of the resident fields' bytes, kept up to date on every change
        self.next_id = 0
        self.reserved = 0
        self.pending = []
        self.inflight = []
        self.lock = threading.Lock()
        self.wake = threading.Event()
        self.running = True
        self.completed = []
        self.thread = threading.Thread(target=self._loop, name="field-server", daemon=True)
        self.thread.start()

    # ------------------------------------------------------------------------------------ client API
    def submit(self, kind, **args) -> Future:
        if kind not in ("build", "edit", "query", "edt"):
            raise ValueError(f"unknown request kind {kind!r}")
        r = _Request(kind, args)
        try:
            _prepare(kind, args)
        except Exception as e:  # an unusable request fails its own future
            r.end = time.perf_counter()
            r.future.set_exception(e)
            return r.future
        with self.lock:
            if not self.running:
                raise RuntimeError("server closed")
            self.pending.append(r)
        self.wake.set()
        return r.future

    def close(self):
        with self.lock:
            self.running = False
        self.wake.set()
        self.thread.join(timeout=60)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def resident_bytes(self):
        return self.resident

    def reserve_pinned(self, nbytes, count):
        """Pre-allocate `count` pinned staging blocks for results of up to nbytes (e.g. query
        outputs: 4 B per point for values, 12 B for gradients), so the first bursts of requests
        of that size meet no pinned allocation."""
        self.pinned.reserve(nbytes, count)

    def _alloc(self, nbytes):
        """uint8 device block for a resident buffer or a request's temporaries: from the arena,
        evicting least-recently-used idle fields while it is full; torch's allocator only when
        nothing more can be evicted."""
        import torch
        if self.arena is not None:
            blk = self.arena.alloc(nbytes)
            while blk is None and self._evict_lru():
                blk = self.arena.alloc(nbytes)
            if blk is not None:
                return blk
        return torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)

    def _keeper(self, keep):
        """alloc(nbytes) for a request's device temporaries: blocks from _alloc, each appended to
        `keep`, the request's list that lives until its last device event has completed (a derived
        tensor does not keep an arena block alive; the block object itself must)."""
        def alloc(nbytes):
            blk = self._alloc(nbytes)
            keep.append(blk)
            return blk
        return alloc

    def _account(self, f):
        """Bring the resident total up to date after field `f` changed its buffers."""
        now = f.nbytes
        self.resident += now - f.accounted
        f.accounted = now

    # ------------------------------------------------------------------------------------ scheduler
    def _estimate(self, r):
        if r.kind in ("build", "edit"):
            meta = r.args["meta"] if r.kind == "build" else self.fields[r.field].meta
            # culling lists + block arrays + a quarter of the blocks active (tiles), grown on demand
            return int(meta.n_blocks * (meta.block ** 3) + meta.n_blocks * 64 + 64e6)
        if r.kind == "query":
            return int(len(r.args["points"]) * 32)
        meta = self.fields[r.field].meta
        return int(meta.nx * meta.ny * meta.nz * 14)

    def _evict_for(self, need):
        """Drop least-recently-used idle fields until `need` more bytes fit in the budget."""
        while self.resident + self.reserved + need > self.budget:
            if not self._evict_lru():
                return False
        return True

    def _evict_lru(self):
        """Drop the least-recently-used idle resident field (its buffers return to the arena once
        nothing holds them); False when every resident field is in use."""
        for f in self.fields.values():  # oldest use first
            if not f.busy and not f.editing:
                del self.fields[f.id]
                self.resident -= f.accounted
                return True
        return False

    def _touch(self, f):
        f.last_use = time.perf_counter()
        if f.id in self.fields:
            self.fields.move_to_end(f.id)

    def _admit(self):
        """Start queued requests, oldest first, while a slot is free and the budget allows; a
        request whose field has an earlier request still queued, or an edit still running, waits
        without holding back requests on other fields.  Returns the requests now waiting on a
        device event."""
        started = []
        with self.lock:
            queue = list(self.pending)
        if not queue:
            return started
        taken = set()
        held = set()  # fields with an earlier request still queued
        for r in queue:
            if not self.free:
                break
            if r.kind != "build":
                f = self.fields.get(r.field)
                if f is None:
                    if r.field in held:
                        continue
                    taken.add(id(r))
                    r.end = time.perf_counter()
                    r.future.set_exception(KeyError(f"field {r.field} is not resident"))
                    continue
                if r.field in held or f.editing:
                    held.add(r.field)
                    continue
            r.estimate = self._estimate(r)
            if not self._evict_for(r.estimate):
                break  # wait for memory, oldest first: in-flight requests release their reservations
            taken.add(id(r))
            r.slot = self.free.popleft()
            self.reserved += r.estimate
            r.start = time.perf_counter()
            if r.kind != "build":
                f = self.fields[r.field]
                f.busy += 1
                f.editing = r.kind == "edit"
            r.gen = getattr(self, f"_run_{r.kind}")(r, self.streams[r.slot])
            if self._step(r):
                started.append(r)
        if taken:
            with self.lock:
                self.pending = [r for r in self.pending if id(r) not in taken]
        return started

    def _finish(self, r, result=None, error=None):
        r.end = time.perf_counter()
        self.free.append(r.slot)
        self.reserved -= r.estimate
        if r.kind != "build" and r.field in self.fields:
            f = self.fields[r.field]
            f.busy -= 1
            self._touch(f)
            if r.kind == "edit":
                f.editing = False
        self.completed.append((r.kind, r.arrival, r.start, r.end))
        if error is not None:
            r.future.set_exception(error)
        else:
            r.future.set_result(result)

    def _step(self, r):
        """Run the request up to its next device event; False when it has finished."""
        try:
            r.event = next(r.gen)
        except StopIteration as stop:
            self._finish(r, result=stop.value)
            return False
        except Exception as e:  # a failed request fails its future; the server stays usable
            self._finish(r, error=e)
            return False
        return True

    def _loop(self):
        try:
            self._loop_body()
        except BaseException as e:  # the scheduler itself failed: fail every request, refuse new ones
            with self.lock:
                self.running = False
                waiting = list(self.pending) + list(self.inflight)
                self.pending = []
            self.inflight = []
            for r in waiting:
                if not r.future.done():
                    r.future.set_exception(RuntimeError(f"field server stopped: {e!r}"))

    def _loop_body(self):
        import torch
        torch.cuda.set_device(self.device)
        while True:
            with self.lock:
                running = self.running
                idle = not self.pending and not self.inflight
            if not running and idle:
                return
            self.wake.clear()
            progressed = False
            still = []
            for r in self.inflight:
                if not r.event.query():
                    if time.perf_counter() - r.start > self.timeout:
                        self._finish(r, error=TimeoutError("request exceeded the server timeout"))
                        progressed = True
                    else:
                        still.append(r)
                    continue
                progressed = True
                if self._step(r):
                    still.append(r)
            self.inflight = still
            started = self._admit()
            self.inflight += started
            if not progressed and not started:
                # new submissions set `wake`; device completions are polled
                self.wake.wait(timeout=0.0001 if self.inflight else 0.01)

    # ------------------------------------------------------------------------------------ request bodies
    def _record(self, stream):
        import torch
        ev = torch.cuda.Event()
        ev.record(stream)
        return ev

    def _build_field(self, comp, meta, stream, slot):
        import torch
        with torch.cuda.stream(stream):
            fb = FieldBuilder(comp, meta, device=self.device, alloc=self._alloc, pinned=self.pinned)
            fb.classify(stream)
            count = self.slot_host[slot].view(torch.int32)[:1]
            count.copy_(fb.count, non_blocking=True)
        yield self._record(stream)
        # the tables' upload (if this build made it) ran on this stream ahead of the classification
        release_staging(comp, self.device, self.pinned)
        n = int(count[0])
        with torch.cuda.stream(stream):
            b3 = meta.block ** 3
            owner = self._alloc(max(n, 1) * b3 * 4)
            tiles = owner.view(torch.float32).view(max(n, 1), b3)
            if n:
                fb.leaf(tiles, n, stream=stream)
        yield self._record(stream)
        return fb, tiles, owner, n

    def _run_build(self, r, stream):
        comp, meta = r.args["recipe"], r.args["meta"]
        fb, tiles, owner, n = yield from self._build_field(comp, meta, stream, r.slot)
        fid = self.next_id
        self.next_id += 1
        self.fields[fid] = _Field(fid, comp, meta, fb, tiles, n)
        self.fields[fid].owners = [owner]
        self._account(self.fields[fid])
        return dict(field=fid, n_active=n, leaf_voxels=n * meta.block ** 3)

    def _run_edit(self, r, stream):
        f = self.fields[r.field]
        comp = X.extend(f.comp, r.args["tool_prims"], r.args["op"])
        fb, tiles, owner, n = yield from self._build_field(comp, f.meta, stream, r.slot)
        f.comp, f.fb, f.tiles, f.n_active = comp, fb, tiles, n
        f.queries = None
        f.edt = None
        f.owners = [owner]
        if f.id in self.fields:
            self._account(f)
        return dict(field=f.id, n_active=n, leaf_voxels=n * f.meta.block ** 3)

    def _run_query(self, r, stream):
        import torch
        f = self.fields[r.field]
        pts = r.args["points"]
        h = float(r.args.get("h", f.meta.pitch))
        keep = []  # device temporaries, alive until the request's device work has completed
        alloc = self._keeper(keep)
        with torch.cuda.stream(stream):
            if f.queries is None:
                # tables prepared on this stream; later queries on other streams wait for them
                f.queries = (RecipeQueries(f.comp, device=self.device, builder=f.fb), self._record(stream))
            q, ready = f.queries
            stream.wait_event(ready)
            n = pts.shape[0]
            if pts.is_cuda:
                p = pts
            else:
                p = alloc(max(n, 1) * 12).view(torch.float32)[:3 * n].view(n, 3)
                p.copy_(pts, non_blocking=True)
            val, grad = q.values_and_gradients(p, h=h, stream=stream, alloc=alloc)
            hv, tok_v = self.pinned.take(max(n, 1) * 4)
            hg, tok_g = self.pinned.take(max(n, 1) * 12)
            out_v = hv.view(torch.float32)[:n]
            out_g = hg.view(torch.float32)[:3 * n].view(n, 3)
            out_v.copy_(val, non_blocking=True)
            out_g.copy_(grad, non_blocking=True)
        try:
            yield self._record(stream)
        except BaseException:
            self.pinned.give_back(tok_v)
            self.pinned.give_back(tok_g)
            raise
        arr_v, arr_g = out_v.numpy(), out_g.numpy()
        # the pinned blocks go back to the pool when the client drops these arrays
        self.pinned.bind(arr_v, tok_v)
        self.pinned.bind(arr_g, tok_g)
        del keep
        return arr_v, arr_g

    def _run_edt(self, r, stream):
        import torch
        f = self.fields[r.field]
        m = f.meta
        lib = _lib.lib()
        fb, tiles, n_active, owners = f.fb, f.tiles, f.n_active, list(f.owners)  # held until the GPU is done
        keep = []  # device temporaries, alive until the request's device work has completed
        alloc = self._keeper(keep)
        with torch.cuda.stream(stream):
            slot = alloc(m.n_blocks * 4).view(torch.int32)
            mask = alloc(m.nx * m.ny * m.nz).view(m.nx, m.ny, m.nz)
            out_owner = self._alloc(m.nx * m.ny * m.nz * 4)
            out = out_owner.view(torch.int32).view(m.nx, m.ny, m.nz)
            scratch = alloc(int(lib.fb_edt_scratch_bytes(m.nx, m.ny, m.nz, 0)))
            _lib.check(lib.fb_field_occupancy_device(fb.kind.data_ptr(), fb.active.data_ptr(), fb.count.data_ptr(),
                                                     tiles.data_ptr(), max(n_active, 1), m.nx, m.ny, m.nz, m.block,
                                                     slot.data_ptr(), mask.data_ptr(), _lib.stream_handle(stream)),
                       "occupancy")
            _lib.check(lib.fb_edt_squared_device(mask.data_ptr(), m.nx, m.ny, m.nz, 1, out.data_ptr(),
                                                 scratch.data_ptr(), scratch.numel(), _lib.stream_handle(stream)),
                       "edt")
            total = self.slot_dev[r.slot, 0:1]
            _lib.check(lib.fb_sum_i32_device(out.data_ptr(), out.numel(), total.data_ptr(),
                                             _lib.stream_handle(stream)), "edt checksum")
            host = self.slot_host[r.slot][1:2]
            host.copy_(total, non_blocking=True)
        yield self._record(stream)
        del keep
        if f.fb is fb:
            f.edt = out
            f.owners = owners + [out_owner]
            if f.id in self.fields:
                self._account(f)
        return dict(field=f.id, checksum=int(host.item()), voxels=int(out.numel()))
