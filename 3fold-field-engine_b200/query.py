"""SDF value and gradient point queries of recipes on the GPU.

Drop-in surfaces:

* ``eval_batch(node, points_mm, device=...)`` -> float32 (N,) -- src/field_engine/ikarus_v1/eval_warp.py:478-488.
* ``gradient_batch(node, points_mm, h=0.05, device=...)`` -> float32 (N, 3) central differences --
  eval_warp.py:718-733.

``RecipeQueries`` keeps a compiled recipe resident and, when given a FieldBuilder of the same
recipe, answers points inside that grid from their superblock's culled list (exact) instead of
the whole chain; it serves value and value+gradient queries of device tensors without host
round trips.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib
from .expr import Compiled, compile_recipe
from .build import device_tables

PRIMF_BYTES = 128


class RecipeQueries:
    """A compiled recipe resident on one device, with optional acceleration by a built field."""

    def __init__(self, recipe, *, device="cuda", builder=None):
        import torch
        self.lib = _lib.lib()
        self.device = torch.device(device)
        self.compiled: Compiled = recipe if isinstance(recipe, Compiled) else compile_recipe(recipe)
        c = self.compiled
        self.mode = 1 if c.chain is not None else 0
        insns = c.chain if self.mode == 1 else c.program
        self.n_chain = len(insns)
        self.prims, self.chain = device_tables(c, self.device, torch.cuda.current_stream(self.device))
        self.primf = torch.empty(len(c.prims) * PRIMF_BYTES, dtype=torch.uint8, device=self.device)
        _lib.check(self.lib.fb_query_prepare(self.prims.data_ptr(), len(c.prims), self.primf.data_ptr(),
                                             _lib.stream_handle()), "query prepare")
        self._accel = None
        if builder is not None and self.mode == 1:
            self.attach(builder)

    def attach(self, builder):
        """Use `builder`'s superblock lists (the builder must have classified this same recipe)."""
        pool, off, ln = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
        boff, blen, bpool = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
        bcap, ball = ct.c_int64(), ct.c_int32()
        st = self.lib.fb_field_accel(ct.addressof(builder.geom), builder.n_prims, builder.n_chain,
                                     builder.scratch.data_ptr(), ct.byref(pool), ct.byref(off), ct.byref(ln),
                                     ct.byref(boff), ct.byref(blen), ct.byref(bpool), ct.byref(bcap), ct.byref(ball))
        _lib.check(st, "field accel")
        m = builder.meta
        self._accel = (pool.value, off.value, ln.value, np.array([m.x0, m.y0, m.z0, m.pitch], np.float64),
                       np.array([m.nx, m.ny, m.nz, m.block], np.int32),
                       (builder.kind.data_ptr(), boff.value, blen.value, bpool.value, bcap.value, ball.value), builder)

    def _run(self, pts, value, grad, h=0.05, stream=None, alloc=None):
        """alloc(nbytes) -> uint8 device tensor for the sorted path's scratch, which the alloc's
        owner keeps alive until the query's kernels have completed (default: torch's allocator,
        with the block tied to `stream`)."""
        import torch
        a = self._accel
        scratch, nscratch = None, 0
        if a is not None and pts.shape[0] > 0:
            nbytes = int(self.lib.fb_query_scratch_bytes(a[4].ctypes.data, pts.shape[0], 1 if grad is not None else 0))
            if nbytes > 0:
                nscratch = nbytes
                if alloc is not None:
                    scratch = alloc(nbytes)
                else:
                    scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
                    if isinstance(stream, torch.cuda.Stream):  # freed only after that stream's kernels
                        scratch.record_stream(stream)
        args = (a[0], a[1], a[2], a[3].ctypes.data, a[4].ctypes.data, *a[5]) if a else (None,) * 5 + (None, None,
                                                                                                     None, None, 0, 0)
        st = self.lib.fb_query_points_device(self.primf.data_ptr(), self.chain.data_ptr(), self.n_chain, self.mode,
                                             *args, pts.data_ptr(), pts.shape[0], float(h),
                                             value.data_ptr() if value is not None else None,
                                             grad.data_ptr() if grad is not None else None,
                                             scratch.data_ptr() if scratch is not None else None, nscratch,
                                             _lib.stream_handle(stream))
        _lib.check(st, "point query")

    def values(self, points, *, stream=None):
        """float32 (N,) values at a float32 (N, 3) CUDA tensor of points."""
        import torch
        pts = points.to(self.device, torch.float32).contiguous()
        out = torch.empty(pts.shape[0], dtype=torch.float32, device=self.device)
        self._run(pts, out, None, stream=stream)
        return out

    def values_and_gradients(self, points, h=0.05, *, stream=None, alloc=None):
        """(float32 (N,), float32 (N, 3)) values and central-difference gradients.  alloc: as in
        _run, also used for the two outputs (whose blocks the alloc's owner keeps alive)."""
        import torch
        pts = points.to(self.device, torch.float32).contiguous()
        n = pts.shape[0]
        if alloc is not None:
            val = alloc(max(n, 1) * 4).view(torch.float32)[:n]
            grad = alloc(max(n, 1) * 12).view(torch.float32)[:3 * n].view(n, 3)
        else:
            val = torch.empty(n, dtype=torch.float32, device=self.device)
            grad = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        self._run(pts, val, grad, h=h, stream=stream, alloc=alloc)
        return val, grad


def _points(points_mm):
    pts = np.asarray(points_mm)
    if pts.ndim != 2 or pts.shape[1] != 3:
        raise ValueError("points must be an (N, 3) array")
    return pts


def eval_batch(node, points_mm, device="cuda"):
    """(N,) float32 SDF values of `node` at (N, 3) points (eval_warp.py:478-488)."""
    import torch
    pts = _points(points_mm)
    q = RecipeQueries(node, device=device)
    return q.values(torch.from_numpy(pts.astype(np.float32))).cpu().numpy()


def gradient_batch(node, points_mm, h=0.05, device="cuda"):
    """(N, 3) float32 central-difference gradients with step h (eval_warp.py:718-733)."""
    import torch
    pts = _points(points_mm)
    q = RecipeQueries(node, device=device)
    pts_t = torch.from_numpy(np.asarray(pts, dtype=np.float32)).to(q.device)
    grad = torch.empty((len(pts), 3), dtype=torch.float32, device=q.device)
    q._run(pts_t, None, grad, h=h)
    return grad.cpu().numpy()


_GRID_UPLOADS = {}  # (leaf identities, device) -> (params tensor, table buffer)


def _pack_gridfields(grid_leaves, device):
    """Every gridfield leaf's table in one device buffer (256-byte aligned parts) and a float32
    record of 12 per leaf (origin, pitch, iso, is_sdf, nx, ny, nz, -, table address halves); loaded
    and uploaded once per (leaves, device), as the reference caches its packing
    (src/field_engine/ikarus_v1/eval_warp.py:430-475)."""
    import torch
    from .expr import _load_gridfield
    key = (tuple((lf["npz_path"], lf["key"], lf["mode"], float(lf["iso"]), lf.get("pitch_override"))
                 for lf in grid_leaves), str(device))
    if key in _GRID_UPLOADS:
        return _GRID_UPLOADS[key]
    loaded = [_load_gridfield(lf) for lf in grid_leaves]
    sizes = [(a.nbytes + 255) // 256 * 256 for a, _, _ in loaded]
    buf = torch.empty(max(sum(sizes), 256), dtype=torch.uint8, device=device)
    params = np.zeros((len(loaded), 12), np.float32)
    at = 0
    for k, ((arr, origin, pitch), lf, size) in enumerate(zip(loaded, grid_leaves, sizes)):
        buf[at:at + arr.nbytes].copy_(torch.from_numpy(arr.view(np.uint8).reshape(-1)))
        addr = buf.data_ptr() + at
        params[k, :9] = (origin[0], origin[1], origin[2], pitch, lf["iso"], 1.0 if lf["mode"] == "sdf" else 0.0,
                         *arr.shape)
        params[k, 10:12] = np.array([addr & 0xFFFFFFFF, addr >> 32], np.uint32).view(np.float32)
        at += size
    entry = (torch.from_numpy(params).to(device), buf)
    _GRID_UPLOADS[key] = entry
    return entry


def eval_batch_multi_pair(points_mm, pair_of_point, leaf_a_of_pair, leaf_b_of_pair, grid_leaves_all,
                          device="cuda"):
    """max(sdf_A, sdf_B) at every point, its pair's two gridfield leaves chosen per point, all pairs
    in one launch (src/field_engine/ikarus_v1/eval_warp.py:545-564): points (N, 3), pair_of_point
    (N,) pair ids, leaf_a_of_pair / leaf_b_of_pair (n_pairs,) indices into grid_leaves_all (gridfield
    node dicts).  Returns (N,) float32."""
    import torch
    pts = _points(points_mm)
    pop = np.ascontiguousarray(pair_of_point, dtype=np.int32).reshape(-1)
    la = np.ascontiguousarray(leaf_a_of_pair, dtype=np.int32).reshape(-1)
    lb = np.ascontiguousarray(leaf_b_of_pair, dtype=np.int32).reshape(-1)
    if len(pop) != len(pts) or len(la) != len(lb) or len(la) < 1 or len(grid_leaves_all) < 1:
        raise ValueError("one pair id per point and two leaves per pair required")
    if pop.size and (pop.min() < 0 or pop.max() >= len(la)):
        raise ValueError("pair id outside the pairs")
    if la.min() < 0 or lb.min() < 0 or max(la.max(), lb.max()) >= len(grid_leaves_all):
        raise ValueError("leaf index outside grid_leaves_all")
    dev = torch.device(device)
    params, _buf = _pack_gridfields(list(grid_leaves_all), dev)
    d_pts = torch.from_numpy(pts.astype(np.float32)).to(dev)
    d_pop, d_la, d_lb = (torch.from_numpy(a).to(dev) for a in (pop, la, lb))
    out = torch.empty(len(pts), dtype=torch.float32, device=dev)
    _lib.check(_lib.lib().fb_grid_pairs_device(params.data_ptr(), len(grid_leaves_all), d_pts.data_ptr(),
                                               d_pop.data_ptr(), len(pts), d_la.data_ptr(), d_lb.data_ptr(), len(la),
                                               out.data_ptr(), _lib.stream_handle()), "eval_batch_multi_pair")
    return out.cpu().numpy()
