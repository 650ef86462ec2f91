"""Per-block pitch (multiresolution) fields on the GPU.

``MultiresField`` keeps the reference's fields (src/field_engine/faltkarna_v1_multires.py:84-104):
a brick lattice of ``block`` coarse voxels per brick edge, ``kind`` (-1 / 0 / +1 per brick),
``niva`` (level per active brick, -1 elsewhere) and, per active brick of level l, a
(block*2^l + 1)^3 float32 sample lattice at pitch h/2^l.  The brick arrays and the sample pool
live on the device; ``tiles`` materialises the reference's {brick id: array} dict on demand.

* ``bygg_multires_fran_recept(recipe, lo, h_grov, brick_shape, block=8, levels=...)`` builds one
  from an analytic recipe (classification of the brick lattice, then the lattices of the active
  bricks at their levels); the reference builds from a mesh (bygg_multires, :254-361), which is
  out of scope here.
* ``avstand(F, punkter)`` and ``gradient(F, punkter)`` -- :405-459 -- answer on the GPU.
* ``lagg_overlappsband(F)`` (:211-251, on the device) and ``kontinuitetscheck(F)`` (:462-521).
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .build import FieldBuilder
from .grid import GridMeta
from .query import PRIMF_BYTES

NIVAER = (0, 1, 2)


@dataclass
class MultiresField:
    lo: np.ndarray
    h_grov: float
    block: int
    brick_shape: tuple
    kind: np.ndarray     # (n_bx, n_by, n_bz) int8
    niva: np.ndarray     # (n_bx, n_by, n_bz) int8, -1 outside active bricks
    margin_mm: float
    stats: dict = field(default_factory=dict)
    _dev: dict = field(default_factory=dict, repr=False)

    @property
    def L(self) -> float:
        return self.block * self.h_grov

    def pitch_of(self, lvl: int) -> float:
        return self.h_grov / float(1 << int(lvl))

    @property
    def tiles(self) -> dict:
        """{brick linear id: (n_l+1)^3 float32 array} copied from the device."""
        pool = self._dev["pool"].cpu().numpy()
        off = self._dev["tile_off_host"]
        out = {}
        for lin in np.flatnonzero(self.kind.ravel() == 0):
            m = self.block * (1 << int(self.niva.ravel()[lin])) + 1
            out[int(lin)] = pool[off[lin]:off[lin] + m ** 3].reshape(m, m, m)
        return out


def levels_by_list_length(list_lengths, thresholds=(2, 4)):
    """Level per active brick from the length of its culled primitive list: 0 below thresholds[0],
    1 below thresholds[1], else 2 (bricks where several primitives interact get the fine pitch);
    a brick whose list did not fit the per-block store (-1) gets level 2."""
    active = list_lengths
    counts = np.asarray(active, dtype=np.int64)
    lv = np.zeros(len(counts), np.int8)
    lv[counts >= thresholds[0]] = 1
    lv[counts >= thresholds[1]] = 2
    lv[counts < 0] = 2
    return lv


def _accel(builder):
    L = builder.lib
    pool, off, ln = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
    boff, blen, bpool = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
    st = L.fb_field_accel(ct.addressof(builder.geom), builder.n_prims, builder.n_chain, builder.scratch.data_ptr(),
                          ct.byref(pool), ct.byref(off), ct.byref(ln), ct.byref(boff), ct.byref(blen), ct.byref(bpool),
                          None, None)
    _lib.check(st, "field accel")
    return pool.value, off.value, ln.value, boff.value, blen.value, bpool.value


def bygg_multires_fran_recept(recipe, lo, h_grov, brick_shape, block=8, levels=None, device="cuda",
                              overlappsband=True):
    """Build a MultiresField of an analytic recipe.

    ``levels``: None (all level 0), an int (one level for every active brick), a callable
    ``levels(list_lengths) -> int8 array`` over the active bricks (e.g. levels_by_list_length) or an
    (n_bx, n_by, n_bz) int array.  ``overlappsband`` (the reference's default, bygg_multires
    :254-361): finish with the overlap band, every fine brick's faces next to an active coarser brick
    taking that brick's field (_lagg_overlappsband); False keeps every lattice point the recipe's own
    value."""
    import torch
    lo = np.asarray(lo, dtype=np.float64)
    bx, by, bz = (int(v) for v in brick_shape)
    meta = GridMeta(float(lo[0]), float(lo[1]), float(lo[2]), float(h_grov), bx * block, by * block, bz * block, block)
    fb = FieldBuilder(recipe, meta, device=device)
    fb.classify()
    n_active = int(fb.count.item())
    kind = fb.kind.cpu().numpy().astype(np.int8)
    active = fb.active[:n_active].cpu().numpy().astype(np.int64)
    pool_p, sb_off, sb_len, blk_off, blk_len, blk_pool = _accel(fb)
    # list lengths of the active bricks (for level rules), copied out of the builder's scratch
    lens_host = np.empty(n_active, np.int32)
    if n_active:
        lengths_all = torch.empty(meta.n_blocks, dtype=torch.int32, device=fb.device)
        _copy_device(lengths_all, blk_len, meta.n_blocks * 4)
        lens_host = lengths_all[torch.from_numpy(active).to(fb.device)].cpu().numpy()
    # a block whose culled list overflowed its capacity (length -1) counts as longer than any threshold
    lens_host = np.where(lens_host < 0, np.iinfo(np.int32).max, lens_host)
    if levels is None:
        lv = np.zeros(n_active, np.int8)
    elif isinstance(levels, (int, np.integer)):
        lv = np.full(n_active, int(levels), np.int8)
    elif callable(levels):
        lv = np.asarray(levels(lens_host), dtype=np.int8)
    else:
        lv = np.asarray(levels, dtype=np.int8).ravel()[active]
    if n_active and (lv.min() < 0 or lv.max() > 3):
        raise ValueError("levels must be 0..3")
    sizes = (block * (1 << lv.astype(np.int64)) + 1) ** 3
    offsets = np.zeros(n_active, np.int64)
    if n_active:
        offsets[1:] = np.cumsum(sizes)[:-1]
    total = int(sizes.sum()) if n_active else 0
    dev = fb.device
    pool = torch.empty(max(total, 1), dtype=torch.float32, device=dev)
    primf = torch.empty(fb.n_prims * PRIMF_BYTES, dtype=torch.uint8, device=dev)
    L = fb.lib
    _lib.check(L.fb_query_prepare(fb.prims.data_ptr(), fb.n_prims, primf.data_ptr(), _lib.stream_handle()), "prepare")
    d_bricks = torch.from_numpy(active.astype(np.int32)).to(dev)
    d_levels = torch.from_numpy(lv).to(dev)
    d_offsets = torch.from_numpy(offsets).to(dev)
    bshape = np.array([bx, by, bz], np.int32)
    if n_active:
        st = L.fb_multires_tiles_device(primf.data_ptr(), fb.chain.data_ptr(), fb.n_chain, fb.mode, fb.prims.data_ptr(),
                                        lo.ctypes.data, float(h_grov), block, bshape.ctypes.data, d_bricks.data_ptr(),
                                        d_levels.data_ptr(), d_offsets.data_ptr(), n_active, blk_off, blk_len,
                                        blk_pool, float(meta.guard()), pool.data_ptr(), _lib.stream_handle())
        _lib.check(st, "multires tiles")
    niva = np.full(kind.shape, -1, np.int8)
    niva.ravel()[active] = lv
    tile_off = np.zeros(kind.size, np.int64)
    tile_off[active] = offsets
    F = MultiresField(lo=lo.copy(), h_grov=float(h_grov), block=block, brick_shape=(bx, by, bz),
                      kind=kind.reshape(bx, by, bz), niva=niva.reshape(bx, by, bz),
                      margin_mm=float(meta.margin_mm),
                      stats=dict(n_bricks=int(kind.size), n_active=n_active, samples=total,
                                 levels={int(l): int(np.sum(lv == l)) for l in NIVAER}))
    F._dev = dict(kind=torch.from_numpy(kind).to(dev), level=torch.from_numpy(niva).to(dev),
                  tile_off=torch.from_numpy(tile_off).to(dev), tile_off_host=tile_off, pool=pool, builder=fb)
    if overlappsband:
        F.stats["overlap_faces"] = lagg_overlappsband(F)
    return F


def lagg_overlappsband(F: MultiresField) -> int:
    """Overwrite every fine brick's face layer with the coarser active neighbour's field on that face,
    in place on the device (faltkarna_v1_multires.py:211-251: the same bricks, faces, order and
    float64 sampling, so the lattices equal the reference's bit for bit).  Returns the number of faces
    written."""
    import torch
    d = F._dev
    lv = F.niva.ravel()
    act = np.flatnonzero(F.kind.ravel() == 0)
    fine = act[lv[act] >= 1]
    if not len(fine):
        return 0
    order = np.lexsort((fine, lv[fine]))  # by level, then by id
    bricks = fine[order].astype(np.int32)
    n_of_level = np.array([0] + [int(np.sum(lv[fine] == l)) for l in (1, 2, 3)], np.int32)
    pool = d["pool"]
    dev = pool.device
    orig = torch.empty_like(pool)
    faces = torch.zeros(1, dtype=torch.int32, device=dev)
    d_bricks = torch.from_numpy(bricks).to(dev)
    bshape = np.array(F.brick_shape, np.int32)
    st = d["builder"].lib.fb_multires_band_device(F.lo.ctypes.data, F.h_grov, F.block, bshape.ctypes.data,
                                                  d["kind"].data_ptr(), d["level"].data_ptr(), d["tile_off"].data_ptr(),
                                                  pool.data_ptr(), pool.numel(), orig.data_ptr(), d_bricks.data_ptr(),
                                                  n_of_level.ctypes.data, faces.data_ptr(), _lib.stream_handle())
    _lib.check(st, "multires overlap band")
    return int(faces.item())


def kontinuitetscheck(F: MultiresField, eps_frac=1.0e-3, max_punkter_per_face=None):
    """Largest jump of the delivered field across every brick face where the pitch changes
    (faltkarna_v1_multires.py:462-521): each such face sampled at the finer side's face lattice,
    avstand evaluated a hair (eps_frac of the finer pitch) inside the fine brick and inside the coarse
    neighbour; the bound is half the coarser pitch.  All faces' points go to the device in two
    queries.  Returns the reference's dict."""
    n_bx, n_by, n_bz = F.brick_shape
    kind, niva = F.kind, F.niva
    faces, p_in, p_out = [], [], []
    grans = 0.0
    for lin in np.flatnonzero(kind.ravel() == 0):
        bi, bj, bk = int(lin // (n_by * n_bz)), int((lin // n_bz) % n_by), int(lin % n_bz)
        lvl = int(niva[bi, bj, bk])
        n_l = F.block * (1 << lvl)
        h_f = F.pitch_of(lvl)
        b_origin = F.lo + np.array([bi, bj, bk], dtype=np.float64) * F.L
        for ax in range(3):
            for sida in (-1, +1):
                nb = [bi, bj, bk]
                nb[ax] += sida
                if not (0 <= nb[0] < n_bx and 0 <= nb[1] < n_by and 0 <= nb[2] < n_bz):
                    continue
                if kind[nb[0], nb[1], nb[2]] != 0:
                    continue
                lvl_n = int(niva[nb[0], nb[1], nb[2]])
                if lvl_n >= lvl:
                    continue
                idx = [np.arange(n_l + 1, dtype=np.float64)] * 3
                idx[ax] = np.array([0.0 if sida < 0 else float(n_l)])
                gi, gj, gk = np.meshgrid(*idx, indexing="ij")
                pts = np.stack([gi.ravel(), gj.ravel(), gk.ravel()], axis=1) * h_f + b_origin
                if max_punkter_per_face is not None and len(pts) > max_punkter_per_face:
                    pts = pts[::int(np.ceil(len(pts) / max_punkter_per_face))]
                e = np.zeros(3)
                e[ax] = eps_frac * h_f
                p_in.append(pts - sida * e)
                p_out.append(pts + sida * e)
                faces.append((len(pts), dict(brick=[bi, bj, bk], axel=ax, sida=sida, niva=lvl, niva_granne=lvl_n)))
                grans = max(grans, 0.5 * F.pitch_of(lvl_n))
    if not faces:
        return dict(n_pitchbyten_faces=0, n_provpunkter=0, max_hopp_mm=0.0, medel_hopp_mm=0.0, grans_mm=0.0,
                    varsta=None, GRON=True)
    hopp = np.abs(avstand(F, np.concatenate(p_in)) - avstand(F, np.concatenate(p_out)))
    bounds = np.cumsum([0] + [n for n, _ in faces])
    per_face = np.array([hopp[a:b].max() for a, b in zip(bounds[:-1], bounds[1:])])
    max_hopp, varsta = 0.0, None
    for (n, info), m in zip(faces, per_face):  # first face with a strictly larger jump, as the reference
        if float(m) > max_hopp:
            max_hopp, varsta = float(m), info
    return dict(n_pitchbyten_faces=len(faces), n_provpunkter=int(len(hopp)), max_hopp_mm=max_hopp,
                medel_hopp_mm=float(hopp.sum()) / len(hopp), grans_mm=grans, varsta=varsta,
                GRON=bool(max_hopp <= grans))


def _copy_device(dst, src_ptr, nbytes):
    """Device-to-device copy from a raw device address (an array inside a builder's scratch)."""
    _lib.check(_lib.lib().fb_copy_device(dst.data_ptr(), src_ptr, int(nbytes), _lib.stream_handle()), "device copy")


def _query(F: MultiresField, punkter, want_grad):
    import torch
    pts = np.atleast_2d(np.asarray(punkter, dtype=np.float64))
    if pts.ndim != 2 or pts.shape[1] != 3:
        raise ValueError("points must be (N, 3)")
    d = F._dev
    dev = d["pool"].device
    p = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    n = len(pts)
    val = torch.empty(n, dtype=torch.float64, device=dev) if not want_grad else None
    grad = torch.empty((n, 3), dtype=torch.float64, device=dev) if want_grad else None
    bshape = np.array(F.brick_shape, np.int32)
    st = d["builder"].lib.fb_multires_query_device(F.lo.ctypes.data, F.h_grov, F.block, bshape.ctypes.data,
                                                   float(F.margin_mm), d["kind"].data_ptr(), d["level"].data_ptr(),
                                                   d["tile_off"].data_ptr(), d["pool"].data_ptr(), p.data_ptr(), n,
                                                   val.data_ptr() if val is not None else None,
                                                   grad.data_ptr() if grad is not None else None,
                                                   _lib.stream_handle())
    _lib.check(st, "multires query")
    return (grad if want_grad else val).cpu().numpy()


def avstand(F: MultiresField, punkter):
    """Signed distance at world points, each at its own brick's pitch; bricks without a lattice
    answer +-margin (faltkarna_v1_multires.py:405-434).  float64 (N,)."""
    return _query(F, punkter, False)


def gradient(F: MultiresField, punkter):
    """Central difference at each point's brick pitch, probes clamped into the brick
    (faltkarna_v1_multires.py:437-459).  float64 (N, 3)."""
    return _query(F, punkter, True)
