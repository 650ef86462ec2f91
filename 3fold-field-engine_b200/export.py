"""Export step: isosurface meshes, volumes and the on-disk field format.

The reference exports a field by reconstructing it densely (``rekonstruera_tat(_gpu)``,
src/field_engine/faltkarna_v1.py:302-350) and running scikit-image's marching cubes on the result;
its volume meters (faltvolym_v1.py:76-104) read that mesh or the occupancy.  Here:

* ``marching_cubes(field, level=0.0, *, keys=False, to_host=True)`` -> ``Mesh`` -- the isosurface of
  a resident ``DeviceField`` (or a host ``SparseField``) straight from its leaf tiles on the GPU:
  the mesh that marching cubes gives on the dense reconstruction, without building it.  Vertices
  are float32 world coordinates, one per grid edge that crosses ``level`` (linear interpolation);
  triangles have outward normals; ``volume`` is the enclosed volume, float64, summed in a fixed
  order (bit-reproducible).
* ``marching_cubes_dense(volume, level=0.0, *, pitch=1.0, origin=(0, 0, 0))`` -> ``Mesh`` -- the same
  on a dense array (every block taken as a leaf).
* ``marching_cubes_volym(falt, pitch, origin=(0, 0, 0))`` -> ``(volume, dropped)`` and
  ``voxel_riemann_volym(falt, pitch)`` -- faltvolym_v1.py:76-104: the volume of the largest
  connected component of the isosurface (and how many components were dropped), 0.0 when the field
  has no zero crossing; the occupancy Riemann sum.
* ``save_field(path, field)`` / ``load_field(path)`` -- the field as an ``.npz`` archive with the
  ``SparseField`` arrays (kind, active_ids, tiles, corner_min_abs) and a JSON ``meta`` record;
  ``field_record(field)`` is that record (grid, margin, statistics) as a JSON-ready dict.

scikit-image is not part of this environment, so the mesh rules are written out in the CUDA source
(csrc/export.cu): the vertex set and positions are those of any edge-interpolating marching cubes;
the triangulation resolves face ambiguities by the asymptotic decider and keeps two loops where
scikit-image's Lewiner tables may join them through a cube's interior.
"""
from __future__ import annotations

import json
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from .grid import BIG, GridMeta, SparseField, stats_of

FORMAT = "field_b200.sparse_field/1"


@dataclass
class Mesh:
    verts: object             # (V, 3) float32 world coordinates (numpy, or a CUDA tensor with to_host=False)
    faces: object             # (T, 3) int32 vertex ids, outward normals
    volume: float             # enclosed volume sum(v0 . (v1 x v2)) / 6, float64
    keys: Optional[object] = None  # (V,) int64 edge of each vertex: (linear index of its lower end) * 3 + axis


def _device_arrays(field, device):
    """(kind, active, n_active, tiles, meta) on the device for a DeviceField or a SparseField."""
    import torch
    if hasattr(field, "tiles") and hasattr(field.tiles, "data_ptr"):
        return field.kind, field.active, int(field.n_active), field.tiles, field.meta
    meta = field.meta
    dev = torch.device(device)
    n = len(field.active_ids)
    kind = torch.from_numpy(np.ascontiguousarray(field.kind, np.int32)).to(dev)
    active = torch.from_numpy(np.ascontiguousarray(field.active_ids, np.int32)).to(dev)
    tiles = torch.from_numpy(np.ascontiguousarray(field.tiles, np.float32).reshape(n, -1)).to(dev)
    return kind, active, n, tiles, meta


def _mesh(kind, active, n, tiles, nx, ny, nz, block, origin, pitch, level, keys, to_host):
    import torch
    lib = _lib.lib()
    dev = kind.device
    if not (1 <= block <= 32):
        raise ValueError(f"marching cubes: block {block} outside 1..32")
    W = int(lib.fb_mc_words(block))
    nb = kind.numel()
    st = _lib.stream_handle()
    i32 = dict(dtype=torch.int32, device=dev)
    slot = torch.empty(nb, **i32)
    bits = torch.empty(max(n, 1) * W, **i32)
    wpre = torch.empty(max(n, 1) * W, **i32)
    vcount = torch.empty(n + 1, **i32)
    tcount = torch.empty(n + 1, **i32)
    totals = torch.empty(2, dtype=torch.int64, device=dev)
    words = int(lib.fb_mc_scan_words(n))
    scan = torch.empty(words, **i32)
    ox, oy, oz = (float(v) for v in origin)
    lv = float(level)
    args = (kind.data_ptr(), active.data_ptr() if n else None, n, tiles.data_ptr() if n else None, nx, ny, nz, block,
            ox, oy, oz, float(pitch), lv, float(BIG))
    _lib.check(lib.fb_mc_count_device(*args, slot.data_ptr(), bits.data_ptr(), wpre.data_ptr(), vcount.data_ptr(),
                                      tcount.data_ptr(), totals.data_ptr(), scan.data_ptr(), words, st),
               "marching cubes (count)")
    nv, nt = (int(v) for v in totals.cpu())
    if nv >= 2 ** 31 or nt >= 2 ** 31:
        raise ValueError(f"marching cubes: {nv} vertices / {nt} triangles exceed int32 ids")
    verts = torch.empty((nv, 3), dtype=torch.float32, device=dev)
    faces = torch.empty((nt, 3), **i32)
    vkey = torch.empty(nv, dtype=torch.int64, device=dev) if keys else None
    vol_part = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    volume = torch.zeros(1, dtype=torch.float64, device=dev)
    err = torch.empty(1, **i32)
    _lib.check(lib.fb_mc_emit_device(*args, slot.data_ptr(), bits.data_ptr(), wpre.data_ptr(), vcount.data_ptr(),
                                     tcount.data_ptr(), verts.data_ptr() if nv else None,
                                     vkey.data_ptr() if (keys and nv) else None, faces.data_ptr() if nt else None,
                                     vol_part.data_ptr(), volume.data_ptr(), err.data_ptr(), st),
               "marching cubes (emit)")
    vol, e = float(volume.cpu()[0]), int(err.cpu()[0])
    if e:
        raise RuntimeError(f"marching cubes: {e} triangle corners without a vertex")
    if to_host:
        return Mesh(verts.cpu().numpy(), faces.cpu().numpy(), vol, vkey.cpu().numpy() if keys else None)
    return Mesh(verts, faces, vol, vkey)


def marching_cubes(field, level=0.0, *, keys=False, to_host=True, device="cuda:0") -> Mesh:
    """Isosurface of a sparse field (DeviceField or SparseField) from its tiles, on the GPU: the
    mesh of marching cubes on rekonstruera_tat(field) (faltkarna_v1.py:302-350)."""
    kind, active, n, tiles, meta = _device_arrays(field, device)
    return _mesh(kind, active, n, tiles, meta.nx, meta.ny, meta.nz, meta.block, (meta.x0, meta.y0, meta.z0),
                 meta.pitch, level, keys, to_host)


def marching_cubes_dense(volume, level=0.0, *, pitch=1.0, origin=(0.0, 0.0, 0.0), keys=False, to_host=True,
                         device="cuda:0", block=8) -> Mesh:
    """Isosurface of a dense (nx, ny, nz) array: every block becomes a leaf (the dense classifier
    with an infinite margin), then the sparse path."""
    import torch
    lib = _lib.lib()
    d = volume if hasattr(volume, "data_ptr") else torch.from_numpy(np.ascontiguousarray(volume, np.float32))
    d = d.to(device=torch.device(device), dtype=torch.float32).contiguous()
    if d.dim() != 3:
        raise ValueError("dense field must be 3-D")
    nx, ny, nz = (int(v) for v in d.shape)
    meta = GridMeta(float(origin[0]), float(origin[1]), float(origin[2]), float(pitch), nx, ny, nz, block)
    dev = d.device
    kind = torch.empty(meta.n_blocks, dtype=torch.int32, device=dev)
    active = torch.empty(meta.n_blocks, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    tiles = torch.empty((meta.n_blocks, block ** 3), dtype=torch.float32, device=dev)
    scratch = torch.empty(int(lib.fb_dense_scratch_bytes(nx, ny, nz, block)), dtype=torch.uint8, device=dev)
    _lib.check(lib.fb_dense_classify_device(d.data_ptr(), nx, ny, nz, block, float("inf"), kind.data_ptr(), None,
                                            active.data_ptr(), count.data_ptr(), tiles.data_ptr(), meta.n_blocks,
                                            scratch.data_ptr(), scratch.numel(), _lib.stream_handle()),
               "dense leaves")
    return _mesh(kind, active, meta.n_blocks, tiles, nx, ny, nz, block, origin, pitch, level, keys, to_host)


def components(mesh: Mesh, device="cuda:0"):
    """(labels, volumes): per vertex the smallest vertex id of its connected component, and a dict
    root -> signed component volume (GPU union-find; faltvolym_v1.py:95-101)."""
    import torch
    lib = _lib.lib()
    dev = torch.device(device)
    verts = mesh.verts if hasattr(mesh.verts, "data_ptr") else torch.from_numpy(np.ascontiguousarray(mesh.verts))
    faces = mesh.faces if hasattr(mesh.faces, "data_ptr") else torch.from_numpy(np.ascontiguousarray(mesh.faces))
    verts = verts.to(dev, torch.float32).contiguous()
    faces = faces.to(dev, torch.int32).contiguous()
    nv, nf = verts.shape[0], faces.shape[0]
    if nf and (int(faces.min()) < 0 or int(faces.max()) >= nv):
        raise ValueError("face vertex id outside [0, n_verts)")
    parent = torch.empty(max(nv, 1), dtype=torch.int32, device=dev)
    label = torch.empty(max(nv, 1), dtype=torch.int32, device=dev)
    vol = torch.empty(max(nv, 1), dtype=torch.float64, device=dev)
    count = torch.empty(1, dtype=torch.int32, device=dev)
    err = torch.empty(1, dtype=torch.int32, device=dev)
    _lib.check(lib.fb_mesh_components_device(faces.data_ptr() if nf else None, nf, verts.data_ptr() if nv else None,
                                             nv, parent.data_ptr(), label.data_ptr(), vol.data_ptr(),
                                             count.data_ptr(), err.data_ptr(), _lib.stream_handle()),
               "mesh components")
    if int(err.cpu()[0]):
        raise RuntimeError("mesh components: a union gave up")
    lab = label[:nv].cpu().numpy()
    roots = np.unique(lab[faces[:, 0].cpu().numpy()]) if nf else np.zeros(0, np.int32)
    v = vol.cpu().numpy()
    return lab, {int(r): float(v[r]) for r in roots}


def voxel_riemann_volym(falt, pitch) -> float:
    """Riemann sum over the occupancy of a dense field: cells with a negative sample, times pitch^3
    (faltvolym_v1.py:78-80)."""
    f = falt.cpu().numpy() if hasattr(falt, "cpu") else np.asarray(falt)
    return float(np.count_nonzero(f < 0.0) * float(pitch) ** 3)


def marching_cubes_volym(falt, pitch, origin=(0.0, 0.0, 0.0)):
    """(volume, dropped) of faltvolym_v1.py:83-104: 0.0 and 0 without a zero crossing; otherwise the
    |volume| of the largest connected component of the zero isosurface and the number of components
    dropped.  ``falt`` is a dense array, a DeviceField or a SparseField."""
    if hasattr(falt, "meta"):
        mesh = marching_cubes(falt, 0.0, to_host=False)
    else:
        import torch
        t = falt if hasattr(falt, "data_ptr") else torch.from_numpy(np.ascontiguousarray(falt, np.float32))
        t = t.cuda().float()
        if not (float(t.min()) < 0.0 < float(t.max())):
            return 0.0, 0
        mesh = marching_cubes_dense(t, 0.0, pitch=pitch, origin=origin, to_host=False)
    nt = int(mesh.faces.shape[0])
    if nt == 0:
        return 0.0, 0
    _, vols = components(mesh)
    if len(vols) > 1:
        root = max(vols, key=lambda r: abs(vols[r]))
        return float(abs(vols[root])), len(vols) - 1
    return float(abs(mesh.volume)), 0


# ------------------------------------------------------------------------------ on-disk format

def field_record(field) -> dict:
    """JSON-ready description: format tag, grid (origin, pitch, shape, block), margin, statistics."""
    meta = field.meta
    n = int(field.n_active) if hasattr(field, "n_active") else len(field.active_ids)
    if hasattr(field, "stats") and field.stats:
        stats = dict(field.stats)
    else:
        kind = field.kind.cpu().numpy() if hasattr(field.kind, "cpu") else np.asarray(field.kind)
        stats = stats_of(meta, kind, n)
    return dict(format=FORMAT, x0=float(meta.x0), y0=float(meta.y0), z0=float(meta.z0), pitch=float(meta.pitch),
                nx=int(meta.nx), ny=int(meta.ny), nz=int(meta.nz), block=int(meta.block),
                margin_mm=float(meta.margin_mm), background=float(BIG),
                stats={k: (float(v) if isinstance(v, float) else int(v)) for k, v in stats.items()})


def save_field(path, field) -> None:
    """Write a field (DeviceField or SparseField) as .npz: kind, active_ids, tiles, corner_min_abs
    and the JSON record under ``meta``."""
    sf = field.to_host() if hasattr(field, "to_host") else field
    rec = field_record(sf)
    np.savez(path, kind=np.asarray(sf.kind, np.int32), active_ids=np.asarray(sf.active_ids, np.int32),
             tiles=np.asarray(sf.tiles, np.float32), corner_min_abs=np.asarray(sf.corner_min_abs, np.float32),
             meta=np.array(json.dumps(rec, sort_keys=True)))


def load_field(path) -> SparseField:
    """Read a field written by save_field; the arrays are checked against the record's grid."""
    with np.load(path, allow_pickle=False) as z:
        rec = json.loads(str(z["meta"]))
        if rec.get("format") != FORMAT:
            raise ValueError(f"not a {FORMAT} archive: {rec.get('format')!r}")
        meta = GridMeta(rec["x0"], rec["y0"], rec["z0"], rec["pitch"], rec["nx"], rec["ny"], rec["nz"], rec["block"])
        kind, active, tiles, cma = (np.array(z[k]) for k in ("kind", "active_ids", "tiles", "corner_min_abs"))
    b = meta.block
    if kind.shape != (meta.n_blocks,) or cma.shape != (meta.n_blocks,):
        raise ValueError("kind / corner_min_abs do not match the grid")
    if tiles.shape != (len(active), b, b, b):
        raise ValueError("tiles do not match active_ids and the block size")
    if len(active) and (np.any(np.diff(active) <= 0) or active[0] < 0 or active[-1] >= meta.n_blocks
                        or np.any(kind[active] != 0)):
        raise ValueError("active_ids must be ascending block ids of kind 0")
    if np.count_nonzero(kind == 0) != len(active) or not np.isin(kind, (-1, 0, 1)).all():
        raise ValueError("kind must be -1 / 0 / +1 with every 0 block listed in active_ids")
    return SparseField(meta=meta, kind=kind, active_ids=active, tiles=tiles, corner_min_abs=cma,
                       stats=rec.get("stats", {}))
