"""Mesh -> signed distance field stage on the GPU.

Drop-in surfaces:

* ``meshsdf_field_cpu`` in libfield_b200.so -- the C entry point of
  src/field_engine/mesh_sdf_native_v1/field.cpp:19 with the same arguments and status codes (the
  reference's loader, mesh_sdf_native_v1.lib(library=...), binds it unchanged); it runs on the GPU.
* ``field_stage(V, T, pitch, lo, ...)`` -- mesh_sdf_native_v1.py:74-116: the grid window around
  the mesh, the jittered ray-winding solid, the paired exact EDT, the half-pitch corrected signed
  distance and the surface layer; returns (gmin, shape, surface, solid, sd, diag).

The solid mask, the surface layer and the statistics are the reference's bit for bit; sd is
float32(sqrt(d_out^2) pitch) - float32(sqrt(d_in^2) pitch) from the exact squared distances, equal to
the reference's feature-offset form except where a value lies within float64 rounding of a float32
rounding boundary (one float32 ulp then).  Windows up to 512 voxels per axis take the banded pair EDT;
longer ones (any grid below 2^31 cells, as the reference) take separable long-axis passes.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib

# The reference's sampling constants (faltkarna_v1_mesh_to_sdf.py:122-123,150): the xy jitter of
# the rays as a fraction of a pitch along a golden-ratio direction, and the default half-pitch
# surface correction.
JITTER_FRAC = 1.0e-4
GOLDEN = (0.3819660112501051, 0.6180339887498949, 0.2360679774997897)
SURFACE_CORRECTION = True

_P, _I64, _D, _I = ct.c_void_p, ct.c_int64, ct.c_double, ct.c_int
SIGNATURE = (_I, [_P, _I64, _P, _I64, _D, _D, _D, _D, _D, _D, _I64, _I64, _I64, _I, _I, _P, _P, _P, _P, _P])


def _entry(library=None):
    L = _lib.lib(library)
    fn = L.meshsdf_field_cpu
    fn.restype, fn.argtypes = SIGNATURE
    return fn


def window(V, pitch, lo, global_shape=None, margin_vox_pad=2):
    """(gmin, shape): the grid window around the vertices in global grid indices, margin_vox_pad
    voxels beyond them, clamped to [0, global_shape) when given (faltkarna_v1_mesh_to_sdf.py:153-166)."""
    v = np.asarray(V, dtype=np.float64)
    lo = np.asarray(lo, dtype=np.float64)
    gmin = np.floor((v.min(0) - lo) / pitch).astype(np.int64) - margin_vox_pad
    gmax = np.ceil((v.max(0) - lo) / pitch).astype(np.int64) + margin_vox_pad + 1
    if global_shape is not None:
        gmin = np.maximum(gmin, 0)
        gmax = np.minimum(gmax, np.array(global_shape, dtype=np.int64))
    gmax = np.maximum(gmax, gmin)
    return gmin, tuple(int(x) for x in (gmax - gmin))


def field_grid(V, T, origin, pitch, shape, *, jitter=None, surface_correction=True, library=None):
    """(solid bool, sd float32, surface bool, stats int64[4], stage seconds[5]) on the grid
    origin + index * pitch of `shape`; jitter (jx, jy) defaults to the reference's."""
    Vf = np.ascontiguousarray(np.asarray(V, dtype=np.float64))
    Ti = np.ascontiguousarray(np.asarray(T, dtype=np.int64))
    if Vf.ndim != 2 or Vf.shape[1] != 3 or Ti.ndim != 2 or Ti.shape[1] != 3:
        raise ValueError(f"vertices and faces must be (n, 3) arrays, got {Vf.shape} and {Ti.shape}")
    if jitter is None:
        jitter = (pitch * JITTER_FRAC * GOLDEN[0], pitch * JITTER_FRAC * GOLDEN[1])
    nx, ny, nz = (int(v) for v in shape)
    solid = np.empty((nx, ny, nz), np.uint8)
    sd = np.empty((nx, ny, nz), np.float32)
    yta = np.empty((nx, ny, nz), np.uint8)
    stats = np.zeros(4, np.int64)
    ts = np.zeros(5, np.float64)
    rc = _entry(library)(Vf.ctypes.data, Vf.shape[0], Ti.ctypes.data, Ti.shape[0], float(origin[0]), float(origin[1]),
                         float(origin[2]), float(pitch), float(jitter[0]), float(jitter[1]), nx, ny, nz,
                         int(bool(surface_correction)), 0, solid.ctypes.data, sd.ctypes.data, yta.ctypes.data,
                         stats.ctypes.data, ts.ctypes.data)
    if rc == 1:
        raise ValueError("mesh field: input outside the contract (status 1)")
    if rc == 2:
        raise ValueError("mesh field: face index outside [0, nv) (status 2)")
    if rc == 3:
        raise ValueError("mesh field: more than 2^31 - 2 ray hits (status 3)")
    if rc:
        raise RuntimeError(f"mesh field: native failure (status {rc})")
    return solid.view(bool), sd, yta.view(bool), stats, ts


def field_stage(V, T, pitch, lo, global_shape=None, margin_vox_pad=2, ytkorrektion=None, nthreads=None,
                library=None):
    """(gmin, shape, surface, solid, sd, diag) of mesh_sdf_native_v1.field_stage (mesh_sdf_native_v1.py:74-116).
    When the solid is empty or fills the window (no surface), sd is the kernel's: -1 for the
    distance to the missing class, 0 for the other (the reference's wrapper recomputes that case on
    the CPU; here nothing runs on the CPU)."""
    v = np.asarray(V, dtype=np.float64)
    if not (np.isfinite(v).all() and np.isfinite(float(pitch)) and np.isfinite(np.asarray(lo, np.float64)).all()):
        raise ValueError("non-finite vertex, pitch or origin: no field and no certified side")
    corr = SURFACE_CORRECTION if ytkorrektion is None else bool(ytkorrektion)
    gmin, shape = window(v, pitch, lo, global_shape, margin_vox_pad)
    origin = np.asarray(lo, dtype=np.float64) + gmin.astype(np.float64) * pitch
    solid, sd, yta, stats, ts = field_grid(v, T, origin, pitch, shape, surface_correction=corr, library=library)
    n = int(np.prod(shape))
    diag = dict(metod="raypar", regel="vindning", backend="cuda", jitter_frac=JITTER_FRAC, n_par=int(stats[0]),
                n_traffar=int(stats[1]), n_vindning_vs_paritet_diff=int(stats[2]),
                andel_vindning_vs_paritet=int(stats[2]) / float(n), ytkorrektion=corr,
                one_class=bool(stats[3] == 0 or stats[3] == n), stage_seconds=[float(t) for t in ts])
    return gmin, shape, yta, solid, sd, diag
