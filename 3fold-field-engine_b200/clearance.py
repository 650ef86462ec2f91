"""Consumers of the EDT on the GPU: the clearance field, the clearance-valid mask and the free space
as a resistor network, with the reference's signatures.

* ``edt_mm(occ, pitch_mm)`` -- ``distance_transform_edt(~occ) * pitch_mm``, the clearance of every
  cell to the nearest occupied one in millimetres (src/field_engine/opt/laplaceflode_v1.py:313-314,
  src/field_engine/opt/f33_1_topologi_v1.py:205-206), from the exact integer EDT: float64 root of the
  squared distance, times the pitch -- the same bits as scipy's.
* ``giltig_frirum(occ, edt_mm, min_r_mm, margin_mm)`` -- ``~occ & (edt_mm >= min_r_mm + margin_mm)``
  (src/field_engine/opt/f33_1_topologi_v1.py:207-218), the cells a route of radius ``min_r_mm`` may
  use.
* ``bygg_gitterlaplacian(occ, edt_mm, pitch_mm, p_kond=1.5)`` -- src/field_engine/opt/laplaceflode_v1.py:69-97:
  node count, node map (-1 on occupied cells), edge endpoints ``u``/``v`` (axis 0, 1, 2; lower cell
  ascending), conductances ``max(0.5 (E_u + E_v) / pitch, 0.1) ** p_kond`` and the Laplacian in CSR
  with sorted columns and the diagonal summed in scipy's order.
* ``fritt_natverk(occ, pitch_mm, p_kond=1.5)`` -- the first two steps of ``rutt_genom_flode``
  (laplaceflode_v1.py:310-316) in one call: clearance, then the network.

Arguments given as NumPy arrays return NumPy arrays (and a ``scipy.sparse.csr_matrix`` for the
Laplacian, as the reference does); CUDA tensors return CUDA tensors (the Laplacian as a
``torch.sparse_csr_tensor``).  Every computation runs on the GPU.  Host results are NumPy arrays
over pooled page-locked blocks, read back with one synchronisation; a block returns to the pool when
its array is dropped.

Bit-exact against the reference: the node map, ``u``, ``v``, the CSR structure, the clearance and the
mask.  The conductances take ``pow`` from CUDA's math library where NumPy takes the host's libm, so
``kond`` and the Laplacian's values agree to within 2 ulp (float64).

Deliberate differences: grids are at most 3-D (1-D and 2-D grids run as 3-D ones with leading axes
of 1, which gives the same arrays), at most (2^31 - 1) / 7 cells; ``edt_mm`` must be float64; the
clearance needs at least one occupied cell (scipy's transform of a grid without one is not a distance)
and at most 512 cells per axis (the EDT's bound).
"""
from __future__ import annotations

from numbers import Real

import numpy as np

from . import _lib

KONDUKTANS_GOLV = 0.1  # laplaceflode_v1.py: the wall conductance floor (applied in the kernel)
MAX_CELLS = (2 ** 31 - 1) // 7


def _torch():
    import torch
    return torch


_POOL = None


def _host_arrays(tensors):
    """NumPy arrays of device tensors over pooled page-locked blocks: every copy is enqueued on the
    current stream, then one synchronisation.  A block returns to the pool when its array (or the
    last object sharing its memory) is dropped, so repeated calls reuse page-locked memory instead
    of faulting in fresh pageable pages at every call."""
    global _POOL
    torch = _torch()
    if _POOL is None:
        from .serve import PinnedPool
        _POOL = PinnedPool()
    staged = []
    for t in tensors:
        nbytes = t.numel() * t.element_size()
        if nbytes == 0:
            staged.append((torch.empty(tuple(t.shape), dtype=t.dtype), None))
            continue
        blk, handle = _POOL.take(nbytes)
        view = blk.view(t.dtype).view(tuple(t.shape))
        view.copy_(t, non_blocking=True)
        staged.append((view, handle))
    torch.cuda.current_stream().synchronize()
    out = []
    for view, handle in staged:
        a = view.numpy()
        if handle is not None:
            _POOL.bind(a, handle)
        out.append(a)
    return out


def _as_device_occ(occ):
    """(uint8 CUDA tensor of shape 3-D, original shape, on_host)."""
    torch = _torch()
    if isinstance(occ, np.ndarray):
        if occ.dtype != np.bool_ or occ.ndim < 1 or occ.ndim > 3:
            raise ValueError('Expected a boolean occupancy array of 1 to 3 dimensions')
        shape = occ.shape
        if min(shape) < 1 or occ.size > MAX_CELLS:
            raise ValueError('Occupancy grid outside the bounded contract')
        t = torch.from_numpy(np.ascontiguousarray(occ).view(np.uint8)).cuda()
        host = True
    elif isinstance(occ, torch.Tensor):
        if occ.dtype not in (torch.bool, torch.uint8) or occ.dim() < 1 or occ.dim() > 3 or not occ.is_cuda:
            raise ValueError('Expected a bool/uint8 CUDA occupancy tensor of 1 to 3 dimensions')
        shape = tuple(occ.shape)
        t = occ.contiguous()
        if t.dtype == torch.bool:
            t = t.view(torch.uint8)
        host = False
    else:
        raise ValueError('Expected a boolean occupancy array')
    if min(shape) < 1 or int(np.prod(shape)) > MAX_CELLS:
        raise ValueError('Occupancy grid outside the bounded contract')
    shape3 = (1,) * (3 - len(shape)) + tuple(shape)
    return t.reshape(shape3), tuple(shape), host


def _as_device_f64(a, shape, what):
    torch = _torch()
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or a.shape != shape:
            raise ValueError(f'Expected a float64 {what} of the grid\'s shape')
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()
    if isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or tuple(a.shape) != shape or not a.is_cuda:
            raise ValueError(f'Expected a float64 CUDA {what} of the grid\'s shape')
        return a.contiguous()
    raise ValueError(f'Expected a float64 {what}')


def _real(x, what):
    if isinstance(x, (bool, np.bool_)) or not isinstance(x, Real):
        raise ValueError(f'Expected a real {what}')
    return float(x)


def edt_mm(occ, pitch_mm):
    """Clearance of every cell to the nearest occupied cell, in millimetres (float64)."""
    from . import edt as E
    torch = _torch()
    pitch = _real(pitch_mm, 'pitch')
    occ3, shape, host = _as_device_occ(occ)
    if max(occ3.shape) > E.MAX_AXIS:
        raise ValueError('Expected bounded larger 3D shape')
    if not bool(occ3.any()):
        raise ValueError('The grid holds no occupied cell')
    sq = E.squared_distance_device(occ3, sites_nonzero=True)
    out = torch.empty(occ3.shape, dtype=torch.float64, device=occ3.device)
    st = _lib.lib().fb_edt_mm_device(sq.data_ptr(), sq.numel(), pitch, out.data_ptr(), _lib.stream_handle())
    _lib.check(st, 'edt_mm')
    out = out.reshape(shape)
    return _host_arrays([out])[0] if host else out


def giltig_frirum(occ, edt_mm, min_r_mm, margin_mm):
    """Cells free of obstacles whose clearance is at least ``min_r_mm + margin_mm`` (bool)."""
    torch = _torch()
    occ3, shape, host = _as_device_occ(occ)
    e = _as_device_f64(edt_mm, shape, 'clearance')
    threshold = _real(min_r_mm, 'radius') + _real(margin_mm, 'margin')
    valid = torch.empty(occ3.shape, dtype=torch.uint8, device=occ3.device)
    st = _lib.lib().fb_clearance_mask_device(occ3.data_ptr(), e.data_ptr(), occ3.numel(), threshold,
                                             valid.data_ptr(), _lib.stream_handle())
    _lib.check(st, 'giltig_frirum')
    valid = valid.view(torch.bool).reshape(shape)
    return _host_arrays([valid])[0] if host else valid


def bygg_gitterlaplacian(occ, edt_mm, pitch_mm, p_kond=1.5):
    """The free space as a resistor network: (n, nodkarta, u, v, kond, L)."""
    torch = _torch()
    occ3, shape, host = _as_device_occ(occ)
    e = _as_device_f64(edt_mm, shape, 'clearance')
    pitch = _real(pitch_mm, 'pitch')
    p = _real(p_kond, 'conductance exponent')
    L = _lib.lib()
    dev = occ3.device
    nx, ny, nz = occ3.shape
    nbytes = L.fb_lattice_scratch_bytes(nx, ny, nz)
    if nbytes < 0:
        raise ValueError('Occupancy grid outside the bounded contract')
    scratch = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
    totals = torch.empty(3, dtype=torch.int32, device=dev)
    stream = _lib.stream_handle()
    _lib.check(L.fb_lattice_count_device(occ3.data_ptr(), nx, ny, nz, totals.data_ptr(), scratch.data_ptr(),
                                         scratch.numel(), stream), 'bygg_gitterlaplacian')
    n, n_edges, nnz = (int(x) for x in totals.cpu().tolist())
    node_map = torch.empty(occ3.shape, dtype=torch.int32, device=dev)
    u = torch.empty(n_edges, dtype=torch.int32, device=dev)
    v = torch.empty(n_edges, dtype=torch.int32, device=dev)
    kond = torch.empty(n_edges, dtype=torch.float64, device=dev)
    indptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
    indices = torch.empty(nnz, dtype=torch.int32, device=dev)
    data = torch.empty(nnz, dtype=torch.float64, device=dev)
    _lib.check(L.fb_lattice_emit_device(occ3.data_ptr(), e.data_ptr(), nx, ny, nz, pitch, p,
                                        node_map.data_ptr(), u.data_ptr(), v.data_ptr(), kond.data_ptr(), n_edges,
                                        indptr.data_ptr(), n + 1, indices.data_ptr(), data.data_ptr(), nnz,
                                        scratch.data_ptr(), scratch.numel(), stream), 'bygg_gitterlaplacian')
    node_map = node_map.reshape(shape)
    if host:
        from scipy import sparse
        node_h, u_h, v_h, kond_h, indptr_h, indices_h, data_h = _host_arrays(
            [node_map, u, v, kond, indptr, indices, data])
        Lh = sparse.csr_matrix((data_h, indices_h, indptr_h), shape=(n, n))
        return n, node_h, u_h, v_h, kond_h, Lh
    Ld = torch.sparse_csr_tensor(indptr, indices, data, size=(n, n), check_invariants=False)
    return n, node_map, u, v, kond, Ld


def fritt_natverk(occ, pitch_mm, p_kond=1.5):
    """Clearance and resistor network of the free space in one call: (edt_mm, n, nodkarta, u, v, kond, L)."""
    e = edt_mm(occ, pitch_mm)
    return (e,) + tuple(bygg_gitterlaplacian(occ, e, pitch_mm, p_kond))
