"""CPU oracle for the block-sparse SDF field path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``oracle/liboracle.so`` (a C restatement of the reference algorithms, each
function citing the reference file:line it follows) plus NumPy restatements of the reference's
Python-level semantics.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker: the product library never calls it.

``ref_library(name)`` loads the reference's own CPU libraries compiled from its sources into
``oracle/_ref/`` (see oracle/Makefile); they pin the restatements where the reference is C++.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None

NODE = np.dtype([("lo", "<i4", (3,)), ("shape", "<i4", (3,)), ("stored_shape", "<i4", (3,)),
                 ("children", "<i4", (2,)), ("offset", "<i8")])
CSG_INSN = np.dtype([("op", "<i4"), ("left", "<i4"), ("right", "<i4"), ("pad", "<i4"), ("offset", "<f8")])
PRIM = np.dtype([("type", "<i4"), ("flags", "<i4"), ("p", "<f8", (12,)), ("A", "<f8", (12,)),
                 ("s", "<f8"), ("off", "<f8")])
INSN = np.dtype([("op", "<i4"), ("arg", "<i4"), ("k", "<f8")])


def lib():
    """The compiled oracle (built on demand with make when missing)."""
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            import subprocess
            subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)
        L = ct.CDLL(str(path))
        P, I, I64, D, F = ct.c_void_p, ct.c_int, ct.c_int64, ct.c_double, ct.c_float
        sig = {
            "or_edt_squared": [P, I, I, I, P],
            "or_edt_squared_brute": [P, I, I, I, P],
            "or_edt_signed": [P, I, I, I, D, P, P],
            "or_classify_dense": [P, I64, I64, I64, I64, F, P, P],
            "or_tiles_dense": [P, I64, I64, I64, I64, P, I64, P],
            "or_csg_execute": [P, ct.c_int32, P, P, ct.c_int32, P],
            "or_eval_points": [P, ct.c_int32, P, ct.c_int32, P, I64, P],
            "or_classify_program": [P, ct.c_int32, P, ct.c_int32, D, D, D, D, I, I, I, I, F, P, P],
            "or_tiles_program": [P, ct.c_int32, P, ct.c_int32, D, D, D, D, I, I, I, I, P, I64, P],
            "or_classify_blocks": [P, ct.c_int32, P, ct.c_int32, D, D, D, D, I, I, I, I, F, P, I64, P, P],
            "or_pack_nodes": [P], "or_pack_samples": [P], "or_pack_copy": [P, P, I64, P, I64],
            "or_pack_free": [P], "or_threads": [],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ct.c_int
        L.or_pack.argtypes = [P, P, I]
        L.or_pack.restype = P
        L.or_pack_nodes.restype = ct.c_int64
        L.or_pack_samples.restype = ct.c_int64
        L.or_pack_free.restype = None
        _LIB = L
    return _LIB


def threads() -> int:
    return int(lib().or_threads())


# ----------------------------------------------------------------------------------------- EDT
def edt_squared(binary, brute=False):
    """int32 squared distance of every voxel to the nearest zero of ``binary``
    (src/field_engine/field_edt_integer_v1.py:14-26)."""
    b = np.ascontiguousarray(binary, dtype=np.uint8)
    out = np.empty(b.shape, np.int32)
    fn = lib().or_edt_squared_brute if brute else lib().or_edt_squared
    rc = fn(b.ctypes.data, *b.shape, out.ctypes.data)
    if rc:
        raise ValueError(f"oracle EDT status {rc}")
    return out


def edt_signed(mask, pitch, with_squared=False):
    """Signed float32 distance, negative inside ``mask``, half-pitch corrected
    (src/field_engine/edt_persistent_pair_v1/edt.cu:36-42)."""
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    out = np.empty(m.shape, np.float32)
    pair = np.empty((2,) + m.shape, np.int32)
    rc = lib().or_edt_signed(m.ctypes.data, *m.shape, float(pitch), out.ctypes.data, pair.ctypes.data)
    if rc:
        raise ValueError(f"oracle EDT status {rc}")
    return (out, pair) if with_squared else out


def edt_signed_numpy(mask, pitch, pair):
    """The reference's NumPy signed reconstruction from a squared pair
    (src/field_engine/field_edt_integer_v1.py:40-43)."""
    outside = (np.sqrt(pair[0].astype(np.float64)) * pitch).astype(np.float32)
    inside = (np.sqrt(pair[1].astype(np.float64)) * pitch).astype(np.float32)
    signed = (outside - inside).astype(np.float32)
    return (signed - np.sign(signed) * np.float32(0.5 * pitch)).astype(np.float32)


# ----------------------------------------------------------------------------------------- dense classify
def classify_dense(dense, pitch, block):
    """dict(kind, active_ids, tiles, ...) exactly as
    src/field_engine/faltkarna_v1_mesh_to_sdf.py:660-692 returns it."""
    import math
    d = np.ascontiguousarray(dense, dtype=np.float32)
    nx, ny, nz = d.shape
    n_bx, n_by, n_bz = -(-nx // block), -(-ny // block), -(-nz // block)
    margin = math.sqrt(3.0) * block * pitch
    kind = np.empty(n_bx * n_by * n_bz, np.int32)
    cma = np.empty(n_bx * n_by * n_bz, np.float32)
    rc = lib().or_classify_dense(d.ctypes.data, nx, ny, nz, block, float(np.float32(margin)), kind.ctypes.data,
                                 cma.ctypes.data)
    if rc:
        raise ValueError(f"oracle classify status {rc}")
    active = np.where(kind == 0)[0].astype(np.int32)
    tiles = np.empty((len(active), block, block, block), np.float32)
    if len(active):
        rc = lib().or_tiles_dense(d.ctypes.data, nx, ny, nz, block, active.ctypes.data, len(active),
                                  tiles.ctypes.data)
        if rc:
            raise ValueError(f"oracle tiles status {rc}")
    return dict(kind=kind, active_ids=active, tiles=tiles, n_bx=n_bx, n_by=n_by, n_bz=n_bz,
                n_blocks=int(len(kind)), n_active=int(len(active)), margin_mm=margin, corner_min_abs=cma)


# ----------------------------------------------------------------------------------------- CSG
def encode_program(instructions, nfields):
    """Encode ('union'|'difference'|'offset', left, right) triples into the reference's 24-byte
    records (src/field_engine/field_csg_batch_v1.py:59-64)."""
    enc = np.zeros(len(instructions), CSG_INSN)
    for i, (op, left, right) in enumerate(instructions):
        enc[i]["op"] = {"union": 0, "difference": 1, "offset": 2}[op]
        enc[i]["left"] = left
        if op == "offset":
            enc[i]["offset"] = right
        else:
            enc[i]["right"] = right
    return enc


def csg_execute(fields, instructions):
    """Dense float32 result of the ordered program; raises ValueError(status) like the reference
    (src/field_engine/csg_batch_native_v1/execute.cpp:10-53)."""
    arrs = [np.ascontiguousarray(f, dtype=np.float32) for f in fields]
    shape = np.array(arrs[0].shape, np.int32)
    ptrs = (ct.c_void_p * len(arrs))(*(a.ctypes.data for a in arrs))
    enc = encode_program(instructions, len(arrs))
    out = np.empty(arrs[0].shape, np.float32)
    rc = lib().or_csg_execute(ptrs, len(arrs), shape.ctypes.data, enc.ctypes.data, len(enc), out.ctypes.data)
    if rc:
        raise ValueError(f"oracle CSG status {rc}")
    return out


# ----------------------------------------------------------------------------------------- packing
def pack(samples, threshold=512):
    """(nodes, payload) with the reference's split decisions
    (src/field_engine/adaptive_pack_native_v1/pack.cpp:18-69)."""
    a = np.ascontiguousarray(samples, dtype=np.float32)
    shape = np.array(a.shape, np.int32)
    h = lib().or_pack(a.ctypes.data, shape.ctypes.data, int(threshold))
    if not h:
        raise ValueError("oracle packing refused the input")
    try:
        nodes = np.empty(lib().or_pack_nodes(h), NODE)
        payload = np.empty(lib().or_pack_samples(h), np.float32)
        if lib().or_pack_copy(h, nodes.ctypes.data, len(nodes), payload.ctypes.data, len(payload)):
            raise RuntimeError("oracle pack copy failed")
    finally:
        lib().or_pack_free(h)
    return nodes, payload


def samples_at(nodes, payload, indices):
    """Exact sample bits at integer indices by walking the packed tree
    (src/field_engine/adaptive_sample_blocks_v1.py:103-128)."""
    idx = np.asarray(indices, dtype=np.int64)
    out = np.empty(len(idx), np.float32)
    pending = [(0, np.arange(len(idx)))]
    while pending:
        nid, sel = pending.pop()
        if not len(sel):
            continue
        node = nodes[nid]
        left, right = node["children"]
        if left < 0:
            local = idx[sel] - node["lo"]
            local[:, node["stored_shape"] == 1] = 0
            lin = np.ravel_multi_index(local.T, tuple(node["stored_shape"]))
            out[sel] = payload[node["offset"] + lin]
        else:
            b = nodes[left]
            inl = np.all((idx[sel] >= b["lo"]) & (idx[sel] < b["lo"] + b["shape"]), axis=1)
            pending.append((int(right), sel[~inl]))
            pending.append((int(left), sel[inl]))
    return out


def query_trilinear(nodes, payload, shape, origin, pitch, points):
    """float32 trilinear value on the fine grid, coordinates clipped into the grid, eight samples
    gathered across leaves, interpolated by scipy.ndimage.map_coordinates(order=1, mode='nearest')
    (src/field_engine/adaptive_sample_blocks_v1.py:130-151)."""
    import itertools
    from scipy import ndimage
    pts = np.asarray(points, dtype=np.float64)
    out = np.empty(len(pts), np.float32)
    offsets = np.array(list(itertools.product((0, 1), repeat=3)), dtype=np.int64)
    shp = np.array(shape)
    for start in range(0, len(pts), 4096):
        batch = pts[start:start + 4096]
        c = np.clip((batch - np.asarray(origin, np.float64)) / pitch, 0, shp - 1)
        lower = np.floor(c).astype(np.int64)
        frac = c - lower
        nb = np.minimum(lower[:, None, :] + offsets, shp - 1)
        corners = samples_at(nodes, payload, nb.reshape(-1, 3)).reshape(-1, 2, 2, 2)
        q = np.vstack((np.arange(len(batch)), frac.T))
        out[start:start + len(batch)] = ndimage.map_coordinates(corners, q, order=1, mode="nearest")
    return out


# ----------------------------------------------------------------------------------------- analytic
def eval_points(prims, prog, points):
    """float64 program values at (N, 3) float64 points (src/field_engine/ikarus_v1/expr.py:263-385)."""
    P = np.ascontiguousarray(prims, PRIM)
    G = np.ascontiguousarray(prog, INSN)
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    out = np.empty(len(pts), np.float64)
    rc = lib().or_eval_points(P.ctypes.data, len(P), G.ctypes.data, len(G), pts.ctypes.data, len(pts),
                              out.ctypes.data)
    if rc:
        raise ValueError(f"oracle eval status {rc}")
    return out


def classify_program(prims, prog, meta):
    """(kind int32, corner_min_abs float64) of every block, float64 corners
    (src/field_engine/faltkarna_v1.py:129-164)."""
    P = np.ascontiguousarray(prims, PRIM)
    G = np.ascontiguousarray(prog, INSN)
    kind = np.empty(meta.n_blocks, np.int32)
    cma = np.empty(meta.n_blocks, np.float64)
    rc = lib().or_classify_program(P.ctypes.data, len(P), G.ctypes.data, len(G), meta.x0, meta.y0, meta.z0,
                                   meta.pitch, meta.nx, meta.ny, meta.nz, meta.block,
                                   float(np.float32(meta.margin_mm)), kind.ctypes.data, cma.ctypes.data)
    if rc:
        raise ValueError(f"oracle classify status {rc}")
    return kind, cma


def classify_blocks(prims, prog, meta, blocks):
    """(kind, corner_min_abs) of the listed blocks only (faltkarna_v1.py:129-164)."""
    P = np.ascontiguousarray(prims, PRIM)
    G = np.ascontiguousarray(prog, INSN)
    b = np.ascontiguousarray(blocks, np.int64)
    kind = np.empty(len(b), np.int32)
    cma = np.empty(len(b), np.float64)
    rc = lib().or_classify_blocks(P.ctypes.data, len(P), G.ctypes.data, len(G), meta.x0, meta.y0, meta.z0,
                                  meta.pitch, meta.nx, meta.ny, meta.nz, meta.block,
                                  float(np.float32(meta.margin_mm)), b.ctypes.data, len(b), kind.ctypes.data,
                                  cma.ctypes.data)
    if rc:
        raise ValueError(f"oracle classify status {rc}")
    return kind, cma


def tiles_program(prims, prog, meta, active_ids):
    """float64 leaf values (n_active, B, B, B) of the given blocks (src/field_engine/faltkarna_v1.py:167-190)."""
    P = np.ascontiguousarray(prims, PRIM)
    G = np.ascontiguousarray(prog, INSN)
    act = np.ascontiguousarray(active_ids, np.int32)
    b = meta.block
    out = np.empty((len(act), b, b, b), np.float64)
    rc = lib().or_tiles_program(P.ctypes.data, len(P), G.ctypes.data, len(G), meta.x0, meta.y0, meta.z0,
                                meta.pitch, meta.nx, meta.ny, meta.nz, b, act.ctypes.data, len(act),
                                out.ctypes.data)
    if rc:
        raise ValueError(f"oracle tiles status {rc}")
    return out


# ----------------------------------------------------------------------------------------- reference libs
def ref_library(name):
    """A reference CPU library compiled from the reference's own sources into oracle/_ref/
    (``pack``, ``csg_batch`` or ``mesh_sdf``); None when it was not built on this machine."""
    path = HERE / "_ref" / f"libref_{name}.so"
    if not path.exists():
        return None
    return ct.CDLL(str(path))


def ref_classify_dense(dense, pitch, block, nthreads=0):
    """The reference's meshsdf_classify_cpu + meshsdf_tiles_cpu (OpenMP), same dict as
    src/field_engine/mesh_sdf_native_v1.py:121-141."""
    import math
    L = ref_library("mesh_sdf")
    if L is None:
        raise RuntimeError("oracle/_ref/libref_mesh_sdf.so is not built")
    P, I64 = ct.c_void_p, ct.c_int64
    L.meshsdf_classify_cpu.argtypes = [P, I64, I64, I64, I64, ct.c_float, P, ct.c_int]
    L.meshsdf_classify_cpu.restype = ct.c_int
    L.meshsdf_tiles_cpu.argtypes = [P, I64, I64, I64, I64, P, I64, P, ct.c_int]
    L.meshsdf_tiles_cpu.restype = ct.c_int
    d = np.ascontiguousarray(dense, dtype=np.float32)
    nx, ny, nz = d.shape
    n_bx, n_by, n_bz = -(-nx // block), -(-ny // block), -(-nz // block)
    margin = math.sqrt(3.0) * block * pitch
    kind = np.empty(n_bx * n_by * n_bz, np.int32)
    rc = L.meshsdf_classify_cpu(d.ctypes.data, nx, ny, nz, block, float(np.float32(margin)), kind.ctypes.data,
                                int(nthreads))
    if rc:
        raise RuntimeError(f"reference classify status {rc}")
    active = np.where(kind == 0)[0].astype(np.int32)
    tiles = np.empty((len(active), block, block, block), np.float32)
    if len(active):
        rc = L.meshsdf_tiles_cpu(d.ctypes.data, nx, ny, nz, block, active.ctypes.data, len(active),
                                 tiles.ctypes.data, int(nthreads))
        if rc:
            raise RuntimeError(f"reference tiles status {rc}")
    return dict(kind=kind, active_ids=active, tiles=tiles, n_bx=n_bx, n_by=n_by, n_bz=n_bz,
                n_blocks=int(len(kind)), n_active=int(len(active)), margin_mm=margin)


def ref_pack(samples, threshold=512):
    """The reference's adaptive_pack compiled from pack.cpp: (nodes, payload)."""
    L = ref_library("pack")
    if L is None:
        raise RuntimeError("oracle/_ref/libref_pack.so is not built")
    L.adaptive_pack.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int]
    L.adaptive_pack.restype = ct.c_void_p
    for name in ("adaptive_nodes", "adaptive_samples"):
        getattr(L, name).argtypes = [ct.c_void_p]
        getattr(L, name).restype = ct.c_int64
    L.adaptive_copy.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_int64]
    L.adaptive_copy.restype = ct.c_int
    L.adaptive_free.argtypes = [ct.c_void_p]
    L.adaptive_free.restype = None
    a = np.ascontiguousarray(samples, dtype=np.float32)
    shape = np.array(a.shape, np.int32)
    h = L.adaptive_pack(a.ctypes.data, shape.ctypes.data, int(threshold))
    if not h:
        raise ValueError("reference packing refused the input")
    try:
        nodes = np.empty(L.adaptive_nodes(h), NODE)
        payload = np.empty(L.adaptive_samples(h), np.float32)
        if L.adaptive_copy(h, nodes.ctypes.data, len(nodes), payload.ctypes.data, len(payload)):
            raise RuntimeError("reference pack copy failed")
    finally:
        L.adaptive_free(h)
    return nodes, payload


# ----------------------------------------------------------------------------------------- multires
def multires_brick(lo, L, brick_shape, kind, pts):
    """Brick per point, preferring the active brick on a face (faltkarna_v1_multires.py:384-402)."""
    rel = (np.asarray(pts, dtype=np.float64) - lo) / L
    b = np.floor(rel).astype(np.int64)
    shp = np.array(brick_shape, dtype=np.int64)
    outside = np.any((b < 0) | (b >= shp), axis=1)
    b = np.clip(b, 0, shp - 1)
    inactive = kind[b[:, 0], b[:, 1], b[:, 2]] != 0
    for ax in range(3):
        on_plane = (rel[:, ax] == np.floor(rel[:, ax])) & (b[:, ax] > 0) & inactive & ~outside
        if not on_plane.any():
            continue
        cand = b[on_plane].copy()
        cand[:, ax] -= 1
        ok = kind[cand[:, 0], cand[:, 1], cand[:, 2]] == 0
        idx = np.where(on_plane)[0][ok]
        b[idx, ax] -= 1
        inactive = kind[b[:, 0], b[:, 1], b[:, 2]] != 0
    return b, outside


def multires_avstand(lo, h, block, brick_shape, kind, niva, tiles, margin, pts):
    """faltkarna_v1_multires.py:405-434 restated: trilinear at the brick's own pitch, +-margin
    elsewhere; float64 (N,)."""
    from scipy import ndimage
    pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
    L = block * h
    b, outside = multires_brick(lo, L, brick_shape, kind, pts)
    n_by, n_bz = brick_shape[1], brick_shape[2]
    lin = (b[:, 0] * n_by + b[:, 1]) * n_bz + b[:, 2]
    kd = kind[b[:, 0], b[:, 1], b[:, 2]]
    out = np.where(kd < 0, -margin, margin).astype(np.float64)
    out[outside] = margin
    act = (kd == 0) & ~outside
    for i in np.where(act)[0]:
        u = int(lin[i])
        bi, bj, bk = u // (n_by * n_bz), (u // n_bz) % n_by, u % n_bz
        lvl = int(niva[bi, bj, bk])
        o = lo + np.array([bi, bj, bk], dtype=np.float64) * L
        lok = (pts[i:i + 1] - o) / (h / float(1 << lvl))
        out[i] = ndimage.map_coordinates(tiles[u], lok.T, order=1, mode="nearest")[0]
    return out


def multires_gradient(lo, h, block, brick_shape, kind, niva, tiles, margin, pts):
    """faltkarna_v1_multires.py:437-459 restated; float64 (N, 3)."""
    pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
    L = block * h
    b, _ = multires_brick(lo, L, brick_shape, kind, pts)
    lvl = niva[b[:, 0], b[:, 1], b[:, 2]].astype(np.int64)
    hh = h / np.power(2.0, np.maximum(lvl, 0))
    o = lo + b.astype(np.float64) * L
    g = np.zeros((len(pts), 3))
    for ax in range(3):
        d = np.zeros((len(pts), 3))
        d[:, ax] = hh
        pa = np.minimum(pts + 0.5 * d, o + L)
        pb = np.maximum(pts - 0.5 * d, o)
        step = pa[:, ax] - pb[:, ax]
        g[:, ax] = (multires_avstand(lo, h, block, brick_shape, kind, niva, tiles, margin, pa) -
                    multires_avstand(lo, h, block, brick_shape, kind, niva, tiles, margin, pb)) / np.maximum(step, 1e-12)
    return g


# ----------------------------------------------------------------------------------------- adaptive block tree
TREE_SIDES = (8, 4, 2, 1)


def tree_build(dense, pitch):
    """The packed adaptive block tree of src/field_engine/field_adaptive_blocks_v1.py:113-147,
    restated level by level: dict(shape, root_shape, root_count, node_count, packed,
    branch_prefix, value_prefix, values, histogram).  Block kinds from classify_dense at sides 8,
    4, 2, 1; a node at corner (x, y, z) is 0 outside the grid or for kind > 0, 1 for kind < 0, 3
    (with dense[x, y, z] appended to the values) for kind 0 at side 1, else 2 with its 8 children
    (x + i h, y + j h, z + k h), i, j, k in C order, appended in breadth-first order."""
    d = np.ascontiguousarray(dense, dtype=np.float32)
    shape = d.shape
    kinds = {}
    for side in TREE_SIDES:
        nb = tuple(-(-n // side) for n in shape)
        kinds[side] = classify_dense(d, pitch, side)["kind"].reshape(nb)
    root_shape = kinds[8].shape
    coords = (np.indices(root_shape).reshape(3, -1).T * 8).astype(np.int64)
    offsets = np.array([(i, j, k) for i in (0, 1) for j in (0, 1) for k in (0, 1)], np.int64)
    codes, values, hist = [], np.zeros(0, np.float32), {}
    for side in TREE_SIDES:
        if len(coords) == 0:
            break
        x, y, z = coords.T
        inside = (x < shape[0]) & (y < shape[1]) & (z < shape[2])
        k = np.ones(len(coords), np.int64)
        k[inside] = kinds[side][x[inside] // side, y[inside] // side, z[inside] // side]
        code = np.zeros(len(coords), np.uint8)
        code[inside & (k < 0)] = 1
        code[inside & (k == 0)] = 3 if side == 1 else 2
        codes.append(code)
        for c in (0, 1, 3):
            cnt = int(np.count_nonzero(code == c))
            if cnt:
                hist[f"side{side}_kind{c}"] = cnt
        if side == 1:
            values = d[x[code == 3], y[code == 3], z[code == 3]].astype(np.float32)
        coords = (coords[code == 2][:, None, :] + offsets[None] * (side // 2)).reshape(-1, 3)
    code = np.concatenate(codes)
    padded = np.pad(code, (0, (-len(code)) % 4))
    packed = (padded.reshape(-1, 4).astype(np.uint32) << np.array([0, 2, 4, 6], np.uint32)).sum(axis=1).astype(np.uint8)
    prefixes = []
    for c in (2, 3):
        per_byte = ((packed[:, None] >> np.array([0, 2, 4, 6], np.uint8)) & 3 == c).sum(axis=1)
        cumulative = np.concatenate(([0], np.cumsum(per_byte)))
        prefixes.append(cumulative[0:len(packed) + 1:64].astype(np.int32))
    return dict(shape=shape, root_shape=root_shape, root_count=int(np.prod(root_shape)), node_count=len(code),
                packed=packed, branch_prefix=prefixes[0], value_prefix=prefixes[1], values=values,
                histogram=dict(sorted(hist.items())))


def tree_sample(tree, indices, pitch):
    """float32 values of a tree_build dict at integer grid coordinates [N, 3]
    (field_adaptive_blocks_v1.py:53-82): descend by child octant, ranking with full prefix counts."""
    ijk = np.asarray(indices, dtype=np.int64)
    codes = ((tree["packed"][:, None] >> np.array([0, 2, 4, 6], np.uint8)) & 3).reshape(-1)
    before = {c: np.concatenate(([0], np.cumsum(codes == c))) for c in (2, 3)}
    rs = tree["root_shape"]
    node = ((ijk[:, 0] // 8) * rs[1] + ijk[:, 1] // 8) * rs[2] + ijk[:, 2] // 8
    size = np.full(len(ijk), 8, np.int64)
    out = np.full(len(ijk), np.nan, np.float32)
    todo = np.arange(len(ijk))
    while len(todo):
        c = codes[node[todo]]
        leaf = todo[c < 2]
        sign = np.where(c[c < 2] == 0, 1.0, -1.0)
        out[leaf] = sign * np.sqrt(3.0) * size[leaf] * pitch
        val = todo[c == 3]
        out[val] = tree["values"][before[3][node[val]]]
        br = todo[c == 2]
        half = size[br] // 2
        octant = (ijk[br] // half[:, None]) % 2
        node[br] = tree["root_count"] + 8 * before[2][node[br]] + 4 * octant[:, 0] + 2 * octant[:, 1] + octant[:, 2]
        size[br] = half
        todo = br
    return out


# ----------------------------------------------------------------------------------------- mesh -> field
def ref_mesh_field(V, T, origin, pitch, jitter, shape, surface_correction=True, nthreads=0):
    """The reference's meshsdf_field_cpu (src/field_engine/mesh_sdf_native_v1/field.cpp:19-226, OpenMP),
    compiled from its source into oracle/_ref: (status, solid bool, sd float32, surface bool,
    stats int64[4])."""
    L = ref_library("mesh_sdf")
    if L is None:
        raise RuntimeError("oracle/_ref/libref_mesh_sdf.so is not built")
    P, I64, D, I = ct.c_void_p, ct.c_int64, ct.c_double, ct.c_int
    L.meshsdf_field_cpu.argtypes = [P, I64, P, I64, D, D, D, D, D, D, I64, I64, I64, I, I, P, P, P, P, P]
    L.meshsdf_field_cpu.restype = I
    Vf = np.ascontiguousarray(V, dtype=np.float64)
    Ti = np.ascontiguousarray(T, dtype=np.int64)
    nx, ny, nz = (int(v) for v in shape)
    solid = np.zeros((nx, ny, nz), np.uint8)
    sd = np.zeros((nx, ny, nz), np.float32)
    yta = np.zeros((nx, ny, nz), np.uint8)
    stats = np.zeros(4, np.int64)
    ts = np.zeros(5, np.float64)
    rc = L.meshsdf_field_cpu(Vf.ctypes.data, len(Vf), Ti.ctypes.data, len(Ti), float(origin[0]), float(origin[1]),
                             float(origin[2]), float(pitch), float(jitter[0]), float(jitter[1]), nx, ny, nz,
                             int(bool(surface_correction)), int(nthreads), solid.ctypes.data, sd.ctypes.data,
                             yta.ctypes.data, stats.ctypes.data, ts.ctypes.data)
    return rc, solid.view(bool), sd, yta.view(bool), stats


# ----------------------------------------------------------------------------------------- machining scene
def cnc_subtract(table, r0_2d, z0_2d, pitch2d, pts, r_blank, z_blank_lo, z_blank_hi, px, py, arch_r, arch_cz,
                 rho_mill, drill_r, drill_z, drill_x_half):
    """float64 material field of the reference's machining kernel at points (N, 3), operation for
    operation (src/field_engine/tillverkningsfalt_v1_kernel.py:248-300): blank, bilinear turned
    profile, max, the pocket subtracted, the bore subtracted."""
    x, y, z = (np.asarray(pts, np.float64)[:, k] for k in range(3))
    nr2d, nz2d = table.shape
    r = np.sqrt(x * x + y * y)
    blank = np.maximum(r - r_blank, np.maximum(z_blank_lo - z, z - z_blank_hi))
    fr = (r - r0_2d) / pitch2d
    fz = (z - z0_2d) / pitch2d
    ir0 = np.clip(np.trunc(fr).astype(np.int64), 0, nr2d - 2)
    iz0 = np.clip(np.trunc(fz).astype(np.int64), 0, nz2d - 2)
    tr = np.clip(fr - ir0, 0.0, 1.0)
    tz = np.clip(fz - iz0, 0.0, 1.0)
    t = table.astype(np.float64)
    turned = (t[ir0, iz0] * (1 - tr) * (1 - tz) + t[ir0, iz0 + 1] * (1 - tr) * tz + t[ir0 + 1, iz0] * tr * (1 - tz)
              + t[ir0 + 1, iz0 + 1] * tr * tz)
    material = np.maximum(blank, turned)
    qx = np.abs(x) - (px - rho_mill)
    qy = np.abs(y) - (py - rho_mill)
    dxy = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2) + np.minimum(np.maximum(qx, qy), 0) - rho_mill
    roof = arch_cz + np.sqrt(np.maximum(arch_r * arch_r - x * x, 0.0))
    material = np.maximum(material, -np.maximum(dxy, z - roof))
    bore = np.maximum(np.sqrt(y * y + (z - drill_z) ** 2) - drill_r, np.abs(x) - drill_x_half)
    return np.maximum(material, -bore)


def multires_overlap_band(lo, h, block, brick_shape, kind, niva, tiles):
    """faltkarna_v1_multires.py:211-251 restated: bricks in ascending id, faces axis 0..2, side -1 then
    +1, each face of a fine brick next to an active coarser brick overwritten in place with
    scipy.ndimage.map_coordinates(order=1, mode='nearest') of that brick's lattice.  Returns (new
    tiles dict, faces written)."""
    from scipy import ndimage
    tiles = {k: v.copy() for k, v in tiles.items()}
    n_bx, n_by, n_bz = brick_shape
    L = block * h
    faces = 0
    for lin in sorted(tiles):
        bi, bj, bk = lin // (n_by * n_bz), (lin // n_bz) % n_by, lin % n_bz
        lvl = int(niva[bi, bj, bk])
        if lvl == 0:
            continue
        n_l = block * (1 << lvl)
        b_origin = lo + np.array([bi, bj, bk], dtype=np.float64) * L
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
                pts = np.stack([gi.ravel(), gj.ravel(), gk.ravel()], axis=1) * (h / float(1 << lvl)) + b_origin
                nb_origin = lo + np.array(nb, dtype=np.float64) * L
                lok = (pts - nb_origin) / (h / float(1 << lvl_n))
                nlin = (nb[0] * n_by + nb[1]) * n_bz + nb[2]
                v = ndimage.map_coordinates(tiles[nlin], lok.T, order=1, mode="nearest")
                sl = [slice(None)] * 3
                sl[ax] = 0 if sida < 0 else n_l
                tiles[lin][tuple(sl)] = v.reshape(tiles[lin][tuple(sl)].shape).astype(np.float32)
                faces += 1
    return tiles, faces


def reconstruct(kind, active_ids, tiles, meta, big=1.0e6):
    """Dense (nx, ny, nz) float32 field of a sparse one: tiles in active blocks, -big / +big by kind
    elsewhere (src/field_engine/faltkarna_v1.py:302-325)."""
    b = meta.block
    nbx, nby, nbz = meta.n_bx, meta.n_by, meta.n_bz
    bg = np.where(np.asarray(kind).reshape(nbx, nby, nbz) < 0, -big, big).astype(np.float32)
    padded = np.repeat(np.repeat(np.repeat(bg, b, 0), b, 1), b, 2)
    view = padded.reshape(nbx, b, nby, b, nbz, b).transpose(0, 2, 4, 1, 3, 5)
    if len(active_ids):
        bi, bj, bk = np.unravel_index(np.asarray(active_ids), (nbx, nby, nbz))
        view[bi, bj, bk] = np.asarray(tiles, np.float32).reshape(len(active_ids), b, b, b)
    return padded[:meta.nx, :meta.ny, :meta.nz]


# Marching cubes of the export step, restated on the dense field (the reference exports through
# rekonstruera_tat and skimage.measure.marching_cubes, faltkarna_v1.py:302-350; scikit-image is not
# part of this environment).  The rules written out: a vertex on every grid edge whose ends lie on
# opposite sides of `level` (inside = value < level), at t = g0 / (g0 - g1), g = float64(value) -
# float64(level), position float32(origin + pitch (index + t)); per cube, segments on each face that
# keep the inside on their left seen from outside (four crossings: the asymptotic decider, inside
# corners joined when the saddle value g00 g11 - g10 g01 over (g00 + g11 - g10 - g01) is negative),
# joined into loops, each loop fanned with outward (increasing value) normals from its first vertex,
# in loop order from the lowest cube edge, that lies on no cube face the loop crosses twice (else
# from the lowest edge): a fan from such a face would lay a flat triangle into it, which the cube
# on the other side may lay too.  Corner c = x | y << 1 | z << 2; edge e = axis * 4 + w, w the other
# two bits (lower axis first); face f = axis * 2 + side.

def _edge_corner0(e):
    a, w = e >> 2, e & 3
    if a == 0:
        return ((w & 1) << 1) | ((w >> 1) << 2)
    if a == 1:
        return (w & 1) | ((w >> 1) << 2)
    return (w & 1) | ((w >> 1) << 1)


def _edge_of(ca, cb):
    d = (ca ^ cb).bit_length() - 1
    c = ca & cb
    if d == 0:
        w = ((c >> 1) & 1) | (((c >> 2) & 1) << 1)
    elif d == 1:
        w = (c & 1) | (((c >> 2) & 1) << 1)
    else:
        w = (c & 1) | (((c >> 1) & 1) << 1)
    return d * 4 + w


def _edge_faces(e):
    """Bit mask of the two cube faces that contain edge e."""
    c0, a = _edge_corner0(e), e >> 2
    return sum(1 << (b * 2 + ((c0 >> b) & 1)) for b in range(3) if b != a)


def _fan_start(loop):
    """The loop rotated to start at its fan centre."""
    seen, twice = 0, 0
    for i in range(len(loop)):
        f = _edge_faces(loop[i]) & _edge_faces(loop[(i + 1) % len(loop)])
        twice |= seen & f
        seen |= f
    for i, e in enumerate(loop):
        if not _edge_faces(e) & twice:
            return loop[i:] + loop[:i]
    return loop


def _cube_loops(g):
    """Loops (lists of cube edges, in traversal order) of one cube; g: 8 float64 values - level."""
    inside = [g[c] < 0.0 for c in range(8)]
    if all(inside) or not any(inside):
        return []
    cross = [inside[_edge_corner0(e)] != inside[_edge_corner0(e) | (1 << (e >> 2))] for e in range(12)]
    nxt = {}
    for f in range(6):
        a, s = f >> 1, f & 1
        u, v = (a + 1) % 3, (a + 2) % 3
        b = s << a
        q = [b, b | (1 << (u if s else v)), b | (1 << u) | (1 << v), b | (1 << (v if s else u))]
        E = [_edge_of(q[i], q[(i + 1) % 4]) for i in range(4)]
        iq = [inside[c] for c in q]
        k = sum(iq[i] != iq[(i + 1) % 4] for i in range(4))
        if k == 2:
            st = [E[i] for i in range(4) if iq[i] and not iq[(i + 1) % 4]][0]
            en = [E[i] for i in range(4) if not iq[i] and iq[(i + 1) % 4]][0]
            nxt[st] = en
        elif k == 4:
            g00, g10, g11, g01 = g[b], g[b | (1 << u)], g[b | (1 << u) | (1 << v)], g[b | (1 << v)]
            num = np.float64(g00) * np.float64(g11) - np.float64(g10) * np.float64(g01)
            joined = (num > 0.0) if g00 < 0.0 else (num < 0.0)
            for i in range(4):
                if iq[i]:
                    nxt[E[i]] = E[(i + 1) % 4] if joined else E[(i + 3) % 4]
    loops, todo = [], sorted(e for e in range(12) if cross[e])
    seen = set()
    for e0 in todo:
        if e0 in seen:
            continue
        loop, e = [], e0
        while True:
            seen.add(e)
            loop.append(e)
            e = nxt[e]
            if e == e0:
                break
        loops.append(loop)
    return loops


def marching_cubes(dense, level=0.0, origin=(0.0, 0.0, 0.0), pitch=1.0):
    """(keys, verts, faces): keys int64 ((i ny + j) nz + k) 3 + axis of each crossing edge in
    ascending order, verts float32 (V, 3), faces (T, 3) as edge keys, cubes in lexicographic order
    and loops by lowest edge (the rules above)."""
    f = np.asarray(dense, np.float32)
    nx, ny, nz = f.shape
    n = (nx, ny, nz)
    g = f.astype(np.float64) - np.float64(level)
    inside = g < 0.0
    keys, pos = [], []
    for a in range(3):
        s0, s1 = [slice(None)] * 3, [slice(None)] * 3
        s0[a], s1[a] = slice(0, n[a] - 1), slice(1, n[a])
        cross = inside[tuple(s0)] != inside[tuple(s1)]
        idx = np.argwhere(cross)
        g0, g1 = g[tuple(s0)][cross], g[tuple(s1)][cross]
        p = idx.astype(np.float64)
        p[:, a] = p[:, a] + g0 / (g0 - g1)
        pos.append((np.asarray(origin, np.float64) + pitch * p).astype(np.float32))
        keys.append(((idx[:, 0].astype(np.int64) * ny + idx[:, 1]) * nz + idx[:, 2]) * 3 + a)
    keys, pos = np.concatenate(keys), np.concatenate(pos)
    order = np.argsort(keys, kind="stable")
    keys, pos = keys[order], pos[order]
    faces = []
    if nx > 1 and ny > 1 and nz > 1:
        c = inside[:-1, :-1, :-1].astype(np.int32)
        cnt = sum(inside[dx:nx - 1 + dx, dy:ny - 1 + dy, dz:nz - 1 + dz].astype(np.int32)
                  for dx in (0, 1) for dy in (0, 1) for dz in (0, 1))
        del c
        for m in np.argwhere((cnt > 0) & (cnt < 8)):
            i, j, k = (int(x) for x in m)
            gc = [g[i + (c & 1), j + ((c >> 1) & 1), k + ((c >> 2) & 1)] for c in range(8)]
            for loop in _cube_loops(gc):
                loop = _fan_start(loop)
                ek = []
                for e in loop:
                    cc = _edge_corner0(e)
                    pi, pj, pk = i + (cc & 1), j + ((cc >> 1) & 1), k + ((cc >> 2) & 1)
                    ek.append(((pi * ny + pj) * nz + pk) * 3 + (e >> 2))
                for t in range(1, len(ek) - 1):
                    faces.append((ek[0], ek[t + 1], ek[t]))
    return keys, pos, np.asarray(faces, np.int64).reshape(-1, 3)


def mesh_volume(verts, faces):
    """Signed volume sum(v0 . (v1 x v2)) / 6 of a triangle mesh, float64 (the divergence theorem,
    as trimesh's volume in faltvolym_v1.py:83-104)."""
    v = np.asarray(verts, np.float64)
    a, b, c = v[faces[:, 0]], v[faces[:, 1]], v[faces[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


# ------------------------------------------------------------------------- EDT consumers
def clearance_mm(occ, pitch):
    """float64 clearance of every cell to the nearest occupied one times the pitch: scipy's
    ``distance_transform_edt(~occ) * pitch`` (src/field_engine/opt/laplaceflode_v1.py:313-314),
    restated as the float64 root of the oracle's exact squared EDT to the occupied cells."""
    occ = np.asarray(occ, bool)
    sq = edt_squared(~occ)  # zeros of ~occ are the occupied cells
    return np.sqrt(sq.astype(np.float64)) * float(pitch)


def lattice_laplacian(occ, edt_mm, pitch, p_kond=1.5):
    """Restatement of bygg_gitterlaplacian (src/field_engine/opt/laplaceflode_v1.py:69-97) that
    builds the CSR directly instead of through a COO sum: returns (n, node_map, u, v, kond, indptr,
    indices, data).  Rows list their columns ascending (p - sx, p - sy, p - 1, p, p + 1, p + sy,
    p + sx in C order); the diagonal is the left-to-right sum of the row's conductances in the COO's
    order (the cell as lower end of its axis 0, 1, 2 edges, then as upper end), which is the order
    scipy's sum_duplicates adds them in.  Absent edges add 0.0, which leaves every sum unchanged."""
    occ = np.asarray(occ, bool)
    shape3 = (1,) * (3 - occ.ndim) + occ.shape
    fri = ~occ.reshape(shape3)
    E = np.asarray(edt_mm, np.float64).reshape(shape3)
    n = int(fri.sum())
    node = np.full(shape3, -1, np.int32)
    node[fri] = np.arange(n, dtype=np.int32)
    fwd, bwd, kf, kb = [], [], [], []
    U, V, K = [], [], []
    for a in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[a], hi[a] = slice(None, -1), slice(1, None)
        lo, hi = tuple(lo), tuple(hi)
        e = np.zeros(shape3, bool)
        e[lo] = fri[lo] & fri[hi]          # cell is the lower end of an axis-a edge
        b = np.zeros(shape3, bool)
        b[hi] = e[lo]                      # cell is the upper end of one
        c = np.zeros(shape3)
        c[lo] = 0.5 * (E[lo] + E[hi]) / pitch
        k = np.where(e, np.maximum(c, 0.1) ** p_kond, 0.0)
        kup = np.zeros(shape3)
        kup[hi] = k[lo]
        fwd.append(e)
        bwd.append(b)
        kf.append(k)
        kb.append(kup)
        U.append(node[lo][e[lo]])
        V.append(node[hi][e[lo]])
        K.append(k[lo][e[lo]])
    u, v, kond = np.concatenate(U), np.concatenate(V), np.concatenate(K)
    strides = (shape3[1] * shape3[2], shape3[2], 1)
    lin = np.arange(fri.size).reshape(shape3)
    diag = ((((kf[0] + kf[1]) + kf[2]) + kb[0]) + kb[1]) + kb[2]
    deg = sum(x.astype(np.int64) for x in fwd + bwd)
    has = fri & (deg > 0)
    # slots in column order: -x, -y, -z, diagonal, +z, +y, +x
    present = [bwd[0], bwd[1], bwd[2], has, fwd[2], fwd[1], fwd[0]]
    cols = [lin - strides[0], lin - strides[1], lin - strides[2], lin, lin + strides[2], lin + strides[1],
            lin + strides[0]]
    vals = [-kb[0], -kb[1], -kb[2], diag, -kf[2], -kf[1], -kf[0]]
    cells = np.nonzero(fri.ravel())[0]
    P = np.stack([p.ravel()[cells] for p in present], axis=1)
    C = np.stack([np.where(p.ravel()[cells], node.ravel()[np.clip(c.ravel()[cells], 0, fri.size - 1)], 0)
                  for p, c in zip(present, cols)], axis=1)
    Vv = np.stack([x.ravel()[cells] for x in vals], axis=1)
    counts = P.sum(axis=1)
    indptr = np.zeros(n + 1, np.int32)
    np.cumsum(counts, out=indptr[1:])
    indices = C[P].astype(np.int32)
    data = Vv[P]
    return n, node.reshape(occ.shape), u, v, kond, indptr, indices, data
