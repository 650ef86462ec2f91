"""Packed adaptive sampled fields and ordered CSG over them, on the GPU.

Drop-in surfaces (same names, arguments, return types and errors):

* ``AdaptiveSampleBlocks(samples, origin, pitch, *, leaf_samples=512)`` and
  ``NativeAdaptiveBlocks(samples, origin, pitch, *, library=None, leaf_samples=512)`` --
  src/field_engine/adaptive_sample_blocks_v1.py:140-230 and adaptive_pack_native_v1.py:249-299:
  lossless packing (52-byte NODE records + float32 payload) with the reference's split decisions,
  ``samples_at(indices)``, ``query(points)``, ``storage_bytes``.
* ``compose(left, right=None, *, operation='union', distance=0.)`` --
  src/field_engine/field_csg_blocks_v1.py:12-43.
* ``evaluate(fields, instructions, *, batch_library=None, pack_library=None)`` --
  src/field_engine/field_csg_batch_v1.py:18-79 (program of ('union'|'difference'|'offset', left,
  right) triples; instruction i produces id len(fields)+i).

Packing, CSG and queries run in libfield_b200.so (csrc/pack.cu); the library arguments name the
CUDA library to bind (default: the in-tree build).
"""
from __future__ import annotations

import ctypes as ct
import operator
import sys
from numbers import Real

import numpy as np

from . import _lib

NODE = np.dtype([("lo", "<i4", (3,)), ("shape", "<i4", (3,)), ("stored_shape", "<i4", (3,)),
                 ("children", "<i4", (2,)), ("offset", "<i8")])
CSG_INSN = np.dtype([("op", "<i4"), ("left", "<i4"), ("right", "<i4"), ("pad", "<i4"), ("offset", "<f8")])

P, I, I64, D = ct.c_void_p, ct.c_int, ct.c_int64, ct.c_double
_SIGS = {
    "adaptive_pack": (P, [P, P, I]),
    "fb_pack_device": (P, [P, P, I, P]),
    "adaptive_nodes": (I64, [P]),
    "adaptive_samples": (I64, [P]),
    "adaptive_copy": (I, [P, P, I64, P, I64]),
    "adaptive_free": (None, [P]),
    "csg_execute": (I, [P, P, P, P, ct.c_int32, P, P, ct.c_int32, P]),
    "fb_packed_samples_at": (I, [P, I64, P, I64, P, I64, P]),
    "fb_packed_query_device": (I, [P, P, P, P, D, P, I64, P, P]),
}


def _bind(library=None):
    L = _lib.lib(library)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def _validate_samples(samples):
    samples = np.asarray(samples)
    if samples.dtype != np.float32 or samples.ndim != 3 or not samples.size:
        raise ValueError("Nonempty three-dimensional float32 samples required")
    if max(samples.shape) > 4096 or samples.size > 16777216 or not np.isfinite(samples).all():
        raise ValueError("Finite bounded field required")
    return samples


def _validate_meta(origin, pitch, leaf_samples):
    origin = np.asarray(origin, dtype=np.float64)
    if origin.shape != (3,) or not np.isfinite(origin).all():
        raise ValueError("Finite three-coordinate origin required")
    if isinstance(pitch, (bool, np.bool_)) or not isinstance(pitch, Real):
        raise ValueError("Positive finite scalar pitch required")
    try:
        pitch = float(pitch)
    except (ValueError, TypeError):
        raise ValueError("Positive finite scalar pitch required") from None
    if not np.isfinite(pitch) or pitch <= 0:
        raise ValueError("Positive finite scalar pitch required")
    if isinstance(leaf_samples, (bool, np.bool_)):
        raise ValueError("Integer leaf size required")
    try:
        leaf_samples = operator.index(leaf_samples)
    except TypeError:
        raise ValueError("Integer leaf size required") from None
    if not 8 <= leaf_samples <= 4096:
        raise ValueError("Leaf size outside bounded contract")
    return origin, pitch, leaf_samples


def _take(L, handle):
    try:
        nodes = np.empty(L.adaptive_nodes(handle), dtype=NODE)
        payload = np.empty(L.adaptive_samples(handle), dtype=np.float32)
        if L.adaptive_copy(handle, nodes.ctypes.data, len(nodes), payload.ctypes.data, len(payload)):
            raise RuntimeError("Native packing copy failed")
    finally:
        L.adaptive_free(handle)
    return nodes, payload


class AdaptiveSampleBlocks:
    """Lossless adaptive blocks on the original fine grid, packed on the GPU
    (src/field_engine/adaptive_sample_blocks_v1.py:140-230)."""

    def __init__(self, samples, origin, pitch, *, leaf_samples=512, library=None):
        samples = _validate_samples(samples)
        origin, pitch, leaf_samples = _validate_meta(origin, pitch, leaf_samples)
        if sys.byteorder != "little":
            raise ValueError("Little-endian host required")
        L = _bind(library)
        array = np.ascontiguousarray(samples)
        shape = np.array(array.shape, dtype=np.int32)
        handle = L.adaptive_pack(array.ctypes.data, shape.ctypes.data, leaf_samples)
        if not handle:
            raise ValueError("Native packing failed")
        self._init(*_take(L, handle), origin, pitch, array.shape, library)

    def _init(self, nodes, payload, origin, pitch, shape, library):
        self.nodes = nodes
        self.payload = payload
        self.origin = origin.copy()
        self.pitch = pitch
        self.shape = tuple(int(s) for s in shape)
        self._library = library
        for value in (self.nodes, self.payload, self.origin):
            value.flags.writeable = False

    @classmethod
    def from_device(cls, samples, origin, pitch, *, leaf_samples=512, library=None):
        """Pack a float32 (nx, ny, nz) CUDA tensor without a host round trip of the dense field."""
        import torch
        origin, pitch, leaf_samples = _validate_meta(origin, pitch, leaf_samples)
        if samples.dtype != torch.float32 or samples.dim() != 3 or not samples.is_cuda or not samples.numel():
            raise ValueError("Nonempty three-dimensional float32 CUDA samples required")
        if max(samples.shape) > 4096 or samples.numel() > 16777216:
            raise ValueError("Finite bounded field required")
        L = _bind(library)
        s = samples.contiguous()
        shape = np.array(s.shape, dtype=np.int32)
        handle = L.fb_pack_device(s.data_ptr(), shape.ctypes.data, leaf_samples, _lib.stream_handle())
        if not handle:
            raise ValueError("Native packing failed (non-finite samples or device failure)")
        obj = cls.__new__(cls)
        obj._init(*_take(L, handle), origin, pitch, s.shape, library)
        return obj

    @property
    def storage_bytes(self):
        # origin, pitch and dimensions as well as every node and sample (adaptive_sample_blocks_v1.py:177-180)
        return self.nodes.nbytes + self.payload.nbytes + self.origin.nbytes + 8 + 3 * 8

    def samples_at(self, indices):
        """Exact stored samples at integer index triples (adaptive_sample_blocks_v1.py:182-207)."""
        indices = np.asarray(indices)
        if indices.ndim != 2 or indices.shape[1] != 3 or not np.issubdtype(indices.dtype, np.integer):
            raise ValueError("Integer index triples required")
        if np.any(indices < 0) or np.any(indices >= np.array(self.shape)):
            raise ValueError("Sample index outside field")
        idx = np.ascontiguousarray(indices, dtype=np.int64)
        out = np.empty(len(idx), dtype=np.float32)
        if len(idx):
            L = _bind(self._library)
            st = L.fb_packed_samples_at(self.nodes.ctypes.data, len(self.nodes), self.payload.ctypes.data,
                                        len(self.payload), idx.ctypes.data, len(idx), out.ctypes.data)
            _lib.check(st, "samples_at")
        return out

    def query(self, points):
        """float32 trilinear values on the fine grid (adaptive_sample_blocks_v1.py:209-230)."""
        import torch
        points = np.asarray(points, dtype=np.float64)
        if points.ndim != 2 or points.shape[1] != 3 or not np.isfinite(points).all():
            raise ValueError("Finite point triples required")
        with np.errstate(over="ignore", invalid="ignore"):
            coordinates = (points - self.origin) / self.pitch
        if not np.isfinite(coordinates).all():
            raise ValueError("Query exceeds finite grid-coordinate range")
        out = np.empty(len(points), dtype=np.float32)
        if not len(points):
            return out
        L = _bind(self._library)
        dev = torch.device("cuda")
        nodes = torch.from_numpy(self.nodes.view(np.uint8).copy()).to(dev)
        payload = torch.from_numpy(np.array(self.payload)).to(dev)
        pts = torch.from_numpy(np.ascontiguousarray(points)).to(dev)
        res = torch.empty(len(points), dtype=torch.float32, device=dev)
        shape = np.array(self.shape, dtype=np.int32)
        st = L.fb_packed_query_device(nodes.data_ptr(), payload.data_ptr(), shape.ctypes.data,
                                      self.origin.ctypes.data, self.pitch, pts.data_ptr(), len(points),
                                      res.data_ptr(), _lib.stream_handle())
        _lib.check(st, "query")
        out[:] = res.cpu().numpy()
        return out


class NativeAdaptiveBlocks(AdaptiveSampleBlocks):
    """The reference's native-packing class name (adaptive_pack_native_v1.py:249-299); ``library``
    names the CUDA library (default: the in-tree build)."""

    def __init__(self, samples, origin, pitch, *, library=None, leaf_samples=512):
        super().__init__(samples, origin, pitch, leaf_samples=leaf_samples, library=library)


def _reference(value, number, nfields, used):
    if isinstance(value, (bool, np.bool_)):
        raise ValueError("Integer reference required")
    try:
        index = operator.index(value)
    except TypeError:
        raise ValueError("Integer reference required") from None
    if not 0 <= index < nfields + number:
        raise ValueError("Reference must name an input or earlier instruction")
    if index < nfields:
        used.add(index)
    return index


def evaluate(fields, instructions, *, batch_library=None, pack_library=None):
    """Ordered CSG in one GPU batch, then exact packing (field_csg_batch_v1.py:18-79)."""
    fields, instructions = tuple(fields), tuple(instructions)
    if not 1 <= len(fields) <= 256 or not 1 <= len(instructions) <= 1024:
        raise ValueError("Bounded nonempty inputs and instructions required")
    if any(not isinstance(f, AdaptiveSampleBlocks) for f in fields):
        raise ValueError("Adaptive block operands required")
    first = fields[0]
    if any(f.shape != first.shape or f.pitch != first.pitch or not np.array_equal(f.origin, first.origin)
           for f in fields):
        raise ValueError("Operands must share the exact sampling grid")
    program = []
    used = set()
    for number, instruction in enumerate(instructions):
        if not isinstance(instruction, (tuple, list)) or len(instruction) != 3:
            raise ValueError("Three-item instruction required")
        operation, left, right = instruction
        if operation not in ("union", "difference", "offset"):
            raise ValueError("Unknown operation")
        left = _reference(left, number, len(fields), used)
        if operation == "offset":
            if isinstance(right, (bool, np.bool_)) or not isinstance(right, Real) or not np.isfinite(right):
                raise ValueError("Finite real offset required")
            right = float(right)
        else:
            right = _reference(right, number, len(fields), used)
        program.append((operation, left, right))
    if sys.byteorder != "little":
        raise ValueError("Little-endian host required")
    encoded = np.zeros(len(program), dtype=CSG_INSN)
    for i, (op, left, right) in enumerate(program):
        encoded[i]["op"] = {"union": 0, "difference": 1, "offset": 2}[op]
        encoded[i]["left"] = left
        encoded[i]["offset" if op == "offset" else "right"] = right
    L = _bind(batch_library)
    pointers = (ct.c_void_p * len(fields))(*(f.nodes.ctypes.data for f in fields))
    payloads = (ct.c_void_p * len(fields))(*(f.payload.ctypes.data for f in fields))
    counts = np.array([len(f.nodes) for f in fields], dtype=np.int64)
    lengths = np.array([len(f.payload) for f in fields], dtype=np.int64)
    shape = np.array(first.shape, dtype=np.int32)
    output = np.empty(first.shape, dtype=np.float32)
    code = L.csg_execute(pointers, counts.ctypes.data, payloads, lengths.ctypes.data, len(fields), shape.ctypes.data,
                         encoded.ctypes.data, len(encoded), output.ctypes.data)
    if code:
        raise ValueError(f"Native CSG validation failed: {code}")
    return NativeAdaptiveBlocks(output, first.origin, first.pitch, library=pack_library)


def compose(left, right=None, *, operation="union", distance=0.):
    """One aligned CSG operation with lossless output packing (field_csg_blocks_v1.py:12-43)."""
    if not isinstance(left, AdaptiveSampleBlocks):
        raise ValueError("Adaptive block operand required")
    if operation not in ("union", "difference", "offset"):
        raise ValueError("Unknown field operation")
    if operation == "offset":
        if right is not None or isinstance(distance, (bool, np.bool_)) or not isinstance(distance, Real) \
                or not np.isfinite(distance):
            raise ValueError("Finite real offset and no second operand required")
        return _compose_native(left, None, [("offset", 0, float(distance))])
    if not isinstance(distance, Real) or isinstance(distance, (bool, np.bool_)) or distance != 0:
        raise ValueError("Offset is only valid for the offset operation")
    if not isinstance(right, AdaptiveSampleBlocks):
        raise ValueError("Second adaptive block operand required")
    if left.shape != right.shape or left.pitch != right.pitch or not np.array_equal(left.origin, right.origin):
        raise ValueError("CSG operands must share the exact sampling grid")
    return _compose_native(left, right, [(operation, 0, 1)])


def _compose_native(left, right, program):
    """One instruction through csg_execute.  The operands are well-formed packed fields, so the only
    input-dependent failure is a non-finite result (status 4), which the reference reports as the
    float32 range error (field_csg_blocks_v1.py:40-41); any other status is a native failure."""
    try:
        return evaluate([left] if right is None else [left, right], program)
    except ValueError as e:
        if str(e) == "Native CSG validation failed: 4":
            raise ValueError("Operation exceeds finite float32 range") from None
        if str(e).startswith("Native CSG validation failed"):
            raise RuntimeError(f"compose: native failure ({e})") from None
        raise
