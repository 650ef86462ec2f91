"""Packed adaptive block tree of a dense SDF, built and sampled on the GPU.

Drop-in for src/field_engine/field_adaptive_blocks_v1.py:

* ``build(wp, dense, pitch, device=...)`` -> ``(AdaptiveBlocks, histogram)`` -- field_adaptive_blocks_v1.py:113-147.
  ``wp`` is accepted and ignored (there is no Warp here).
* ``AdaptiveBlocks`` with the reference's fields (shape, pitch, root_shape, root_count, node_count,
  packed, branch_prefix, value_prefix, values) and methods ``kinds``, ``rank_before``, ``sample``,
  ``stored_bytes``, ``fingerprint`` (field_adaptive_blocks_v1.py:20-98); ``sample`` runs on the GPU.

The format: one 2-bit code per node -- 0 a leaf outside the surface (its value is
+sqrt(3) * side * pitch), 1 inside (-sqrt(3) * side * pitch), 2 a branch, 3 a side-1 leaf holding a
dense sample -- packed four per byte in breadth-first order; the children of the b-th branch are
nodes root_count + 8b ... + 7, so ranks replace pointers; rank checkpoints every 64 bytes (256
nodes) for codes 2 and 3.  The tree is decided by the dense block classification at sides 8, 4, 2
and 1 (the 8-corner rule with the full block-diagonal margin of ``fb_dense_classify_device``),
evaluated for the tree's nodes only.
"""
from __future__ import annotations

import hashlib
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib

SIDES = (8, 4, 2, 1)


def _check(st, what):
    _lib.check(st, what)


@dataclass
class AdaptiveBlocks:
    shape: tuple
    pitch: float
    root_shape: tuple
    root_count: int
    node_count: int
    packed: np.ndarray
    branch_prefix: np.ndarray
    value_prefix: np.ndarray
    values: np.ndarray
    device: str = "cuda"
    _dev: dict = field(default=None, repr=False, compare=False)

    def kinds(self, nodes):
        """2-bit codes of node indices."""
        nodes = np.asarray(nodes, dtype=np.int64)
        return (self.packed[nodes // 4] >> (2 * (nodes % 4))) & 3

    def rank_before(self, nodes, code):
        """Number of nodes of `code` (2 or 3) before each node: its 256-node checkpoint plus the codes
        counted in the bytes between (host-side, for inspection; sampling ranks on the GPU)."""
        nodes = np.asarray(nodes, dtype=np.int64)
        prefix = self.branch_prefix if code == 2 else self.value_prefix
        codes = (self.packed[:, None] >> np.array([0, 2, 4, 6], np.uint8)) & 3
        running = np.concatenate(([0], np.cumsum((codes.reshape(-1) == code).astype(np.int64))))
        group = nodes // 256
        return prefix[group].astype(np.int64) + running[nodes] - running[group * 256]

    @classmethod
    def from_device(cls, t, pitch, *, host=True):
        """The tree of a build_device result, sampling from its device arrays; with host=False the
        host arrays stay empty (no copies) and only sample / sample_device are meaningful."""
        import torch
        dev = t["packed"].device
        if host:
            arrays = (t["packed"][:t["nbytes"]].cpu().numpy(), t["branch"].cpu().numpy(), t["value"].cpu().numpy(),
                      t["values"].cpu().numpy().astype(np.float32))
        else:
            arrays = (np.zeros(0, np.uint8), np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
        tree = cls(tuple(int(v) for v in t["shape"]), float(pitch), tuple(t["root_shape"]), t["root_count"],
                   t["node_count"], *arrays, device=str(dev))
        n_values = int(t["values"].numel())
        tree._dev = dict(packed=t["packed"], branch=t["branch"], value=t["value"], n_values=n_values,
                         values=t["values"] if n_values else torch.zeros(1, dtype=torch.float32, device=dev),
                         status=torch.zeros(1, dtype=torch.int32, device=dev))
        tree._rank_words()
        return tree

    def _rank_words(self):
        """The sampler's per-word rank tables (nodes of code 2 / 3 before each 16-node word): a rank
        is then one table read and one popcount instead of a walk from the 64-byte checkpoint."""
        import torch
        d = self._dev
        nwords = (self.node_count + 15) // 16
        dev = d["packed"].device
        d["bword"] = torch.empty(nwords + 1, dtype=torch.int32, device=dev)
        d["vword"] = torch.empty(nwords + 1, dtype=torch.int32, device=dev)
        lib = _lib.lib()
        scratch = torch.empty(int(lib.fb_tree_rank_words_scratch_bytes(self.node_count)), dtype=torch.uint8, device=dev)
        _check(lib.fb_tree_rank_words_device(d["packed"].data_ptr(), self.node_count, d["bword"].data_ptr(),
                                             d["vword"].data_ptr(), scratch.data_ptr(), scratch.numel(),
                                             _lib.stream_handle()), "tree rank words")

    def _device(self):
        import torch
        if self._dev is None:
            dev = torch.device(self.device)
            nb = len(self.packed)
            packed = torch.zeros((nb + 3) // 4 * 4, dtype=torch.uint8, device=dev)
            packed[:nb] = torch.from_numpy(self.packed).to(dev)
            n_values = len(self.values)
            self._dev = dict(packed=packed, n_values=n_values,
                             branch=torch.from_numpy(self.branch_prefix.astype(np.int32)).to(dev),
                             value=torch.from_numpy(self.value_prefix.astype(np.int32)).to(dev),
                             values=torch.from_numpy(np.ascontiguousarray(self.values, np.float32)).to(dev)
                             if n_values else torch.zeros(1, dtype=torch.float32, device=dev),
                             status=torch.zeros(1, dtype=torch.int32, device=dev))
            self._rank_words()
        return self._dev

    def sample_device(self, ijk, *, stream=None):
        """float32 values at an int64 (N, 3) CUDA tensor of grid indices (no host round trip;
        indices must lie in the grid -- outside ones read NaN and set the status word)."""
        import torch
        d = self._device()
        ijk = ijk.to(device=d["packed"].device, dtype=torch.int64).contiguous()
        out = torch.empty(ijk.shape[0], dtype=torch.float32, device=ijk.device)
        _check(_lib.lib().fb_tree_sample_device(
            d["packed"].data_ptr(), self.node_count, d["branch"].data_ptr(), d["value"].data_ptr(),
            d["bword"].data_ptr(), d["vword"].data_ptr(),
            d["values"].data_ptr() if d["n_values"] else None, d["n_values"], self.root_count,
            *self.root_shape, *self.shape, float(self.pitch), ijk.data_ptr(), ijk.shape[0], out.data_ptr(),
            d["status"].data_ptr(), _lib.stream_handle(stream)), "tree sample")
        return out

    def sample(self, indices):
        """float32 values at integer grid coordinates [N, 3] (field_adaptive_blocks_v1.py:53-82)."""
        import torch
        ijk = np.asarray(indices, dtype=np.int64)
        if ijk.ndim != 2 or ijk.shape[1] != 3 or np.any(ijk < 0) or np.any(ijk >= self.shape):
            raise ValueError("Expected in-domain integer grid coordinates[N,3]")
        d = self._device()
        d["status"].zero_()
        out = self.sample_device(torch.from_numpy(np.ascontiguousarray(ijk)).to(d["packed"].device))
        status = int(d["status"].item())
        if status & 2:
            raise RuntimeError("Invalid tree depth")
        if status:
            raise RuntimeError(f"tree sample failed (status {status})")
        return out.cpu().numpy()

    def stored_bytes(self):
        """Bytes of the stored arrays plus an 80-byte numeric header (field_adaptive_blocks_v1.py:84-86)."""
        return 80 + sum(a.nbytes for a in (self.packed, self.branch_prefix, self.value_prefix, self.values))

    def fingerprint(self):
        """SHA-256 over the header numbers and the stored arrays (field_adaptive_blocks_v1.py:88-95)."""
        h = hashlib.sha256()
        h.update(np.array([*self.shape, *self.root_shape, self.root_count, self.node_count], np.int64).tobytes())
        h.update(np.float64(self.pitch).tobytes())
        for a in (self.packed, self.branch_prefix, self.value_prefix, self.values):
            h.update(a.tobytes())
        return h.hexdigest()


def build_device(dense, pitch, *, stream=None):
    """Device arrays of the tree of a float32 (nx, ny, nz) CUDA tensor: dict with the padded packed
    codes, the two checkpoint arrays, the values, node / root counts and each level's node count."""
    import torch
    lib = _lib.lib()
    dev = dense.device
    nx, ny, nz = (int(v) for v in dense.shape)
    dense = dense.to(torch.float32).contiguous()
    sh = _lib.stream_handle(stream)
    root_shape = tuple(-(-v // 8) for v in (nx, ny, nz))
    n = root_shape[0] * root_shape[1] * root_shape[2]
    coords = None
    level_codes, level_sizes = [], []
    values = torch.empty(0, dtype=torch.float32, device=dev)
    total = torch.empty(1, dtype=torch.int32, device=dev)
    for side in SIDES:
        margin = float(np.float32(math.sqrt(3.0) * side * pitch))  # the dense classification's margin
        codes = torch.empty(n, dtype=torch.uint8, device=dev)
        rank = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        scratch = torch.empty(int(lib.fb_tree_scan_bytes(n)), dtype=torch.uint8, device=dev)
        _check(lib.fb_tree_codes_device(dense.data_ptr(), nx, ny, nz, side, margin,
                                        coords.data_ptr() if coords is not None else None, *root_shape, n,
                                        codes.data_ptr(), rank.data_ptr(), total.data_ptr(), scratch.data_ptr(),
                                        scratch.numel(), sh), "tree codes")
        ranked = int(total.item())  # branches (or value leaves at side 1): sizes the next arrays
        level_codes.append(codes)
        level_sizes.append(n)
        if side > 1:
            child = torch.empty((max(ranked, 1) * 8, 3), dtype=torch.int32, device=dev)
            _check(lib.fb_tree_expand_device(codes.data_ptr(), rank.data_ptr(),
                                             coords.data_ptr() if coords is not None else None, *root_shape, n, side,
                                             child.data_ptr(), sh), "tree expand")
            coords = child[:ranked * 8]
            n = ranked * 8
        else:
            values = torch.empty(max(ranked, 1), dtype=torch.float32, device=dev)
            _check(lib.fb_tree_values_device(dense.data_ptr(), nx, ny, nz, codes.data_ptr(), rank.data_ptr(),
                                             coords.data_ptr(), n, values.data_ptr(), sh), "tree values")
            values = values[:ranked]
        if n == 0 and side > 1:  # no branch: the deeper levels are empty
            for _ in SIDES[SIDES.index(side) + 1:]:
                level_codes.append(torch.empty(0, dtype=torch.uint8, device=dev))
                level_sizes.append(0)
            break
    all_codes = torch.cat(level_codes)
    node_count = int(all_codes.numel())
    nbytes = (node_count + 3) // 4
    packed = torch.empty((nbytes + 3) // 4 * 4, dtype=torch.uint8, device=dev)
    nprefix = nbytes // 64 + 1
    branch = torch.empty(nprefix, dtype=torch.int32, device=dev)
    value = torch.empty(nprefix, dtype=torch.int32, device=dev)
    scratch = torch.empty(int(lib.fb_tree_pack_scratch_bytes(node_count)), dtype=torch.uint8, device=dev)
    _check(lib.fb_tree_pack_device(all_codes.data_ptr(), node_count, packed.data_ptr(), branch.data_ptr(),
                                   value.data_ptr(), scratch.data_ptr(), scratch.numel(), sh), "tree pack")
    return dict(packed=packed, nbytes=nbytes, branch=branch, value=value, values=values, node_count=node_count,
                root_shape=root_shape, root_count=root_shape[0] * root_shape[1] * root_shape[2],
                level_sizes=level_sizes, shape=(nx, ny, nz))


def _histogram(packed, level_sizes):
    """Leaf counts per side and code, labelled as the reference labels them."""
    codes = ((packed[:, None] >> np.array([0, 2, 4, 6], np.uint8)) & 3).reshape(-1)
    hist, at = {}, 0
    for side, size in zip(SIDES, level_sizes):
        counts = np.bincount(codes[at:at + size], minlength=4)
        for code in (0, 1, 3):
            if counts[code]:
                hist[f"side{side}_kind{code}"] = int(counts[code])
        at += size
    return dict(sorted(hist.items()))


def build(wp, dense, pitch, *, device="cuda"):
    """(AdaptiveBlocks, leaf histogram) of a dense float32 SDF (field_adaptive_blocks_v1.py:113-147),
    built on the GPU; ``wp`` is ignored."""
    import torch
    d = np.ascontiguousarray(dense, dtype=np.float32)
    if d.ndim != 3:
        raise ValueError("dense field must be 3-D")
    t = build_device(torch.from_numpy(d).to(device), float(pitch))
    tree = AdaptiveBlocks.from_device(t, pitch)
    return tree, _histogram(tree.packed, t["level_sizes"])
