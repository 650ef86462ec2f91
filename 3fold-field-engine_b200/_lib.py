"""Loader of the CUDA library and the ctypes signatures of its C ABI (include/field_b200.h).

There is no fallback: ``lib()`` raises ``RuntimeError`` when ``libfield_b200.so`` is missing or no
CUDA device is visible, so every product call fails loudly instead of computing elsewhere.
"""
from __future__ import annotations

import ctypes as ct
import threading
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libfield_b200.so"

_lock = threading.Lock()
_LIBS: dict[str, ct.CDLL] = {}

P, I, I64, D, F, U64 = ct.c_void_p, ct.c_int, ct.c_int64, ct.c_double, ct.c_float, ct.c_uint64

# name -> (restype, argtypes)
SIGNATURES = {
    # runtime
    "fb_abi_version": (I, []),
    "fb_device_arch": (I, []),
    # EDT, device pointers
    "fb_edt_scratch_bytes": (I64, [I, I, I, I]),
    "fb_edt_squared_device": (I, [P, I, I, I, I, P, P, I64, P]),
    "fb_edt_pair_device": (I, [P, I, I, I, D, P, P, P, I64, P]),
    "fb_edt_validate_device": (I, [P, I, I, I, P, I64, P]),
    "fb_edt_squared_device_noalloc": (I, [P, I, I, I, I, P, P]),
    "fb_edt_noalloc_capacity": (I64, [P]),
    # EDT, host pointers (reference names)
    "edt_squared_large": (I, [P, I, I, I, P]),
    "edt_squared": (I, [P, I, I, I, P]),
    "edt_pair_create": (P, [I, I, I]),
    "edt_pair_query": (I, [P, P, D, P, P]),
    "edt_pair_destroy": (None, [P]),
    # field build
    "fb_field_scratch_bytes": (I64, [P, I, I]),
    "fb_field_classify_device": (I, [P, P, I, P, I, I, P, P, P, P, P, I64, P]),
    "fb_field_leaf_device": (I, [P, P, I, P, I, I, P, P, P, P, I64, P, I64, P]),
    "fb_field_build_device": (I, [P, P, I, P, I, I, P, P, P, P, P, I64, P, I64, P]),
    "fb_field_compact_error": (I, [P, I, I, P, P]),
    "fb_compact_timeout_probe": (I, [P, I64, P, P, P, I64, I64, P]),
    "fb_sqrt_sum_probe": (I, [P, P, I64, P]),
    "fb_quotient_probe": (I, [P, P, P, I64, P]),
    # batched builds
    "fb_batch_create": (P, [P, I, P]),
    "fb_batch_build_device": (I, [P, P, I64, I, P]),
    "fb_batch_build_timed_device": (I, [P, P, I64, I, P, P, P]),
    "fb_batch_outputs": (I, [P, P, P]),
    "fb_batch_occupancy_device": (I, [P, P, P]),
    "fb_batch_launches": (I, [P]),
    "fb_batch_status": (I, [P, P]),
    "fb_batch_destroy": (None, [P]),
    "fb_dense_scratch_bytes": (I64, [I64, I64, I64, I]),
    "fb_dense_classify_device": (I, [P, I64, I64, I64, I, F, P, P, P, P, P, I64, P, I64, P]),
    "fb_field_reconstruct_device": (I, [P, P, I64, P, I64, I64, I64, I, F, P, P, P]),
    "fb_checksum_i64_device": (I, [P, I64, D, P, P]),
    "fb_sum_i32_device": (I, [P, I64, P, P]),
    # mesh -> field stage (host pointers)
    "meshsdf_field_cpu": (I, [P, I64, P, I64, D, D, D, D, D, D, I64, I64, I64, I, I, P, P, P, P, P]),
    # packed adaptive block tree
    "fb_tree_scan_bytes": (I64, [I64]),
    "fb_tree_codes_device": (I, [P, I64, I64, I64, I, F, P, I64, I64, I64, I64, P, P, P, P, I64, P]),
    "fb_tree_expand_device": (I, [P, P, P, I64, I64, I64, I64, I, P, P]),
    "fb_tree_values_device": (I, [P, I64, I64, I64, P, P, P, I64, P, P]),
    "fb_tree_pack_scratch_bytes": (I64, [I64]),
    "fb_tree_pack_device": (I, [P, I64, P, P, P, P, I64, P]),
    "fb_tree_rank_words_scratch_bytes": (I64, [I64]),
    "fb_tree_rank_words_device": (I, [P, I64, P, P, P, I64, P]),
    "fb_tree_sample_device": (I, [P, I64, P, P, P, P, P, I64, I64, I64, I64, I64, I64, I64, I64, D, P, I64, P, P, P]),
    "fb_field_occupancy_device": (I, [P, P, P, P, I64, I64, I64, I64, I, P, P, P]),
    # export: marching cubes on the resident leaves
    "fb_mc_words": (I64, [I]),
    "fb_mc_scan_words": (I64, [I64]),
    "fb_mc_count_device": (I, [P, P, I64, P, I64, I64, I64, I, D, D, D, D, D, F, P, P, P, P, P, P, P, I64, P]),
    "fb_mc_emit_device": (I, [P, P, I64, P, I64, I64, I64, I, D, D, D, D, D, F, P, P, P, P, P, P, P, P, P, P, P,
                              P]),
    "fb_mesh_components_device": (I, [P, I64, P, I64, P, P, P, P, P, P]),
    "fb_field_leaf_work_device": (I, [P, P, I, P, I, I, P, P, P, P, I64, P, I64, P, P]),
    "fb_fp32_peak_launch": (I64, [P, I, I, P]),
    "fb_sm_count_c": (I, []),
    "fb_copy_device": (I, [P, P, I64, P]),
    # queries
    "fb_query_prepare": (I, [P, I, P, P]),
    "fb_field_accel": (I, [P, I, I, P, P, P, P, P, P, P, P, P]),
    "fb_query_points_device": (I, [P, P, I, I, P, P, P, P, P, P, P, P, P, I64, I, P, I64, D, P, P, P, I64, P]),
    "fb_query_scratch_bytes": (I64, [P, I64, I]),
    "fb_multires_tiles_device": (I, [P, P, I, I, P, P, D, I, P, P, P, P, I64, P, P, P, F, P, P]),
    "fb_multires_query_device": (I, [P, D, I, P, D, P, P, P, P, P, I64, P, P, P]),
    "fb_grid_pairs_device": (I, [P, I, P, P, I64, P, P, I, P, P]),
    "fb_multires_band_device": (I, [P, D, I, P, P, P, P, P, I64, P, P, P, P, P]),
    # EDT consumers: clearance, valid mask, lattice Laplacian
    "fb_edt_mm_device": (I, [P, I64, D, P, P]),
    "fb_clearance_mask_device": (I, [P, P, I64, D, P, P]),
    "fb_lattice_scratch_bytes": (I64, [I, I, I]),
    "fb_lattice_count_device": (I, [P, I, I, I, P, P, I64, P]),
    "fb_lattice_emit_device": (I, [P, P, I, I, I, D, D, P, P, P, P, I64, P, I64, P, P, I64, P, I64, P]),
}


def _bind(L: ct.CDLL) -> ct.CDLL:
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return L


def load(path: str | Path | None = None) -> ct.CDLL:
    """The CUDA library at ``path`` (default: the in-tree build), loaded once per path."""
    p = Path(path).resolve() if path is not None else LIBRARY
    key = str(p)
    with _lock:
        if key not in _LIBS:
            if not p.exists():
                raise RuntimeError(f"CUDA library {p} is not built; run __graft_entry__.build() "
                                   "(there is no CPU fallback)")
            _LIBS[key] = _bind(ct.CDLL(key))
        return _LIBS[key]


def lib(path=None) -> ct.CDLL:
    """The CUDA library, after checking that a CUDA device is present."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("field_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    return load(path)


def stream_handle(stream=None) -> int:
    """Raw cudaStream_t of a torch stream (default: the current stream)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def check(status: int, what: str) -> None:
    if status == 1:
        raise ValueError(f"{what}: invalid input (status 1)")
    if status:
        raise RuntimeError(f"{what}: native failure (status {status})")
