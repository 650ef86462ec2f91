"""The EDT against the reference's own CUDA EDT on the same GPU, through the same host-pointer C ABI
(edt_squared_large; edt_pair_create / query / destroy): identical bits on masks within the
reference's contract (at most 2^20 voxels, 512 per axis), and both calls timed (printed with -s).
The reference libraries are compiled from its sources into oracle/_ref by oracle/Makefile."""
import ctypes as ct
import time
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


def _masks():
    rng = np.random.default_rng(17)
    out = {}
    shape = (128, 128, 64)  # 2^20 voxels, the reference's limit
    boxes = np.zeros(shape, np.uint8)
    for _ in range(120):
        c = rng.integers(0, shape)
        h = rng.integers(1, 7, size=3)
        boxes[max(c[0] - h[0], 0):c[0] + h[0], max(c[1] - h[1], 0):c[1] + h[1], max(c[2] - h[2], 0):c[2] + h[2]] = 1
    out["boxes"] = boxes
    out["random30"] = (rng.random(shape) < 0.3).astype(np.uint8)
    sparse = np.zeros((100, 90, 110), np.uint8)
    sparse[tuple(rng.integers(0, 90, size=(3, 12)))] = 1
    out["sparse"] = sparse
    return out


def _load(name):
    path = REF / name
    if not path.exists():
        pytest.skip(f"{path.name} not built (reference checkout absent when oracle/ was built)")
    return ct.CDLL(str(path))


def _bind_pair(lib):
    lib.edt_pair_create.argtypes = [ct.c_int] * 3
    lib.edt_pair_create.restype = ct.c_void_p
    lib.edt_pair_query.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_double, ct.c_void_p, ct.c_void_p]
    lib.edt_pair_query.restype = ct.c_int
    lib.edt_pair_destroy.argtypes = [ct.c_void_p]
    lib.edt_pair_destroy.restype = None
    return lib


def _best(fn, reps=5):
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best


def test_squared_edt_equals_the_reference_cuda_edt():
    import field_b200._lib as L
    ref = _load("libref_edt_large.so")
    ref.edt_squared_large.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p]
    ref.edt_squared_large.restype = ct.c_int
    ours = L.lib()
    for name, m in _masks().items():
        m = np.ascontiguousarray(m)
        a = np.empty(m.shape, np.int32)
        b = np.empty(m.shape, np.int32)
        assert ref.edt_squared_large(m.ctypes.data, *m.shape, a.ctypes.data) == 0
        assert ours.edt_squared_large(m.ctypes.data, *m.shape, b.ctypes.data) == 0
        assert np.array_equal(a, b), name
        t_ref = _best(lambda: ref.edt_squared_large(m.ctypes.data, *m.shape, a.ctypes.data))
        t_ours = _best(lambda: ours.edt_squared_large(m.ctypes.data, *m.shape, b.ctypes.data))
        print(f"edt_squared_large {name} {m.shape}: reference {t_ref * 1e3:.2f} ms, ours {t_ours * 1e3:.2f} ms "
              f"(host buffers, copies included)")


def test_paired_edt_equals_the_reference_cuda_edt():
    import field_b200._lib as L
    ref = _bind_pair(_load("libref_edt_pair.so"))
    ours = L.lib()
    for name, m in _masks().items():
        m = np.ascontiguousarray(m)
        outs = []
        times = []
        for lib in (ref, ours):
            h = lib.edt_pair_create(*m.shape)
            assert h
            try:
                sd = np.empty(m.shape, np.float32)
                sq = np.empty((2,) + m.shape, np.int32)
                assert lib.edt_pair_query(h, m.ctypes.data, 0.25, sd.ctypes.data, sq.ctypes.data) == 0
                outs.append((sd, sq))
                times.append(_best(lambda: lib.edt_pair_query(h, m.ctypes.data, 0.25, sd.ctypes.data, sq.ctypes.data)))
            finally:
                lib.edt_pair_destroy(h)
        (sd_r, sq_r), (sd_o, sq_o) = outs
        assert np.array_equal(sq_r, sq_o), name
        assert sd_r.tobytes() == sd_o.tobytes(), name
        print(f"edt_pair_query {name} {m.shape}: reference {times[0] * 1e3:.2f} ms, ours {times[1] * 1e3:.2f} ms "
              f"(host buffers, copies included)")
