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


def _events_ms(fn, reps=5, warmup=2):
    import torch
    s = torch.cuda.current_stream()
    for _ in range(warmup):
        fn(s.cuda_stream)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn(s.cuda_stream)
        e1.record(s)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def test_full_size_edt_equals_the_reference_cuda_kernels():
    """512^3 obstacle grid (2000 boxes, ~8 % fill): the reference's own linear and paired CUDA
    envelope kernels, launched on device buffers, against fb_edt_squared_device and
    fb_edt_pair_device -- identical bits, and both timed on the device."""
    import torch
    import field_b200._lib as L
    import field_b200.recipes as R
    lin = _load("libref_edt_linear_dev.so")
    pair = _load("libref_edt_pair_dev.so")
    P, I, D = ct.c_void_p, ct.c_int, ct.c_double
    lin.ref_edt_linear_device.argtypes = [P, I, I, I, P, P, ct.POINTER(ct.c_void_p), P]
    lin.ref_edt_linear_device.restype = I
    pair.ref_edt_pair_device.argtypes = [P, I, I, I, D, P, P, P, ct.POINTER(ct.c_void_p), P]
    pair.ref_edt_pair_device.restype = I
    ours = L.lib()

    n = 512
    size = n ** 3
    mask_np = R.obstacle_grid(seed=2, n=n, n_boxes=2000, fill=0.08)
    dev = torch.device("cuda", 0)
    mask = torch.from_numpy(mask_np).to(dev)
    inverted = (1 - mask).contiguous()  # the reference's single-polarity sites are the zero voxels
    a = torch.empty(2 * size, dtype=torch.int32, device=dev)
    b = torch.empty(2 * size, dtype=torch.int32, device=dev)
    dist_ref = torch.empty(size, dtype=torch.float32, device=dev)
    res = ct.c_void_p()

    # single polarity: squared distance to the obstacles
    def ref_lin(stream):
        assert lin.ref_edt_linear_device(inverted.data_ptr(), n, n, n, a.data_ptr(), b.data_ptr(), ct.byref(res),
                                         stream) == 0
    sb = ours.fb_edt_scratch_bytes(n, n, n, 1)
    scratch = torch.empty(sb, dtype=torch.uint8, device=dev)
    out = torch.empty(size, dtype=torch.int32, device=dev)

    def ours_sq(stream):
        assert ours.fb_edt_squared_device(mask.data_ptr(), n, n, n, 1, out.data_ptr(), scratch.data_ptr(), sb,
                                          stream) == 0
    t_ref = _events_ms(ref_lin, reps=3, warmup=1)
    ref_out = a if res.value == a.data_ptr() else b
    ref_sq = ref_out[:size].clone()
    t_ours = _events_ms(ours_sq)
    torch.cuda.synchronize()
    assert torch.equal(ref_sq, out)
    print(f"\nsquared EDT 512^3 obstacles: reference linear kernels {t_ref:.2f} ms, field_b200 {t_ours:.3f} ms "
          f"({t_ref / t_ours:.0f}x)")

    # paired: signed float32 and both squared polarities
    pitch = 1.0 / 512

    def ref_pair(stream):
        assert pair.ref_edt_pair_device(mask.data_ptr(), n, n, n, pitch, a.data_ptr(), b.data_ptr(),
                                        dist_ref.data_ptr(), ct.byref(res), stream) == 0
    sb2 = ours.fb_edt_scratch_bytes(n, n, n, 1 + 1)
    scratch2 = torch.empty(sb2, dtype=torch.uint8, device=dev)
    sd = torch.empty(size, dtype=torch.float32, device=dev)
    sq = torch.empty(2 * size, dtype=torch.int32, device=dev)

    def ours_pair(stream):
        assert ours.fb_edt_pair_device(mask.data_ptr(), n, n, n, pitch, sd.data_ptr(), sq.data_ptr(),
                                       scratch2.data_ptr(), sb2, stream) == 0
    t_ref = _events_ms(ref_pair, reps=3, warmup=1)
    ref_out = a if res.value == a.data_ptr() else b
    t_ours = _events_ms(ours_pair)
    torch.cuda.synchronize()
    assert torch.equal(ref_out, sq)
    assert torch.equal(dist_ref.view(torch.int32), sd.view(torch.int32))
    print(f"paired signed EDT 512^3 obstacles: reference persistent-pair kernels {t_ref:.2f} ms, "
          f"field_b200 {t_ours:.3f} ms ({t_ref / t_ours:.0f}x)")
