"""The allocation-free EDT entry point, called through the C ABI (GPU).

Callers that cannot allocate device memory -- a host that owns every device byte through its own
allocator, or a loop that must never meet the implicit synchronisation of cudaMalloc -- use
fb_edt_squared_device_noalloc, whose scratch is a fixed array inside the library.  This file is
collected last so that a failure here never hides another test; it must pass alone in a fresh
process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry_points():
    import field_b200._lib as L
    lib = L.lib()
    fn = lib.fb_edt_squared_device_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn


def test_no_alloc_edt_matches_allocating_entry_point_twice():
    import torch
    import field_b200._lib as L
    lib, noalloc = _entry_points()
    stream = L.stream_handle()
    # two calls in a row with different grids and site conventions: the second call reuses the
    # fixed scratch the first one left behind
    cases = [((64, 80, 96), 0, 0.3), ((101, 97, 103), 1, 0.05)]
    for (shape, sites_nonzero, fill) in cases:
        g = torch.Generator(device="cuda").manual_seed(sum(shape))
        mask = (torch.rand(shape, device="cuda", generator=g) < fill).to(torch.uint8)
        ref = torch.empty(shape, dtype=torch.int32, device="cuda")
        scratch = torch.empty(int(lib.fb_edt_scratch_bytes(*shape, 0)), dtype=torch.uint8, device="cuda")
        assert lib.fb_edt_squared_device(mask.data_ptr(), *shape, sites_nonzero, ref.data_ptr(), scratch.data_ptr(),
                                         scratch.numel(), stream) == 0
        out = torch.full(shape, -1, dtype=torch.int32, device="cuda")
        assert noalloc(mask.data_ptr(), *shape, sites_nonzero, out.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        assert torch.equal(out, ref)  # integer distances: exact


def test_no_alloc_edt_at_exactly_its_limit_both_site_conventions():
    """A 512 x 512 x 4 grid fills the fixed array exactly (2^20 voxels, where the bit words'
    bound nx*ny*ceil(nz/32) is tightest); two calls in a row on the same grid with opposite site
    conventions, bit-exact against the allocating entry point and against the CPU oracle."""
    import torch
    import oracle
    import field_b200._lib as L
    lib, noalloc = _entry_points()
    stream = L.stream_handle()
    shape = (512, 512, 4)
    assert shape[0] * shape[1] * shape[2] == 1 << 20
    rng = np.random.default_rng(20)
    host = (rng.random(shape) < 0.02).astype(np.uint8)
    mask = torch.from_numpy(host).cuda()
    scratch = torch.empty(int(lib.fb_edt_scratch_bytes(*shape, 0)), dtype=torch.uint8, device="cuda")
    for sites_nonzero in (1, 0):
        ref = torch.empty(shape, dtype=torch.int32, device="cuda")
        assert lib.fb_edt_squared_device(mask.data_ptr(), *shape, sites_nonzero, ref.data_ptr(), scratch.data_ptr(),
                                         scratch.numel(), stream) == 0
        out = torch.full(shape, -1, dtype=torch.int32, device="cuda")
        assert noalloc(mask.data_ptr(), *shape, sites_nonzero, out.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        # the oracle measures to the zero bytes of its argument
        binary = (1 - host) if sites_nonzero else host
        assert (out.cpu().numpy() == oracle.edt_squared(binary)).all()


def test_no_alloc_edt_rejects_grids_beyond_its_fixed_scratch():
    import torch
    import field_b200._lib as L
    lib, noalloc = _entry_points()
    limit = ctypes.c_int64(0)
    assert lib.fb_edt_noalloc_capacity(ctypes.byref(limit)) > 0
    assert limit.value == 1 << 20
    shape = (128, 128, 65)  # 1064960 voxels > 2^20
    mask = torch.zeros(shape, dtype=torch.uint8, device="cuda")
    out = torch.full(shape, -1, dtype=torch.int32, device="cuda")
    assert noalloc(mask.data_ptr(), *shape, 0, out.data_ptr(), L.stream_handle()) == 7
    # an axis above 512 is beyond the array too, although the voxel count is small
    long_axis = torch.zeros((600, 4, 4), dtype=torch.uint8, device="cuda")
    long_out = torch.full((600, 4, 4), -1, dtype=torch.int32, device="cuda")
    assert noalloc(long_axis.data_ptr(), 600, 4, 4, 0, long_out.data_ptr(), L.stream_handle()) == 7
    # a null pointer or an empty axis is invalid input
    assert noalloc(None, 8, 8, 8, 0, out.data_ptr(), L.stream_handle()) == 1
    assert noalloc(mask.data_ptr(), 0, 8, 8, 0, out.data_ptr(), L.stream_handle()) == 1
    torch.cuda.synchronize()
    assert int(out.min()) == -1 and int(out.max()) == -1
    assert int(long_out.min()) == -1 and int(long_out.max()) == -1
