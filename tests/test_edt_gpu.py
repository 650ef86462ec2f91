"""CUDA EDT parity: bit-exact against the reference's captures and the oracle (GPU)."""
import numpy as np
import pytest

import oracle
from conftest import Golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def edt():
    return Golden("edt_golden")


@pytest.fixture(scope="module")
def fe():
    import field_b200.edt as E
    return E


def test_large_squared_matches_reference_captures(edt, fe):
    native = fe.NativeEDTLarge()
    n = 0
    for name in edt.names():
        m = edt.mask(name)
        for pol, binary in enumerate((~m, m)):
            key = f"squared{pol}"
            if key in edt.meta[name]["sha256"]:
                assert edt.matches(name, key, native.squared_distance(binary)), (name, key)
                n += 1
    assert n >= 40


def test_persistent_pair_matches_reference_captures(edt, fe):
    n = 0
    for name in edt.names():
        m = edt.mask(name)
        with fe.PersistentPairEDT(m.shape) as handle:
            for p in edt.meta[name]["pitches"]:
                signed, pair = handle.query(m, p, with_squared=True)
                assert edt.matches(name, f"signed_{p!r}", signed), (name, p)
                for pol in range(2):
                    if f"squared{pol}" in edt.meta[name]["sha256"]:
                        assert edt.matches(name, f"squared{pol}", pair[pol]), (name, pol)
                n += 1
    assert n >= 80


def test_small_api_matches_integer_reference(edt, fe):
    for name in edt.names("integer/"):
        m = edt.mask(name)
        assert edt.matches(name, "squared0", fe.squared_distance(~m).astype(np.int32))
        p = edt.meta[name]["pitches"][1]
        assert edt.matches(name, f"signed_{p!r}", fe.signed_distance(m, p))


@pytest.mark.parametrize("shape", [(1, 1, 2), (3, 1, 1), (33, 17, 65), (64, 64, 64), (5, 512, 3),
                                   (512, 3, 5), (2, 3, 512), (100, 37, 31)])
@pytest.mark.parametrize("fill", [0.02, 0.5, 0.97])
def test_random_masks_against_oracle(fe, shape, fill):
    rng = np.random.default_rng(hash((shape, fill)) % 2**32)
    m = rng.random(shape) < fill
    m.flat[0] = True
    m.flat[-1] = False
    native = fe.NativeEDTLarge()
    for binary in (m, ~m):
        assert (native.squared_distance(binary) == oracle.edt_squared(binary)).all()
    with fe.PersistentPairEDT(shape) as h:
        s, pair = h.query(m, 0.37, with_squared=True)
    o, opair = oracle.edt_signed(m, 0.37, with_squared=True)
    assert (pair == opair).all() and s.tobytes() == o.tobytes()


def test_device_api_512_cube_properties(fe):
    """Full 512^3 size: zero exactly on sites, the device pair equals the single-polarity
    transforms, and sampled voxels equal an exact nearest-site search (KD-tree over all sites)."""
    import torch
    from scipy.spatial import cKDTree
    g = torch.Generator(device="cuda").manual_seed(7)
    mask = (torch.rand((512, 512, 512), device="cuda", generator=g) < 0.002).to(torch.uint8)
    sq_obst = fe.squared_distance_device(mask, sites_nonzero=True)
    assert int(sq_obst[mask.bool()].abs().max()) == 0
    assert int(sq_obst[~mask.bool()].min()) >= 1
    sd, pair = fe.signed_distance_device(mask, 0.5, with_squared=True)
    assert torch.equal(pair[0], sq_obst)
    sq_free = fe.squared_distance_device(mask, sites_nonzero=False)
    assert torch.equal(pair[1], sq_free)
    sites = np.argwhere(mask.cpu().numpy().astype(bool))
    tree = cKDTree(sites)
    rng = np.random.default_rng(1)
    probe = rng.integers(0, 512, size=(20000, 3))
    d, _ = tree.query(probe)
    expect = np.rint(d ** 2).astype(np.int64)
    got = sq_obst.cpu().numpy()[probe[:, 0], probe[:, 1], probe[:, 2]]
    assert (got == expect).all()


def test_invalid_inputs_rejected(fe):
    native = fe.NativeEDTLarge()
    for bad in [np.zeros((2, 2, 2), bool), np.ones((2, 2, 2), bool), np.zeros((513, 1, 2), bool),
                np.zeros((1, 2), bool), np.zeros((2, 2, 2), np.uint8)]:
        with pytest.raises(ValueError):
            native.squared_distance(bad)
    with fe.PersistentPairEDT((4, 4, 4)) as h:
        m = np.zeros((4, 4, 4), bool)
        m[0, 0, 0] = True
        for pitch in (0, -1, float("nan"), float("inf"), True, 1e13, 1e-13):
            with pytest.raises(ValueError):
                h.query(m, pitch)
        with pytest.raises(ValueError):
            h.query(np.zeros((4, 4, 5), bool), 1.0)


def test_raw_abi_rejects_invalid_mask_bytes(fe):
    import field_b200._lib as L
    lib = L.lib()
    m = np.zeros((4, 5, 6), np.uint8)
    m[1, 1, 1] = 2
    out = np.full((4, 5, 6), -7, np.int32)
    assert lib.edt_squared_large(m.ctypes.data, 4, 5, 6, out.ctypes.data) == 1
    assert (out == -7).all()
    m[1, 1, 1] = 0
    assert lib.edt_squared_large(m.ctypes.data, 4, 5, 6, out.ctypes.data) == 1  # one class only
    m[0, 0, 0] = 1
    assert lib.edt_squared_large(m.ctypes.data, 4, 5, 6, out.ctypes.data) == 0


def test_handle_lifecycle(fe):
    import threading
    h = fe.PersistentPairEDT((3, 4, 5))
    m = np.zeros((3, 4, 5), bool)
    m[1, 2, 3] = True
    h.query(m, 1.0)
    errors = []

    def other():
        try:
            h.query(m, 1.0)
        except RuntimeError:
            errors.append(True)
    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert errors == [True]
    h.close()
    h.close()
    with pytest.raises(RuntimeError):
        h.query(m, 1.0)
