"""GPU packing, ordered CSG on packed fields and packed-field queries: bit-exact against the
reference's compiled packer, its captured CSG outputs and its captured query values."""
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from conftest import Golden, sha

pytestmark = pytest.mark.gpu
sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))


@pytest.fixture(scope="module")
def pk():
    import field_b200.packed as P
    return P


def test_pack_matches_compiled_reference(pk):
    g = Golden("pack_golden")
    n = 0
    for name in g.names("pack/"):
        meta = g.meta[name]
        key = f"source/{meta['source']}"
        if key not in g.z.files:
            continue
        f = pk.NativeAdaptiveBlocks(g.z[key], [0.1, -2, 3], 0.7, leaf_samples=meta["threshold"])
        assert sha(f.nodes) == meta["nodes_sha256"], name
        assert sha(f.payload) == meta["payload_sha256"], name
        n += 1
    assert n >= 6


@pytest.mark.parametrize("threshold", [8, 64, 512, 4096])
def test_pack_random_fields_match_oracle(pk, threshold):
    rng = np.random.default_rng(threshold)
    for shape in [(19, 23, 17), (29, 1, 17), (1, 19, 31), (40, 33, 70), (3, 4, 5)]:
        raw = rng.normal(size=shape).astype(np.float32)
        raw[:, :, : shape[2] // 2] = 0.25  # invariant slabs
        raw.ravel()[::7] = np.float32(-0.0)
        a = pk.AdaptiveSampleBlocks(raw, [0, 0, 0], 1, leaf_samples=threshold)
        nodes, payload = oracle.pack(raw, threshold)
        assert a.nodes.tobytes() == nodes.tobytes() and a.payload.tobytes() == payload.tobytes()


def test_pack_device_input_equals_host_input(pk):
    import torch
    rng = np.random.default_rng(5)
    raw = rng.normal(size=(64, 48, 80)).astype(np.float32)
    raw[10:40] = 1.5
    a = pk.AdaptiveSampleBlocks(raw, [0, 0, 0], 0.5)
    b = pk.AdaptiveSampleBlocks.from_device(torch.from_numpy(raw).cuda(), [0, 0, 0], 0.5)
    assert a.nodes.tobytes() == b.nodes.tobytes() and a.payload.tobytes() == b.payload.tobytes()


def test_csg_evaluate_matches_reference_captures(pk):
    import csg_inputs
    g = Golden("csg_golden")
    for name in g.names("csg/"):
        m = g.meta[name]
        fields, origin, shape, program = csg_inputs.case(m["curved"], m["pitch"])
        blocks = [pk.AdaptiveSampleBlocks(f, origin, m["pitch"]) for f in fields]
        out = pk.evaluate(blocks, program)
        dense = out.samples_at(np.indices(shape).reshape(3, -1).T).reshape(shape)
        assert g.matches(name, "output", dense), name
        # the packed result equals the reference packer's packing of the same samples
        nodes, payload = oracle.ref_pack(dense) if oracle.ref_library("pack") else oracle.pack(dense)
        assert out.nodes.tobytes() == nodes.tobytes() and out.payload.tobytes() == payload.tobytes()


def test_query_matches_reference_capture(pk):
    import csg_inputs
    g = Golden("csg_golden")
    fields = {}
    for name in g.names("csg/"):
        m = g.meta[name]
        f, origin, shape, program = csg_inputs.case(m["curved"], m["pitch"])
        out = oracle.csg_execute(f, program)
        fields[sha(out)] = out
    for name in g.names("query/"):
        raw = fields[g.meta[name]["field_sha256"]]
        blocks = pk.NativeAdaptiveBlocks(raw, [0, 0, 0], 1)
        got = blocks.query(g.z[f"{name}__points"])
        want = g.z[f"{name}__values"]
        assert np.abs(got - want).max() <= 4 * np.spacing(np.abs(want).max()), name
        assert got.tobytes() == want.tobytes(), name


def test_compose_ties_signed_zeros_and_offsets(pk):
    zeros = np.zeros((17, 19, 23), np.float32)
    negative = zeros.copy()
    negative.ravel()[::2] = np.float32(-0.0)
    tiny = np.full_like(zeros, np.nextafter(np.float32(0), np.float32(1)))
    specials = [pk.AdaptiveSampleBlocks(a, [0, 0, 0], 1) for a in (zeros, negative, tiny)]
    dense = [zeros, negative, tiny]
    idx = np.indices(zeros.shape).reshape(3, -1).T
    for program in ([("union", 0, 1)], [("union", 1, 0)], [("difference", 0, 1)], [("offset", 2, 0.0)],
                    [("offset", 1, .1), ("offset", 3, -.1)], [("union", 0, 1), ("difference", 3, 2), ("union", 4, 3)]):
        got = pk.evaluate(specials, program).samples_at(idx).reshape(zeros.shape)
        want = oracle.csg_execute(dense, program)
        assert got.tobytes() == want.tobytes(), program
    u = pk.compose(specials[0], specials[1])
    assert u.samples_at(idx).tobytes() == oracle.csg_execute(dense, [("union", 0, 1)]).tobytes()


def test_invalid_programs_and_operands_rejected(pk):
    valid = pk.AdaptiveSampleBlocks(np.ones((4, 4, 4), np.float32), [0, 0, 0], 1)
    for program in ([("union", 0, 99)], [("offset", 0, float("nan"))], [("offset", 0, 1e39), ("union", 1, 0)],
                    [("intersect", 0, 0)], [("union", True, 0)]):
        with pytest.raises(ValueError):
            pk.evaluate([valid], program)
    for bad in [(np.ones((2, 2, 2), np.float64), [0, 0, 0], 1, 512), (np.ones((2, 2), np.float32), [0, 0, 0], 1, 512),
                (np.full((2, 2, 2), np.nan, np.float32), [0, 0, 0], 1, 512),
                (np.ones((2, 2, 2), np.float32), [0, 0], 1, 512), (np.ones((2, 2, 2), np.float32), [0, 0, 0], 0, 512),
                (np.ones((2, 2, 2), np.float32), [0, 0, 0], True, 512),
                (np.ones((2, 2, 2), np.float32), [0, 0, 0], 1, True), (np.ones((2, 2, 2), np.float32), [0, 0, 0], 1, 4)]:
        with pytest.raises(ValueError):
            pk.NativeAdaptiveBlocks(bad[0], bad[1], bad[2], leaf_samples=bad[3])
    # malformed nodes: status 3 (shape) / 4 (overlap, gap) through the C ABI
    import copy
    for mode in ("offset", "shape", "overlap", "gap"):
        broken = copy.copy(valid)
        nodes = valid.nodes.copy()
        if mode == "offset":
            nodes["offset"][0] = 1000000
        if mode == "shape":
            nodes["stored_shape"][0] = [5, 4, 4]
        if mode == "overlap":
            nodes = np.concatenate((nodes, nodes))
        if mode == "gap":
            nodes["shape"][0] = [1, 1, 1]
        broken.nodes = nodes
        with pytest.raises(ValueError):
            pk.evaluate([broken], [("offset", 0, 0.0)])
