"""Packed adaptive block tree built and sampled on the GPU (field_b200.tree): equal to the trees the
reference module built (tests/golden/tree_golden.*) and to the oracle restatement, byte for byte,
with the reconstruction of every voxel identical; edge cases of all-outside / all-inside fields and
out-of-grid indices."""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from tree_cases import CASES, dense_case  # noqa: E402

ARRAYS = ("packed", "branch_prefix", "value_prefix", "values")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "tree_golden.npz"), json.loads((GOLDEN / "tree_golden.json").read_text())


def _same_tree(tree, hist, expect):
    for key in ARRAYS:
        assert np.array_equal(getattr(tree, key), expect[key]), key
        assert getattr(tree, key).dtype == np.asarray(expect[key]).dtype, key
    assert tree.node_count == expect["node_count"] and tree.root_count == expect["root_count"]
    assert tuple(tree.root_shape) == tuple(expect["root_shape"])
    assert hist == expect["histogram"]


@pytest.mark.parametrize("name", list(CASES))
def test_gpu_tree_equals_the_reference_trees(golden, name):
    import field_b200.tree as T
    arrays, meta = golden
    dense, pitch = dense_case(**CASES[name])
    tree, hist = T.build(None, dense, pitch)
    m = meta[name]
    _same_tree(tree, hist, dict(m, **{k: arrays[f"{name}/{k}"] for k in ARRAYS}))
    assert tree.fingerprint() == m["fingerprint"] and tree.stored_bytes() == m["stored_bytes"]
    coords = np.indices(dense.shape).reshape(3, -1).T
    recon = tree.sample(coords).reshape(dense.shape)
    assert hashlib.sha256(recon.tobytes()).hexdigest() == m["reconstruction_sha256"]
    assert np.array_equal(tree.sample(arrays[f"{name}/pick"]), arrays[f"{name}/pick_values"])


def test_host_array_tree_samples_on_the_device(golden):
    """A tree made from stored arrays (no device state yet) uploads them once and samples exactly."""
    import field_b200.tree as T
    arrays, meta = golden
    name = "mixed_70x64x53"
    m = meta[name]
    tree = T.AdaptiveBlocks(tuple(m["shape"]), m["pitch"], tuple(m["root_shape"]), m["root_count"], m["node_count"],
                            *(arrays[f"{name}/{k}"] for k in ARRAYS))
    coords = np.indices(tree.shape).reshape(3, -1).T
    recon = tree.sample(coords).reshape(tree.shape)
    assert hashlib.sha256(recon.tobytes()).hexdigest() == m["reconstruction_sha256"]


@pytest.mark.parametrize("shape,seed", [((150, 131, 97), 11), ((8, 8, 8), 12), ((200, 41, 129), 13)])
def test_gpu_tree_equals_oracle_on_larger_grids(shape, seed):
    import field_b200.tree as T
    dense, pitch = dense_case(shape=shape, n_spheres=12, n_boxes=8, seed=seed)
    tree, hist = T.build(None, dense, pitch)
    _same_tree(tree, hist, oracle.tree_build(dense, pitch))
    rng = np.random.default_rng(seed)
    pts = np.stack([rng.integers(0, n, size=200_000) for n in shape], axis=1)
    ref = oracle.tree_sample(oracle.tree_build(dense, pitch), pts, pitch)
    assert np.array_equal(tree.sample(pts), ref)
    # the reference's narrow-band gate: every voxel with |d| <= pitch reads back its dense value
    # byte for byte, and no sign flips anywhere
    band = np.abs(dense) <= pitch
    assert np.array_equal(tree.sample(np.argwhere(band)), dense[band])
    every = tree.sample(np.indices(shape).reshape(3, -1).T).reshape(shape)
    assert np.array_equal(every < 0, dense < 0)


@pytest.mark.parametrize("value", [5.0, -5.0])
def test_one_sided_fields_are_roots_only(value):
    import field_b200.tree as T
    dense = np.full((19, 16, 33), value, np.float32)
    pitch = 0.1
    tree, hist = T.build(None, dense, pitch)
    _same_tree(tree, hist, oracle.tree_build(dense, pitch))
    assert tree.node_count == tree.root_count == 3 * 2 * 5 and len(tree.values) == 0
    out = tree.sample(np.array([[0, 0, 0], [18, 15, 32]]))
    expect = np.float32(np.sign(value) * np.sqrt(3.0) * 8 * pitch)
    assert (out == expect).all()


def test_out_of_grid_indices():
    import torch
    import field_b200.tree as T
    dense, pitch = dense_case(**CASES["spheres_37x41x29"])
    tree, _ = T.build(None, dense, pitch)
    for bad in ([[37, 0, 0]], [[-1, 2, 3]], [[1, 2]]):
        with pytest.raises(ValueError):
            tree.sample(np.array(bad))
    # on the device the kernel checks instead: NaN and the status bit, the rest unaffected
    d = tree._device()
    d["status"].zero_()
    ijk = torch.tensor([[1, 2, 3], [37, 0, 0], [0, 41, 0]], dtype=torch.int64, device="cuda")
    out = tree.sample_device(ijk).cpu().numpy()
    assert int(d["status"].item()) & 1
    assert np.isnan(out[1:]).all()
    assert out[0] == tree.sample(np.array([[1, 2, 3]]))[0]
