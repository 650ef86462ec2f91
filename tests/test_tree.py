"""Packed adaptive block tree (src/field_engine/field_adaptive_blocks_v1.py) on the CPU: the oracle
restatement against the fixtures the reference module itself produced, and the host-side methods
of field_b200.tree.AdaptiveBlocks (kinds, rank_before, stored_bytes, fingerprint) on those trees."""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from tree_cases import CASES, dense_case  # noqa: E402

ARRAYS = ("packed", "branch_prefix", "value_prefix", "values")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "tree_golden.npz"), json.loads((GOLDEN / "tree_golden.json").read_text())


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_tree_matches_reference_fixtures(golden, name):
    arrays, meta = golden
    dense, pitch = dense_case(**CASES[name])
    assert hashlib.sha256(dense.tobytes()).hexdigest() == meta[name]["dense_sha256"]
    t = oracle.tree_build(dense, pitch)
    for key in ARRAYS:
        assert np.array_equal(t[key], arrays[f"{name}/{key}"]), key
    assert t["node_count"] == meta[name]["node_count"] and t["root_count"] == meta[name]["root_count"]
    assert list(t["root_shape"]) == meta[name]["root_shape"] and t["histogram"] == meta[name]["histogram"]
    coords = np.indices(dense.shape).reshape(3, -1).T
    recon = oracle.tree_sample(t, coords, pitch).reshape(dense.shape)
    assert hashlib.sha256(recon.tobytes()).hexdigest() == meta[name]["reconstruction_sha256"]
    assert np.array_equal(oracle.tree_sample(t, arrays[f"{name}/pick"], pitch), arrays[f"{name}/pick_values"])


@pytest.mark.parametrize("name", list(CASES))
def test_host_methods_on_reference_trees(golden, name):
    import field_b200.tree as T
    arrays, meta = golden
    m = meta[name]
    tree = T.AdaptiveBlocks(tuple(m["shape"]), m["pitch"], tuple(m["root_shape"]), m["root_count"], m["node_count"],
                            *(arrays[f"{name}/{k}"] for k in ARRAYS))
    assert tree.stored_bytes() == m["stored_bytes"] and tree.fingerprint() == m["fingerprint"]
    nodes = np.arange(m["node_count"])
    codes = ((tree.packed[:, None] >> np.array([0, 2, 4, 6], np.uint8)) & 3).reshape(-1)[:m["node_count"]]
    assert np.array_equal(tree.kinds(nodes), codes)
    for code in (2, 3):
        expect = np.concatenate(([0], np.cumsum(codes == code)))[:-1]
        assert np.array_equal(tree.rank_before(nodes, code), expect)
