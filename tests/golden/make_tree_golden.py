"""Generate tests/golden/tree_golden.{npz,json}: the reference's packed adaptive block tree
(src/field_engine/field_adaptive_blocks_v1.py) on seeded dense fields.

Run where the reference is mounted (it is read, never written) after `make -C oracle`:

    FIELD_REFERENCE=<reference checkout> python tests/golden/make_tree_golden.py   (or the checkout as argv[1])

The reference module itself builds and samples every tree: its `build(wp, dense, pitch)` and
`AdaptiveBlocks.sample`.  Its one Warp call, the dense block classification
`faltkarna_v1_mesh_to_sdf.klassificera_och_evaluera_fran_tatt_falt`, is served by the reference's
compiled CPU classifier of the same rule (`meshsdf_classify_cpu`, mesh_sdf_native_v1/field.cpp,
built into oracle/_ref), since Warp is not installed here.

The dense inputs are regenerated by `tree_cases.dense_case` in the tests; small outputs are stored
whole, the reconstruction as a SHA-256 digest plus values at seeded coordinates.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
_ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FIELD_REFERENCE")
if not _ref_root:
    sys.exit("set FIELD_REFERENCE (or pass the reference checkout as the first argument)")
REF = Path(_ref_root)
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))

import oracle  # noqa: E402
from tree_cases import CASES, dense_case  # noqa: E402


def main():
    fake = types.ModuleType("faltkarna_v1_mesh_to_sdf")

    def classify(wp, dense, pitch, block, device):
        return oracle.ref_classify_dense(dense, pitch, block)

    fake.klassificera_och_evaluera_fran_tatt_falt = classify
    sys.modules["faltkarna_v1_mesh_to_sdf"] = fake
    sys.path.insert(0, str(REF / "src" / "field_engine"))
    import field_adaptive_blocks_v1 as ref

    arrays, meta = {}, {}
    for name, params in CASES.items():
        dense, pitch = dense_case(**params)
        tree, histogram = ref.build(None, dense, pitch)
        coords = np.indices(dense.shape, dtype=np.int64).reshape(3, -1).T
        recon = tree.sample(coords).reshape(dense.shape)
        rng = np.random.default_rng(7)
        pick = np.stack([rng.integers(0, n, size=64) for n in dense.shape], axis=1)
        for key in ("packed", "branch_prefix", "value_prefix", "values"):
            arrays[f"{name}/{key}"] = getattr(tree, key)
        arrays[f"{name}/pick"] = pick
        arrays[f"{name}/pick_values"] = tree.sample(pick)
        meta[name] = dict(params=params, shape=list(tree.shape), pitch=tree.pitch,
                          root_shape=[int(v) for v in tree.root_shape], root_count=int(tree.root_count),
                          node_count=int(tree.node_count), histogram=histogram,
                          stored_bytes=int(tree.stored_bytes()), fingerprint=tree.fingerprint(),
                          dense_sha256=hashlib.sha256(dense.tobytes()).hexdigest(),
                          reconstruction_sha256=hashlib.sha256(recon.astype(np.float32).tobytes()).hexdigest(),
                          sign_mismatches=int(np.count_nonzero((dense < 0) != (recon < 0))))
        print(name, meta[name]["node_count"], len(tree.values), meta[name]["sign_mismatches"])
    np.savez_compressed(HERE / "tree_golden.npz", **arrays)
    (HERE / "tree_golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()
