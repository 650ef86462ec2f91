"""Generate the golden fixtures in tests/golden/ from the reference checkout.

Run once where the reference is mounted (it is read, never written):

    FIELD_REFERENCE=<reference checkout> python tests/golden/make_golden.py   (or the checkout as argv[1])

Sources, all the reference's own:
* EDT -- the captured arrays of its probes (artifacts/field_edt_integer_v1_arrays.npz,
  reports/edt_large_arrays.npz, reports/field_persistent_edt_arrays.npz,
  reports/field_linear_edt_arrays.npz) with the input masks they were computed from
  (artifacts/field_rt_changed_query_reference_arrays.npz, reports/stage_scale_mechanism_arrays.npz,
  and the rng(441) masks of probes/field_engine/field_persistent_edt_probe.py:24-27, regenerated
  here exactly as the probe does).
* Dense classification and tiles -- meshsdf_classify_cpu / meshsdf_tiles_cpu compiled from
  src/field_engine/mesh_sdf_native_v1/field.cpp (oracle/_ref), on the reference's captured
  distance fields.
* Sampled-field CSG -- reports/field_csg_batch_arrays.npz (outputs of the reference's batched
  native CSG) for the two programs of probes/field_engine/field_csg_batch_probe.py:41-46.
* Packing -- adaptive_pack compiled from src/field_engine/adaptive_pack_native_v1/pack.cpp.
* Expressions -- src/field_engine/ikarus_v1/expr.py: constructors and eval_sdf_py at seeded points.

Small arrays are stored whole; large ones as SHA-256 digests of their bytes.  Masks are bit-packed.
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
_ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FIELD_REFERENCE")
if not _ref_root:
    sys.exit("set FIELD_REFERENCE (or pass the reference checkout as the first argument)")
REF = Path(_ref_root)
FULL_LIMIT = 70000  # voxels up to which expected arrays are stored whole


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def pack_mask(m):
    return np.packbits(np.ascontiguousarray(m, dtype=bool).ravel())


class Writer:
    def __init__(self):
        self.arrays = {}
        self.meta = {}

    def mask(self, name, m):
        self.arrays[f"{name}__mask"] = pack_mask(m)
        self.meta.setdefault(name, {})["shape"] = list(m.shape)

    def expect(self, name, key, a):
        entry = self.meta.setdefault(name, {})
        if a.size <= FULL_LIMIT:
            self.arrays[f"{name}__{key}"] = a
        entry.setdefault("sha256", {})[key] = digest(a)
        entry.setdefault("dtype", {})[key] = str(a.dtype)

    def save(self, stem):
        np.savez_compressed(HERE / f"{stem}.npz", **self.arrays)
        (HERE / f"{stem}.json").write_text(json.dumps(self.meta, indent=1, sort_keys=True) + "\n")


def edt_fixtures():
    w = Writer()
    # (1) integer EDT probe: masks from the changed-query capture + boundary/tie cases.
    with np.load(REF / "artifacts/field_rt_changed_query_reference_arrays.npz") as z:
        masks = {k: z[k] for k in z.files if k.endswith("_mask")}
    boundary = np.zeros((5, 7, 9), bool)
    boundary[0, 0, 0] = True
    masks["boundary_single_site"] = boundary
    masks["boundary_single_hole"] = ~boundary
    masks["checkerboard_ties"] = np.indices((7, 8, 9)).sum(axis=0) % 2 == 0
    masks["singleton_axis"] = np.indices((1, 5, 7)).sum(axis=0) % 3 == 0
    pitches = (0.125, 0.3, 0.7483641718372458)
    with np.load(REF / "artifacts/field_edt_integer_v1_arrays.npz") as z:
        for key, m in masks.items():
            name = f"integer/{key}"
            w.mask(name, m)
            w.meta[name]["pitches"] = list(pitches)
            for pol in range(2):
                w.expect(name, f"squared{pol}", z[f"{key}_square_{pol}"].astype(np.int32))
            for i in range(3):
                w.expect(name, f"signed_{pitches[i]!r}", z[f"{key}_signed_{i}"])
    # (2) large EDT probe: plate masks and tie cases (probes/field_engine/field_edt_large_probe.py:23-26).
    with np.load(REF / "reports/stage_scale_mechanism_arrays.npz") as z:
        cases = {f"plate_{p}": (z[f"{p}_0_solid"], p) for p in (2.0, 1.0, 0.5)}
    site = np.ones((512, 2, 1), bool)
    site[0, 0, 0] = False
    cases.update(single_site=(site, 1.0), checker=(np.indices((129, 3, 7)).sum(axis=0) % 2 == 0, 0.25))
    with np.load(REF / "reports/edt_large_arrays.npz") as z:
        for key, (m, p) in cases.items():
            name = f"large/{key}"
            w.mask(name, m)
            w.meta[name]["pitches"] = [p]
            for pol in range(2):
                w.expect(name, f"squared{pol}", z[f"{key}_0_squared{pol}"])
            w.expect(name, f"signed_{p!r}", z[f"{key}_0_signed"])
    # (3) persistent pair probe: rng(441) masks, 5 pitches incl. the contract ends.
    rng = np.random.default_rng(441)
    pcases = []
    for shape in ((1, 1, 2), (512, 1, 7), (1, 512, 7), (7, 1, 512), (31, 27, 19), (97, 65, 89)):
        m = rng.random(shape) > .4
        m.flat[0] = False
        m.flat[-1] = True
        pcases.append(("random_" + str(shape), m))
    single = np.ones((37, 41, 43), bool)
    single[18, 20, 21] = False
    pcases += [("single_zero", single), ("single_one", ~single)]
    ppitches = (1e-12, .125, .7, 2., 1e12)
    with np.load(REF / "reports/field_persistent_edt_arrays.npz") as z:
        plate = z.get("plate_L_0_0.5") if "plate_L_0_0.5" in z.files else None
        for key, m in pcases:
            name = f"persistent/{key}"
            w.mask(name, m)
            w.meta[name]["pitches"] = list(ppitches)
            for p in ppitches:
                w.expect(name, f"signed_{p!r}", z[f"{key}_0_{p}"])
        # The plate_L mask came from a mesh that is not in the checkout; the stage-scale plate
        # mask at pitch 0.5 has the same shape.  It is kept only if it reproduces the capture.
        if plate is not None:
            with np.load(REF / "reports/stage_scale_mechanism_arrays.npz") as s:
                cand = s["0.5_0_solid"]
            sys.path.insert(0, str(REPO))
            import oracle
            if oracle.edt_signed(cand, 0.5).tobytes() == plate.tobytes():
                name = "persistent/plate_L"
                w.mask(name, cand)
                w.meta[name]["pitches"] = list(ppitches)
                for p in ppitches:
                    w.expect(name, f"signed_{p!r}", z[f"plate_L_0_{p}"])
    # (4) linear envelope probe: squared pairs for the same rng(441) masks.  That probe stores
    # squared_distance(b) for b in (mask, ~mask) (probes/field_engine/field_linear_edt_probe.py:41),
    # i.e. index 0 measures to the empty voxels: our polarity 1.
    with np.load(REF / "reports/field_linear_edt_arrays.npz") as z:
        for key, m in pcases:
            if f"{key}_0_squared_0" not in z.files:
                continue
            name = f"persistent/{key}"
            for i in range(2):
                w.expect(name, f"squared{1 - i}", z[f"{key}_0_squared_{i}"])
    w.save("edt_golden")
    print("edt cases:", len(w.meta))


def classify_fixtures():
    sys.path.insert(0, str(REPO))
    import oracle
    w = Writer()
    with np.load(REF / "reports/stage_scale_mechanism_arrays.npz") as z:
        fields = {f"plate_{p}": (z[f"{p}_0_distance"], p) for p in (2.0, 1.0, 0.5)}
    with np.load(REF / "reports/field_csg_curved_arrays.npz") as z:
        fields["bracket_0.25"] = (z["bracket_plate_rectangular_holes_0.25_0_field"], 0.25)
        fields["sphere_plate_0.5"] = (z["sphere_plate_round_hole_0.5_0_field"], 0.5)
    for key, (dense, pitch) in fields.items():
        for block in (4, 8, 16):
            name = f"dense/{key}/B{block}"
            r = oracle.ref_classify_dense(dense, pitch, block)
            w.arrays[f"{name}__kind"] = r["kind"].astype(np.int8)
            w.meta[name] = dict(field=key, pitch=pitch, block=block, n_active=r["n_active"],
                                tiles_sha256=digest(r["tiles"]))
        w.arrays[f"field/{key}"] = dense.astype(np.float32)
    w.save("classify_golden")
    print("classify cases:", len(w.meta))


def csg_fixtures():
    """Programs and outputs of probes/field_engine/field_csg_batch_probe.py:41-51, inputs restated in
    csg_inputs.py and checked here against the capture through the oracle; plus the packed-field
    query capture of probes/field_engine/field_native_pack_probe.py:26-40 (rng 445, 4097 points per
    field, origin 0, pitch 1)."""
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(HERE))
    import oracle
    import csg_inputs
    w = Writer()
    with np.load(REF / "reports/field_csg_batch_arrays.npz") as z:
        for curved in (False, True):
            for pitch in (.5, .25):
                name = f"csg/{curved}/{pitch}"
                out = z[f"{curved}_{pitch}_0"]
                fields, origin, shape, program = csg_inputs.case(curved, pitch)
                assert oracle.csg_execute(fields, program).tobytes() == out.tobytes(), name
                w.meta[name] = dict(curved=curved, pitch=pitch, program=program, shape=list(out.shape))
                w.expect(name, "output", out)
    rng = np.random.default_rng(445)
    with np.load(REF / "reports/field_csg_curved_arrays.npz") as data:
        cases = [(name, data[name]) for name in data.files if name.endswith("_0_field")]
    with np.load(REF / "reports/field_native_pack_arrays.npz") as cap:
        for name, raw in cases:
            points = rng.uniform(-1, np.array(raw.shape) + 1, (4097, 3))
            key = f"query/{name}"
            w.meta[key] = dict(field_sha256=digest(raw), shape=list(raw.shape))
            w.arrays[f"{key}__points"] = points
            w.arrays[f"{key}__values"] = cap[f"{name}_0"]
            assert cap[f"{name}_0"].tobytes() == cap[f"{name}_1"].tobytes()
    w.save("csg_golden")
    print("csg cases:", len(w.meta))


def pack_fixtures():
    sys.path.insert(0, str(REPO))
    import oracle
    w = Writer()
    sources = {}
    with np.load(REF / "reports/field_csg_batch_arrays.npz") as z:
        sources["csg_false_0.5"] = z["False_0.5_0"]
        sources["csg_true_0.25"] = z["True_0.25_0"]
    with np.load(REF / "reports/stage_scale_mechanism_arrays.npz") as z:
        sources["plate_1.0"] = z["1.0_0_distance"]
    rng = np.random.default_rng(77)
    raw = rng.normal(size=(19, 21, 17)).astype(np.float32)
    raw.ravel()[::2] = np.float32(-0.)
    sources["signed_zeros"] = raw
    sources["constant"] = np.full((17, 19, 23), .25, np.float32)
    for key, a in sources.items():
        for thr in (8, 512, 4096):
            name = f"pack/{key}/{thr}"
            nodes, payload = oracle.ref_pack(a, thr)
            w.meta[name] = dict(source=key, threshold=thr, n_nodes=int(len(nodes)), n_samples=int(len(payload)),
                                nodes_sha256=digest(nodes), payload_sha256=digest(payload))
        if a.size <= FULL_LIMIT:
            w.arrays[f"source/{key}"] = a
    w.save("pack_golden")
    print("pack cases:", len(w.meta))


def expr_fixtures():
    sys.path.insert(0, str(REF / "src/field_engine/ikarus_v1"))
    import expr as E
    rng = np.random.default_rng(5)
    trees = {}
    c = E.cylinder(radius=12.5, height=40.0)
    b = E.box(half_extents=(8.0, 8.0, 8.0), center=(3.0, 0.0, 5.0))
    s = E.sphere(radius=6.0, center=(-4.0, 2.0, -3.0))
    trees["selftest_smooth"] = E.union(E.subtract(c, b, k=0.0), E.rotate(s, "y", 37.0), k=2.0)
    trees["expr_main"] = E.subtract(E.cylinder(radius=12.5, height=40.0),
                                    E.translate(E.box(half_extents=(8.0, 8.0, 8.0), center=(0.0, 0.0, 15.0)), 0, 0, 0))
    trees["cone_x"] = E.intersect(E.cone(4.0, 9.0, 20.0, axis="x", center=(1.0, -2.0, 0.5)),
                                  E.halfspace((0.3, -1.0, 0.2), 1.5))
    trees["frustum"] = E.union(E.rect_frustum(-3.0, 5.0, 4.0, 3.0, 2.0, 1.5, 0.2, -0.1, 1.0, 0.7),
                               E.offset(E.sphere(3.0, (0.0, 0.0, 8.0)), 0.5), k=1.5)
    trees["scaled_rot"] = E.scale(E.rotate(E.cylinder(3.0, 10.0, axis="y", center=(1.0, 1.0, 0.0)), "z", 23.0,
                                           about=(1.0, 0.0, 0.0)), 1.7)
    trees["axis_project"] = E.intersect(E.axis_project(E.box((5.0, 4.0, 3.0), (0.0, 0.0, 1.0)), 2, 1.0),
                                        E.subtract(E.halfspace((0, 0, 1), 4.0), E.halfspace((0, 0, 1), -2.0),
                                                   k=0.5))
    trees["smooth_intersect"] = E.intersect(E.sphere(7.0), E.box((6.0, 6.0, 6.0), (1.0, 0.0, 0.0)), k=2.5)
    arrays = {}
    meta = {}
    for name, tree in trees.items():
        pts = rng.uniform(-25, 25, size=(3000, 3))
        vals = np.array([E.eval_sdf_py(tree, tuple(p)) for p in pts])
        arrays[f"{name}__points"] = pts
        arrays[f"{name}__values"] = vals
        meta[name] = tree
    np.savez_compressed(HERE / "expr_golden.npz", **arrays)
    (HERE / "expr_golden.json").write_text(json.dumps(meta, indent=1) + "\n")
    print("expr trees:", len(trees))


if __name__ == "__main__":
    subprocess.run(["make", "-C", str(REPO / "oracle"), f"REF={REF}"], check=True, capture_output=True)
    edt_fixtures()
    classify_fixtures()
    csg_fixtures()
    pack_fixtures()
    expr_fixtures()
