"""The oracle against the reference's captured arrays and compiled code (CPU only).

These pins make the oracle trustworthy before it is used to check the CUDA library.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from conftest import Golden, sha


@pytest.fixture(scope="module")
def edt():
    return Golden("edt_golden")


def test_edt_squared_matches_reference_captures(edt):
    checked = 0
    for name in edt.names():
        m = edt.mask(name)
        for pol, binary in enumerate((~m, m)):
            key = f"squared{pol}"
            if key not in edt.meta[name]["sha256"]:
                continue
            got = oracle.edt_squared(binary)
            assert edt.matches(name, key, got), (name, key)
            checked += 1
    assert checked >= 40


def test_edt_signed_matches_reference_captures(edt):
    checked = 0
    for name in edt.names():
        m = edt.mask(name)
        for p in edt.meta[name]["pitches"]:
            got = oracle.edt_signed(m, p)
            assert edt.matches(name, f"signed_{p!r}", got), (name, p)
            checked += 1
    assert checked >= 80


def test_edt_envelope_equals_brute_force():
    rng = np.random.default_rng(3)
    for shape in [(1, 1, 2), (9, 1, 33), (17, 13, 11), (2, 40, 3)]:
        b = rng.random(shape) > 0.7
        b.flat[0] = False
        assert (oracle.edt_squared(b) == oracle.edt_squared(b, brute=True)).all()


def test_dense_classify_matches_compiled_reference():
    g = Golden("classify_golden")
    for name in g.names("dense/"):
        meta = g.meta[name]
        dense = g.z[f"field/{meta['field']}"]
        r = oracle.classify_dense(dense, meta["pitch"], meta["block"])
        assert (r["kind"] == g.z[f"{name}__kind"]).all(), name
        assert sha(r["tiles"]) == meta["tiles_sha256"], name


def test_pack_matches_compiled_reference():
    g = Golden("pack_golden")
    for name in g.names("pack/"):
        meta = g.meta[name]
        key = f"source/{meta['source']}"
        if key not in g.z.files:
            continue
        nodes, payload = oracle.pack(g.z[key], meta["threshold"])
        assert sha(nodes) == meta["nodes_sha256"], name
        assert sha(payload) == meta["payload_sha256"], name


def test_csg_restated_inputs_reproduce_reference_captures():
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import csg_inputs
    g = Golden("csg_golden")
    for name in g.names("csg/"):
        m = g.meta[name]
        fields, origin, shape, program = csg_inputs.case(m["curved"], m["pitch"])
        assert g.matches(name, "output", oracle.csg_execute(fields, program)), name


def test_query_restatement_matches_reference_capture():
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import csg_inputs
    g = Golden("csg_golden")
    fields = {}
    for name in g.names("csg/"):
        m = g.meta[name]
        f, origin, shape, program = csg_inputs.case(m["curved"], m["pitch"])
        fields[sha(oracle.csg_execute(f, program))] = oracle.csg_execute(f, program)
    for name in g.names("query/"):
        raw = fields[g.meta[name]["field_sha256"]]
        nodes, payload = oracle.pack(raw, 512)
        got = oracle.query_trilinear(nodes, payload, raw.shape, np.zeros(3), 1.0, g.z[f"{name}__points"])
        assert got.tobytes() == g.z[f"{name}__values"].tobytes(), name
