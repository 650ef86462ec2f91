"""Export step on the CPU: the oracle's marching cubes (closed, consistently oriented, the analytic
volume of a sphere to 0.5 %, crack-free on random fields with ambiguous faces and exact zeros) and
the .npz field format (round trip, record, refusals)."""
import json
from collections import Counter

import numpy as np
import pytest

import oracle


def _sphere(n=40, pitch=0.05, r=0.7, c=(1.0, 1.0, 1.0)):
    idx = np.indices((n, n, n)).reshape(3, -1).T * pitch
    return (np.linalg.norm(idx - np.asarray(c), axis=1) - r).reshape(n, n, n).astype(np.float32)


def _ids(keys, faces):
    kid = {int(k): i for i, k in enumerate(keys)}
    return np.vectorize(kid.get)(faces) if len(faces) else faces


def test_oracle_sphere_closed_oriented_volume():
    f = _sphere()
    keys, pos, faces = oracle.marching_cubes(f, 0.0, (0.0, 0.0, 0.0), 0.05)
    assert (np.diff(keys) > 0).all()
    F = _ids(keys, faces)
    de = Counter((int(u), int(v)) for a, b, c in F for u, v in ((a, b), (b, c), (c, a)))
    assert all(n == 1 for n in de.values()) and all(de[(v, u)] == 1 for (u, v) in de)
    vol = oracle.mesh_volume(pos, F)
    assert abs(vol - 4.0 / 3.0 * np.pi * 0.7 ** 3) < 5e-3 * vol  # outward normals: positive
    # every vertex lies on its edge, between the two samples
    lin, ax = keys // 3, keys % 3
    ijk = np.stack(np.unravel_index(lin, f.shape), 1).astype(np.float64)
    off = pos / 0.05 - ijk
    for a in range(3):
        m = ax == a
        assert (off[m, a] >= -1e-4).all() and (off[m, a] <= 1 + 1e-4).all()
        assert np.abs(np.delete(off[m], a, axis=1)).max() < 1e-4


@pytest.mark.parametrize("seed", range(6))
def test_oracle_random_fields_have_no_cracks(seed):
    rng = np.random.default_rng(seed)
    shp = (9, 10, 11)
    f = rng.normal(size=shp).astype(np.float32)
    f[rng.random(shp) < 0.1] = 0.0
    keys, pos, faces = oracle.marching_cubes(f, 0.0)
    F = _ids(keys, faces)
    de = Counter((int(u), int(v)) for a, b, c in F for u, v in ((a, b), (b, c), (c, a)))

    def on_boundary(k):
        lin, a = k // 3, k % 3
        p = np.unravel_index(lin, shp)
        return any((p[d] == 0 or p[d] == shp[d] - 1) and d != a for d in range(3))
    open_edges = [(u, v) for (u, v) in de if de[(u, v)] != de.get((v, u), 0)
                  and not (on_boundary(keys[u]) and on_boundary(keys[v]))]
    assert not open_edges


def _field(seed=0):
    from field_b200.grid import GridMeta, SparseField
    rng = np.random.default_rng(seed)
    meta = GridMeta(0.5, -1.0, 2.0, 0.1, 20, 21, 17, 8)
    kind = rng.choice([-1, 1], meta.n_blocks).astype(np.int32)
    act = np.sort(rng.choice(meta.n_blocks, 5, replace=False)).astype(np.int32)
    kind[act] = 0
    return SparseField(meta, kind, act, rng.random((5, 8, 8, 8)).astype(np.float32),
                       rng.random(meta.n_blocks).astype(np.float32))


def test_npz_round_trip_and_record(tmp_path):
    import field_b200.export as E
    sf = _field()
    p = tmp_path / "field.npz"
    E.save_field(p, sf)
    g = E.load_field(p)
    assert g.meta == sf.meta
    for k in ("kind", "active_ids", "tiles", "corner_min_abs"):
        assert np.array_equal(getattr(g, k), getattr(sf, k))
    rec = E.field_record(sf)
    assert json.loads(json.dumps(rec)) == rec
    assert rec["stats"]["n_active"] == 5 and rec["format"] == E.FORMAT
    # the dense reconstruction of the loaded field equals the original's
    assert np.array_equal(oracle.reconstruct(g.kind, g.active_ids, g.tiles, g.meta),
                          oracle.reconstruct(sf.kind, sf.active_ids, sf.tiles, sf.meta))


def test_npz_refusals(tmp_path):
    import field_b200.export as E
    sf = _field(1)
    bad_tiles = _field(1)
    bad_tiles.tiles = bad_tiles.tiles[:4]
    unlisted = _field(1)
    unlisted.kind = unlisted.kind.copy()
    unlisted.kind[np.setdiff1d(np.arange(sf.meta.n_blocks), sf.active_ids)[0]] = 0
    for i, f in enumerate((bad_tiles, unlisted)):
        p = tmp_path / f"bad{i}.npz"
        E.save_field(p, f)
        with pytest.raises(ValueError):
            E.load_field(p)
    p = tmp_path / "other.npz"
    np.savez(p, kind=sf.kind, active_ids=sf.active_ids, tiles=sf.tiles, corner_min_abs=sf.corner_min_abs,
             meta=np.array(json.dumps({"format": "something/else"})))
    with pytest.raises(ValueError):
        E.load_field(p)
