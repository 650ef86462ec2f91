"""Export step on the GPU (field_b200.export through fb_mc_* and fb_mesh_components_device)
against the oracle's marching cubes on the dense reconstruction: the same vertex edges with
bit-equal float32 positions, the same oriented triangles, the volume; on analytic fields (ragged
grids, block sizes 4 / 8 / 16, a nonzero level), dense random fields with ambiguous faces and exact
zeros, empty fields; bit-reproducible; the component split of faltvolym_v1.py:83-104; the .npz
round trip of a resident field."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _canon(faces_as_keys):
    f = np.asarray(faces_as_keys, np.int64).reshape(-1, 3)
    if not len(f):
        return f
    r = np.argmin(f, axis=1)
    rolled = np.stack([f[np.arange(len(f)), (r + i) % 3] for i in range(3)], 1)
    return rolled[np.lexsort(rolled.T[::-1])]


def _compare(mesh, dense, level, origin, pitch):
    keys, pos, faces = oracle.marching_cubes(dense, level, origin, pitch)
    order = np.argsort(mesh.keys)
    assert np.array_equal(mesh.keys[order], keys)
    assert mesh.verts[order].tobytes() == pos.tobytes()
    assert np.array_equal(_canon(mesh.keys[mesh.faces]), _canon(faces))
    kid = np.searchsorted(keys, faces)
    want = oracle.mesh_volume(pos, kid) if len(faces) else 0.0
    v = pos.astype(np.float64)
    scale = np.abs(np.einsum("ij,ij->i", v[kid[:, 0]], np.cross(v[kid[:, 1]], v[kid[:, 2]]))).sum() if len(faces) else 0
    assert abs(mesh.volume - want) <= 1e-12 * scale  # summation order only
    return len(keys), len(faces)


def _recipe_field(n, block, seed=0, origin=(0.0, 0.0, 0.0)):
    import field_b200.build as B
    import field_b200.expr as X
    import field_b200.grid as G
    import field_b200.recipes as R
    rng = np.random.default_rng(seed)
    recipe = X.union_all(R.parts(rng, 6, 6, 3, 2))
    meta = G.GridMeta(origin[0], origin[1], origin[2], 1.0 / 64, n[0], n[1], n[2], block)
    return B.FieldBuilder(X.compile_recipe(recipe), meta).build(), meta


@pytest.mark.parametrize("n,block,level", [((64, 64, 64), 8, 0.0), ((61, 50, 37), 8, 0.0), ((45, 64, 29), 4, 0.0),
                                            ((70, 33, 48), 16, 0.0), ((64, 64, 64), 8, 0.01)])
def test_sparse_field_mesh_equals_the_oracle(n, block, level):
    import field_b200.export as E
    field, meta = _recipe_field(n, block, origin=(-0.05, 0.02, 0.01))
    mesh = E.marching_cubes(field, level, keys=True)
    sf = field.to_host()
    dense = oracle.reconstruct(sf.kind, sf.active_ids, sf.tiles, meta)
    nv, nt = _compare(mesh, dense, level, (meta.x0, meta.y0, meta.z0), meta.pitch)
    assert nv > 500 and nt > 1000
    again = E.marching_cubes(field, level, keys=True)
    assert again.verts.tobytes() == mesh.verts.tobytes() and again.faces.tobytes() == mesh.faces.tobytes()
    assert again.volume == mesh.volume


@pytest.mark.parametrize("seed", range(3))
def test_dense_random_fields_equal_the_oracle(seed):
    import field_b200.export as E
    rng = np.random.default_rng(seed)
    shp = (23, 30, 19)
    f = rng.normal(size=shp).astype(np.float32)
    f[rng.random(shp) < 0.1] = 0.0
    mesh = E.marching_cubes_dense(f, 0.0, pitch=0.5, origin=(1.0, 2.0, 3.0), keys=True)
    _compare(mesh, f, 0.0, (1.0, 2.0, 3.0), 0.5)


def test_empty_and_single_sign_fields():
    import field_b200.export as E
    for v in (1.0, -1.0):
        mesh = E.marching_cubes_dense(np.full((12, 9, 10), v, np.float32), keys=True)
        assert mesh.verts.shape == (0, 3) and mesh.faces.shape == (0, 3) and mesh.volume == 0.0
    assert E.marching_cubes_volym(np.full((12, 9, 10), 1.0, np.float32), 0.1) == (0.0, 0)
    assert E.marching_cubes_volym(np.full((12, 9, 10), -1.0, np.float32), 0.1) == (0.0, 0)


def test_volume_meters_and_components():
    import field_b200.export as E
    n, h = 64, 1.0 / 32
    idx = np.indices((n, n, n)).reshape(3, -1).T * h
    big = np.linalg.norm(idx - np.array([0.7, 1.0, 1.0]), axis=1) - 0.45
    small = np.linalg.norm(idx - np.array([1.5, 1.0, 1.0]), axis=1) - 0.2
    f = np.minimum(big, small).reshape(n, n, n).astype(np.float32)
    vol, dropped = E.marching_cubes_volym(f, h)
    assert dropped == 1
    assert abs(vol - 4.0 / 3.0 * np.pi * 0.45 ** 3) < 0.01 * vol
    assert abs(E.voxel_riemann_volym(f, h) - np.count_nonzero(f < 0) * h ** 3) == 0.0
    mesh = E.marching_cubes_dense(f, 0.0, pitch=h)
    lab, vols = E.components(mesh)
    assert len(vols) == 2
    assert abs(sum(vols.values()) - mesh.volume) < 1e-9 * mesh.volume


def test_npz_round_trip_of_a_resident_field(tmp_path):
    import field_b200.export as E
    field, meta = _recipe_field((48, 40, 56), 8, seed=3)
    p = tmp_path / "f.npz"
    E.save_field(p, field)
    loaded = E.load_field(p)
    a, b = E.marching_cubes(field), E.marching_cubes(loaded)
    assert a.verts.tobytes() == b.verts.tobytes() and a.faces.tobytes() == b.faces.tobytes()
    assert loaded.stats["n_active"] == field.n_active
