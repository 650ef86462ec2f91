"""gridfield leaves (src/field_engine/ikarus_v1/expr.py:143-152, sampled as eval_warp.py:94-147) in
recipes, field builds and point queries, and the one-launch multi-pair sweep (eval_warp.py:545-564),
against the float64 oracle (GPU).  The sampler computes in float32 like the reference's, so values
are compared within 1e-5 pitch plus 2e-6 of their magnitude."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _write(tmp_path, name, arr, origin=None, pitch=None):
    extra = {}
    if origin is not None:
        extra["global_origin_mm"] = np.asarray(origin, np.float64)
    if pitch is not None:
        extra["pitch_mm"] = np.float64(pitch)
    path = tmp_path / f"{name}.npz"
    np.savez(path, **{name: arr.astype(np.float32)}, **extra)
    return str(path)


def _torus_sdf(shape, origin, pitch):
    x, y, z = (np.asarray(origin)[:, None, None, None] + np.indices(shape) * pitch)
    q = np.sqrt(x * x + y * y) - 0.15
    return (np.sqrt(q * q + z * z) - 0.06).astype(np.float32)


def _close(got, want, pitch):
    return np.abs(got - want) <= 1e-5 * pitch + 2e-6 * np.abs(want)


def test_gridfield_recipe_builds_and_queries_match_oracle(tmp_path):
    import field_b200.build as B
    import field_b200.expr as X
    import field_b200.query as Q
    from field_b200.grid import GridMeta
    origin, gp = np.array([-0.3, -0.28, -0.12]), 0.01
    arr = _torus_sdf((61, 57, 25), origin, gp)
    npz = _write(tmp_path, "sdf", arr, origin, gp)
    recipe = X.subtract(X.union(X.gridfield(npz, key="sdf", mode="sdf"), X.sphere(0.08, (0.25, 0.1, 0.0))),
                        X.capsule((-0.3, 0.0, 0.0), (0.3, 0.02, 0.01), 0.03))
    comp = X.compile_recipe(recipe)
    assert len(comp.tables) == 1
    meta = GridMeta(-0.34, -0.32, -0.16, 1.0 / 160, 112, 104, 52, 8)  # reaches past the grid's extent
    field = B.FieldBuilder(comp, meta).build()
    hp = comp.host_prims()
    kind, cma = oracle.classify_program(hp, comp.program, meta)
    gk, gc = field.kind.cpu().numpy(), field.corner_min_abs.cpu().numpy()
    bad = np.where(gk != kind)[0]
    assert not len(bad), (f"{len(bad)} kinds differ; first: ids {bad[:6].tolist()}, gpu {gk[bad[:6]].tolist()}, "
                          f"oracle {kind[bad[:6]].tolist()}, oracle min|corner| {cma[bad[:6]].tolist()}, "
                          f"gpu {gc[bad[:6]].tolist()}, margin {meta.margin_mm}")
    n = field.n_active
    ids = field.active[:n].cpu().numpy().astype(np.int32)
    want = oracle.tiles_program(hp, comp.program, meta, ids).reshape(n, -1)
    got = field.tiles[:n].cpu().numpy().astype(np.float64).reshape(n, -1)
    assert int(np.count_nonzero((got >= 0) != (want >= 0))) == 0
    assert _close(got, want, meta.pitch).all(), np.abs(got - want).max() / meta.pitch
    rng = np.random.default_rng(3)
    pts = rng.uniform([-0.4, -0.35, -0.2], [0.4, 0.35, 0.2], (20000, 3))  # some outside the grid
    v = Q.eval_batch(comp, pts)
    w = oracle.eval_points(hp, comp.program, pts.astype(np.float32).astype(np.float64))
    assert _close(v, w, gp).all()


def test_occupancy_mode_and_pitch_precedence(tmp_path):
    import field_b200.expr as X
    import field_b200.query as Q
    rng = np.random.default_rng(5)
    occ = (rng.random((20, 22, 18)) < 0.4).astype(np.float32)
    with_pitch = _write(tmp_path, "occupancy", occ, [0.5, -1.0, 2.0], 0.25)
    pts = rng.uniform([0.5, -1.0, 2.0], [0.5 + 19 * 0.25, -1.0 + 21 * 0.25, 2.0 + 17 * 0.25], (5000, 3))
    for node, pitch in ((X.gridfield(with_pitch, iso=0.5), 0.25), (X.gridfield(with_pitch, iso=0.3, pitch_override=0.2), 0.2)):
        comp = X.compile_recipe(node)
        v = Q.eval_batch(comp, pts)
        w = oracle.eval_points(comp.host_prims(), comp.program, pts.astype(np.float32).astype(np.float64))
        assert _close(v, w, pitch).all()
    # without pitch_mm in the file the reference samples at pitch 1 whatever the override says
    path = tmp_path / "bare.npz"
    np.savez(path, occupancy=occ)
    comp = X.compile_recipe(X.gridfield(str(path), pitch_override=0.2))
    assert comp.prims["p"][0, 3] == 1.0 and (comp.prims["p"][0, :3] == 0).all()


def test_multi_pair_sweep_matches_oracle(tmp_path):
    import field_b200.expr as X
    import field_b200.query as Q
    rng = np.random.default_rng(9)
    leaves, comps = [], []
    for k in range(4):
        origin = rng.uniform(-0.2, 0.0, 3)
        arr = _torus_sdf((30 + k, 28, 26 - k), origin, 0.015)
        path = _write(tmp_path, f"sdf{k}", arr, origin, 0.015)
        leaves.append(X.gridfield(path, key=f"sdf{k}", mode="sdf"))
    pairs = [(0, 1), (2, 3), (1, 3), (0, 2), (3, 3)]
    la = np.array([a for a, _ in pairs], np.int32)
    lb = np.array([b for _, b in pairs], np.int32)
    pts = rng.uniform(-0.25, 0.35, (50000, 3))
    pop = rng.integers(0, len(pairs), len(pts)).astype(np.int32)
    got = Q.eval_batch_multi_pair(pts, pop, la, lb, leaves)
    p32 = pts.astype(np.float32).astype(np.float64)
    for j, (a, b) in enumerate(pairs):
        comp = X.compile_recipe(X.intersect(leaves[a], leaves[b]))
        sel = pop == j
        w = oracle.eval_points(comp.host_prims(), comp.program, p32[sel])
        assert _close(got[sel], w, 0.015).all(), j
    with pytest.raises(ValueError):
        Q.eval_batch_multi_pair(pts[:3], [0, 1, 9], la, lb, leaves)
