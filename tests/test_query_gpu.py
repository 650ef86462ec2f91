"""Point queries (eval_batch, gradient_batch, accelerated resident queries) and per-block-pitch
fields (avstand, gradient) against the float64 oracle and the reference's own formulas (GPU)."""
import json

import numpy as np
import pytest

import oracle
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_eval_batch_matches_reference_evaluator():
    """The reference's eval_sdf_py values at 3000 seeded points per tree (float32 evaluation;
    the reference's own gate is 1e-3, src/field_engine/ikarus_v1/eval_warp.py:737-775)."""
    import field_b200.query as Q
    g = np.load(GOLDEN / "expr_golden.npz")
    trees = json.loads((GOLDEN / "expr_golden.json").read_text())
    for name, tree in trees.items():
        pts = g[f"{name}__points"]
        got = Q.eval_batch(tree, pts)
        err = np.abs(got.astype(np.float64) - g[f"{name}__values"]).max()
        assert err < 2e-5, (name, err)


def test_gradient_batch_matches_float64_central_difference():
    import field_b200.query as Q
    import field_b200.expr as X
    trees = json.loads((GOLDEN / "expr_golden.json").read_text())
    rng = np.random.default_rng(2)
    for name in ("selftest_smooth", "cone_x", "frustum"):
        tree = trees[name]
        pts = rng.uniform(-20, 20, size=(2000, 3)).astype(np.float32).astype(np.float64)
        got = Q.gradient_batch(tree, pts, h=0.05)
        comp = X.compile_recipe(tree)
        want = np.zeros_like(got, dtype=np.float64)
        for a in range(3):
            d = np.zeros(3)
            d[a] = 0.05
            p = (pts + d).astype(np.float32).astype(np.float64)
            m = (pts - d).astype(np.float32).astype(np.float64)
            want[:, a] = (oracle.eval_points(comp.prims, comp.program, p) -
                          oracle.eval_points(comp.prims, comp.program, m)) / 0.1
        assert np.abs(got - want).max() < 2e-3, name


# 256^3 / B8: every block keeps a culled list (warp-per-block cull); 512^3 / B8: only surface blocks do
@pytest.mark.parametrize("n", [256, 512])
def test_accelerated_queries_equal_full_chain(n):
    import torch
    import field_b200.build as B
    import field_b200.query as Q
    import field_b200.recipes as R
    recipe, meta = R.milled_part(seed=3, n=n, block=8, n_parts=512, n_tools=64)
    fb = B.FieldBuilder(recipe, meta)
    fb.classify()
    plain = Q.RecipeQueries(fb.compiled)
    fast = Q.RecipeQueries(fb.compiled, builder=fb)
    g = torch.Generator(device="cuda").manual_seed(4)
    pts = torch.rand((200000, 3), device="cuda", generator=g) * 1.1 - 0.05  # some outside the grid
    a = plain.values(pts)
    b = fast.values(pts)
    assert torch.equal(a, b)
    va, ga = plain.values_and_gradients(pts[:50000], h=1e-3)
    vb, gb = fast.values_and_gradients(pts[:50000], h=1e-3)
    assert torch.equal(va, vb) and torch.equal(ga, gb)
    comp = fb.compiled
    sel = pts[:3000].double().cpu().numpy().astype(np.float32).astype(np.float64)
    want = oracle.eval_points(comp.prims, comp.program, sel)
    assert np.abs(b[:3000].cpu().numpy() - want).max() < 1e-6


def _multires_check(F, recipe, n_check=12, seed=0):
    """Lattice values of a sample of active bricks against the float64 oracle.  Returns (worst error
    in units of the brick's pitch inside the 3-voxel band, worst error relative to max(|d|, pitch)
    anywhere, sign disagreements)."""
    import field_b200.expr as X
    comp = X.compile_recipe(recipe)
    tiles = F.tiles
    rng = np.random.default_rng(seed)
    ids = sorted(tiles)
    worst = 0.0
    rel = 0.0
    sign = 0
    for u in rng.choice(ids, size=min(n_check, len(ids)), replace=False):
        u = int(u)
        bi, bj, bk = np.unravel_index(u, F.brick_shape)
        lvl = int(F.niva[bi, bj, bk])
        pitch = F.h_grov / (1 << lvl)
        m = tiles[u].shape[0]
        idx = np.indices((m, m, m)).reshape(3, -1).T
        o = F.lo + np.array([bi, bj, bk]) * F.L
        pts = o + idx * pitch
        want = oracle.eval_points(comp.prims, comp.program, pts)
        got = tiles[u].reshape(-1).astype(np.float64)
        err = np.abs(got - want)
        band = np.abs(want) <= 3 * pitch
        if band.any():
            worst = max(worst, float(err[band].max() / pitch))
        rel = max(rel, float((err / np.maximum(np.abs(want), pitch)).max()))
        sign += int(np.count_nonzero((got >= 0) != (want >= 0)))
    return worst, rel, sign


def test_multires_tiles_and_queries():
    import field_b200.multires as M
    import field_b200.recipes as R
    import field_b200.expr as X
    rng = np.random.default_rng(9)
    recipe = X.union_all(R.parts(rng, 12, 12, 6, 6, scale=0.8))
    F = M.bygg_multires_fran_recept(recipe, [0, 0, 0], 1.0 / 64, (8, 8, 8), block=8,
                                    levels=lambda lens: M.levels_by_list_length(lens, (2, 3)), overlappsband=False)
    assert F.stats["n_active"] > 0
    worst, rel, sign = _multires_check(F, recipe)
    assert sign == 0 and worst <= 1e-5 and rel <= 1e-5, (worst, rel)
    tiles = F.tiles
    pts = rng.uniform(-0.05, 1.05, size=(4000, 3))
    # points exactly on brick faces exercise the active-brick preference
    pts[:200, 0] = np.round(pts[:200, 0] * 8) / 8
    args = (F.lo, F.h_grov, F.block, F.brick_shape, F.kind, F.niva, tiles, F.margin_mm)
    got = M.avstand(F, pts)
    want = oracle.multires_avstand(*args, pts)
    bad = np.flatnonzero(got != want)
    assert not len(bad), (len(bad), pts[bad[:3]], got[bad[:3]], want[bad[:3]])
    g = M.gradient(F, pts[:1000])
    gw = oracle.multires_gradient(*args, pts[:1000])
    assert np.allclose(g, gw, rtol=1e-12, atol=1e-9)


def test_precision_stress_near_tangent_pairs_and_thin_walls():
    """Near-tangent sphere pairs (gap U[0, 0.5] * fine pitch) and walls half a fine voxel thick, at
    a mixed per-block pitch of 1/128 and 1/512: values within 1e-5 of the fine pitch of float64 and
    no sign disagreement, on sampled bricks of both levels."""
    import field_b200.multires as M
    import field_b200.recipes as R
    recipe = R.tangent_pairs(seed=4, n_pairs=150, pitch=1.0 / 512, walls=16)
    F = M.bygg_multires_fran_recept(recipe, [0, 0, 0], 1.0 / 128, (16, 16, 16), block=8, overlappsband=False,
                                    levels=lambda lens: np.where(np.asarray(lens) >= 2, 2, 0))
    assert F.stats["levels"][2] > 0 and F.stats["levels"][0] > 0
    worst, rel, sign = _multires_check(F, recipe, n_check=16, seed=1)
    assert sign == 0
    assert worst <= 1e-5 and rel <= 1e-5, (worst, rel)


def test_multires_overlap_band_and_continuity_match_oracle():
    """The overlap band on the device equals the reference's sequential band (restated with scipy's
    map_coordinates) lattice for lattice, bit for bit, and kontinuitetscheck's jumps equal the
    oracle-evaluated ones; with the band the jump across pitch changes stays within the reference's
    bound (half the coarser pitch)."""
    import field_b200.multires as M
    import field_b200.recipes as R
    import field_b200.expr as X
    rng = np.random.default_rng(12)
    recipe = X.union_all(R.parts(rng, 14, 12, 6, 6, scale=0.8))
    lv = lambda lens: M.levels_by_list_length(lens, (2, 3))
    F0 = M.bygg_multires_fran_recept(recipe, [0, 0, 0], 1.0 / 64, (8, 8, 8), block=8, levels=lv, overlappsband=False)
    F = M.bygg_multires_fran_recept(recipe, [0, 0, 0], 1.0 / 64, (8, 8, 8), block=8, levels=lv)
    assert len(set(F.niva[F.kind == 0].ravel())) >= 3  # levels 0, 1 and 2 meet
    want, faces = oracle.multires_overlap_band(F0.lo, F0.h_grov, F0.block, F0.brick_shape, F0.kind, F0.niva, F0.tiles)
    assert faces > 0 and F.stats["overlap_faces"] == faces
    got = F.tiles
    assert sorted(got) == sorted(want)
    for k in want:
        assert got[k].tobytes() == want[k].tobytes(), k
    rep = M.kontinuitetscheck(F)
    assert rep["n_pitchbyten_faces"] == faces and rep["GRON"]
    # the same jumps from the oracle's avstand
    args = (F.lo, F.h_grov, F.block, F.brick_shape, F.kind, F.niva, want, F.margin_mm)
    pts = np.array([[0.2, 0.3, 0.4]])
    assert oracle.multires_avstand(*args, pts)[0] == M.avstand(F, pts)[0]
