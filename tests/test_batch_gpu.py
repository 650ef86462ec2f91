"""Batched builds (one launch per phase over work-lists spanning every recipe) equal the
recipe-by-recipe path bit for bit, and the autotuner picks a timed leaf size per bucket (GPU)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _recipes(count, sizes=(64, 128), seed=13):
    import field_b200.recipes as R
    import field_b200.batch as BT
    import field_b200.expr as X
    out = []
    for k, (recipe, n, n_prims) in enumerate(R.batch_recipes(count=count, seed=seed, sizes=sizes)):
        out.append((X.compile_recipe(recipe), BT.cube_meta(n, (4, 8, 16)[k % 3])))
    return out


def _plain_fields(recipes):
    """Recipe by recipe through the single-build path: (kind, active ids, tiles) on the host."""
    import field_b200.build as FB
    out = []
    for comp, meta in recipes:
        f = FB.FieldBuilder(comp, meta).build()
        n = f.n_active
        out.append((f.kind.cpu().numpy(), f.active[:n].cpu().numpy(), f.tiles[:n].cpu().numpy()))
    return out


def _batch_fields(bb):
    off, cnt = bb.tile_offsets(), bb.leaf_counts()
    out = []
    for i in range(len(bb)):
        f = bb.field(i, off, cnt)
        n = f.n_active
        out.append((f.kind.cpu().numpy(), f.active[:n].cpu().numpy(), f.tiles.cpu().numpy()))
    return out


def test_batch_equals_plain_builds():
    """One batched build (work-lists over every recipe, device-side sizing) gives every recipe the
    kinds, ascending active ids and tiles of its own single build, bit for bit -- small grids
    (16-voxel superblocks) and large ones (256^3 at 4^3 leaves and 512^3 at 8^3, above 2^17 blocks)."""
    import torch
    import field_b200.batch as BT
    import field_b200.expr as X
    import field_b200.recipes as R
    recipes = _recipes(9)
    for n, b, seed in ((256, 4, 31), (512, 8, 32)):
        recipe, n_, _ = R.batch_recipes(count=1, seed=seed, sizes=(n,))[0]
        recipes.append((X.compile_recipe(recipe), BT.cube_meta(n, b)))
    bb = BT.BatchBuilder(recipes)
    bb.enqueue()
    torch.cuda.synchronize()
    assert bb.status() == 0
    got = _batch_fields(bb)
    want = _plain_fields(recipes)
    assert any(fb.meta.n_blocks > (1 << 17) for fb in bb.builders)  # a large grid is covered
    for i, ((k1, a1, t1), (k2, a2, t2)) in enumerate(zip(got, want)):
        assert np.array_equal(k1, k2), i
        assert np.array_equal(a1, a2), i
        assert t1.tobytes() == t2.tobytes(), i
    # one small recipe against the oracle
    comp, meta = recipes[0]
    kind, _ = oracle.classify_program(comp.prims, comp.program, meta)
    assert (got[0][0] == kind).all()
    bb.close()


def test_batch_arena_overflow_is_reported_and_recovered():
    import torch
    import field_b200.batch as BT
    recipes = _recipes(6, seed=19)
    bb = BT.BatchBuilder(recipes, capacity=1000)
    bb.enqueue()
    assert bb.status() == 8
    counts = bb.active_counts()
    assert (bb.leaf_counts() <= counts).all() and bb.leaf_counts().sum() < counts.sum()
    assert bb.ensure_capacity()
    assert bb.status() == 0
    assert (bb.leaf_counts() == counts).all()
    got = _batch_fields(bb)
    for (k1, a1, t1), (k2, a2, t2) in zip(got, _plain_fields(recipes)):
        assert np.array_equal(k1, k2) and np.array_equal(a1, a2) and t1.tobytes() == t2.tobytes()


def test_graph_replays_equal_eager_builds_and_are_deterministic():
    import torch
    import field_b200.batch as BT
    bb = BT.BatchBuilder(_recipes(8, seed=21))
    bb.enqueue()
    bb.ensure_capacity()  # the default arena may be short for the 16^3-leaf recipes
    torch.cuda.synchronize()
    eager = [f[2].copy() for f in _batch_fields(bb)]
    bb.tiles.zero_()
    for _ in range(3):
        bb.replay()
    torch.cuda.synchronize()
    assert bb.status() == 0
    assert all(a.tobytes() == f[2].tobytes() for a, f in zip(eager, _batch_fields(bb)))
    assert bb.launches <= 20


def test_batch_with_edt_equals_plain_path():
    """Each recipe followed by its occupancy and the squared EDT of that occupancy: batched
    occupancy and side-stream EDTs equal the recipe-by-recipe path, and one EDT the oracle."""
    import torch
    import field_b200.batch as BT
    recipes = _recipes(7, seed=23)
    bb = BT.BatchBuilder(recipes, edt=True, streams=3)
    bb.enqueue(edt=True)
    bb.ensure_capacity(edt=True)
    bb.replay(edt=True)
    torch.cuda.synchronize()
    assert bb.status() == 0
    masks = [m.clone() for m in bb.masks]
    edts = [e.clone() for e in bb.edts]
    buf = BT.PlainBuffers(bb.builders, bb.active_counts(), edt=True)
    BT.plain_build(buf, bb.edt_scratch[0])
    for i in range(len(bb)):
        assert torch.equal(masks[i], buf.mask[i]), i
        assert torch.equal(edts[i], buf.edt[i]), i
    m = masks[0].cpu().numpy()
    if 0 < m.sum() < m.size:
        assert (edts[0].cpu().numpy() == oracle.edt_squared(1 - m)).all()


def test_autotuner_times_each_bucket(tmp_path):
    import field_b200.batch as BT
    recipes = _recipes(6, sizes=(64,), seed=5)
    tuner = BT.Autotuner(tmp_path / "tune.json")
    blocks = tuner.tune([(c, m.nx) for c, m in recipes])
    assert set(blocks) <= {4, 8, 16}
    for entry in tuner.table.values():
        assert set(entry["ms"]) == {"4", "8", "16"}
        assert entry["block"] == min((int(b) for b in entry["ms"]), key=lambda b: entry["ms"][str(b)])
    again = BT.Autotuner(tmp_path / "tune.json")
    assert again.table == tuner.table


@pytest.mark.parametrize("block,shape", [(4, (37, 41, 45)), (8, (64, 72, 80)), (16, (50, 33, 96)), (8, (40, 40, 29))])
def test_occupancy_matches_the_host_layout(block, shape):
    """The device occupancy mask equals the one read off the host SparseField: tile values < 0 in
    active blocks, kind == -1 elsewhere; ragged grids (rows not a multiple of 16) included."""
    import torch
    import field_b200._lib as L
    import field_b200.build as FB
    import field_b200.recipes as R
    import field_b200.expr as X
    from field_b200.grid import GridMeta
    rng = np.random.default_rng(block + shape[2])
    nx, ny, nz = shape
    meta = GridMeta(0.0, 0.0, 0.0, 1.0 / max(shape), nx, ny, nz, block)
    comp = X.compile_recipe(X.union_all(R.parts(rng, 6, 6, 4, 4, scale=0.8)))
    fb = FB.FieldBuilder(comp, meta)
    field = fb.build()
    slot = torch.empty(meta.n_blocks, dtype=torch.int32, device="cuda")
    mask = torch.empty(shape, dtype=torch.uint8, device="cuda")
    L.check(L.lib().fb_field_occupancy_device(field.kind.data_ptr(), field.active.data_ptr(), field.count.data_ptr(),
                                              field.tiles.data_ptr(), max(field.n_active, 1), nx, ny, nz, block,
                                              slot.data_ptr(), mask.data_ptr(), L.stream_handle()), "occupancy")
    sf = field.to_host()
    nbx, nby, nbz = meta.n_bx, meta.n_by, meta.n_bz
    pad = np.repeat(np.repeat(np.repeat((sf.kind.reshape(nbx, nby, nbz) < 0).astype(np.uint8), block, 0), block, 1),
                    block, 2)
    for t, blk in enumerate(sf.active_ids):
        bi, rem = divmod(int(blk), nby * nbz)
        bj, bk = divmod(rem, nbz)
        pad[bi * block:(bi + 1) * block, bj * block:(bj + 1) * block, bk * block:(bk + 1) * block] = sf.tiles[t] < 0
    want = pad[:nx, :ny, :nz]
    assert 0 < want.sum() < want.size
    assert np.array_equal(mask.cpu().numpy(), want)
