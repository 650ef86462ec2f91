"""Batched builds (one CUDA graph over many recipes and streams) equal the recipe-by-recipe path
bit for bit, and the autotuner picks a timed leaf size per bucket (GPU)."""
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


def test_graph_batch_equals_plain_builds():
    import torch
    import field_b200.batch as BT
    recipes = _recipes(12)
    bb = BT.BatchBuilder(recipes, streams=4)
    bb.capture()
    bb.replay()
    torch.cuda.synchronize()
    assert bb.check_counts()
    got = [(it.fb.kind.clone(), it.tiles.clone(), it.mask.clone(), it.edt.clone()) for it in bb.items]
    # recipe by recipe through the single-build path, into the same buffers
    for it in bb.items:
        it.tiles.zero_()
        it.edt.zero_()
    BT.plain_build(bb.items, bb.edt_scratch[0])
    for (kind, tiles, mask, edt), it in zip(got, bb.items):
        assert torch.equal(kind, it.fb.kind)
        assert torch.equal(tiles, it.tiles)
        assert torch.equal(mask, it.mask)
        assert torch.equal(edt, it.edt)
    # one recipe end to end against the oracle: block kinds and the EDT of the occupancy
    comp, meta = recipes[0]
    it = bb.items[0]
    kind, _ = oracle.classify_program(comp.prims, comp.program, meta)
    assert (it.fb.kind.cpu().numpy() == kind).all()
    m = it.mask.cpu().numpy()
    if 0 < m.sum() < m.size:
        assert (it.edt.cpu().numpy() == oracle.edt_squared(1 - m)).all()


def test_build_only_graph_equals_plain_builds():
    """The build-only graph (no occupancy / EDT) gives the same kinds and tiles as the plain
    build-only path, and a builder made without EDT buffers refuses the EDT form."""
    import torch
    import field_b200.batch as BT
    recipes = _recipes(9, seed=17)
    bb = BT.BatchBuilder(recipes, streams=3, edt=False)
    assert all(it.edt is None for it in bb.items)
    bb.replay(edt=False)
    torch.cuda.synchronize()
    assert bb.check_counts()
    got = [(it.fb.kind.clone(), it.tiles.clone()) for it in bb.items]
    for it in bb.items:
        it.tiles.zero_()
    BT.plain_build(bb.items)
    for (kind, tiles), it in zip(got, bb.items):
        assert torch.equal(kind, it.fb.kind)
        assert torch.equal(tiles, it.tiles)
    with pytest.raises(ValueError):
        bb.capture(edt=True)


def test_replays_are_deterministic():
    import torch
    import field_b200.batch as BT
    bb = BT.BatchBuilder(_recipes(6, seed=21), streams=3)
    bb.replay()
    torch.cuda.synchronize()
    first = [it.tiles.clone() for it in bb.items]
    for _ in range(3):
        bb.replay()
    torch.cuda.synchronize()
    assert all(torch.equal(a, it.tiles) for a, it in zip(first, bb.items))


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
