"""Host-side logic without a GPU: edits appended to a compiled recipe equal the recompiled edited
recipe byte for byte, edit tools must be single primitives, and the server's pinned staging pool
recycles a block only once its result array is gone."""
import numpy as np
import pytest


def _base(seed):
    import field_b200.expr as X
    import field_b200.recipes as R
    rng = np.random.default_rng(seed)
    return X.union_all(R.parts(rng, 4, 3, 3, 2, scale=0.6)), rng


@pytest.mark.parametrize("op", ["subtract", "union"])
def test_extend_equals_recompiled_recipe(op):
    import field_b200.expr as X
    import field_b200.recipes as R
    base, rng = _base(1)
    tools = R.tools(rng, 7)
    edited = base
    for t in tools:
        edited = X.subtract(edited, t) if op == "subtract" else X.union(edited, t)
    want = X.compile_recipe(edited)
    got = X.extend(X.compile_recipe(base), X.compile_tools(tools), op)
    for key in ("prims", "chain", "program"):
        assert np.array_equal(getattr(want, key).view(np.uint8), getattr(got, key).view(np.uint8)), key


def test_extend_twice_equals_one_recompile():
    import field_b200.expr as X
    import field_b200.recipes as R
    base, rng = _base(2)
    t1, t2 = R.tools(rng, 3), R.tools(rng, 4)
    got = X.extend(X.extend(X.compile_recipe(base), X.compile_tools(t1)), X.compile_tools(t2))
    want = X.compile_recipe(X.subtract_all(X.subtract_all(base, t1), t2))
    for key in ("prims", "chain", "program"):
        assert np.array_equal(getattr(want, key).view(np.uint8), getattr(got, key).view(np.uint8)), key


def test_extend_keeps_non_chain_recipes_as_programs():
    import field_b200.expr as X
    import field_b200.recipes as R
    base, rng = _base(3)
    # a smooth union whose right operand is itself a union has no chain form
    smooth = X.union(base, X.union(X.sphere(0.1, (0.5, 0.5, 0.5)), X.sphere(0.05, (0.3, 0.5, 0.5))), k=0.02)
    comp = X.compile_recipe(smooth)
    assert comp.chain is None
    tools = R.tools(rng, 2)
    got = X.extend(comp, X.compile_tools(tools))
    want = X.compile_recipe(X.subtract_all(smooth, tools))
    assert got.chain is None
    assert np.array_equal(want.program.view(np.uint8), got.program.view(np.uint8))
    assert np.array_equal(want.prims.view(np.uint8), got.prims.view(np.uint8))


def test_composite_tools_and_bad_ops_are_rejected():
    import field_b200.expr as X
    base, _ = _base(4)
    with pytest.raises(ValueError):
        X.compile_tools([X.union(X.sphere(0.1), X.sphere(0.2, (0.3, 0.0, 0.0)))])
    with pytest.raises(ValueError):
        X.extend(X.compile_recipe(base), X.compile_tools([X.sphere(0.1)]), "intersect")


def test_pinned_pool_recycles_a_block_when_its_array_is_dropped():
    """Query results are numpy views of pooled pinned blocks: a block stays out of the pool while
    the array (or any slice of it) lives, and the next request of that size class reuses it."""
    import gc
    import torch
    import field_b200.serve as S

    class HostPool(S.PinnedPool):  # plain host memory: the recycling rule needs no GPU
        def _new(self, cls):
            return torch.empty(cls, dtype=torch.uint8)

    pool = HostPool()
    view, handle = pool.take(1000)
    arr = view.view(torch.float32).numpy()
    pool.bind(arr, handle)
    part = arr[10:]
    del arr, view
    gc.collect()
    assert sum(len(v) for v in pool.free.values()) == 0  # the slice still holds it
    del part
    gc.collect()
    assert sum(len(v) for v in pool.free.values()) == 1
    _, again = pool.take(900)
    assert again[1].data_ptr() == handle[1].data_ptr()
    assert pool.allocated == S.PinnedPool.MIN
    _, other = pool.take(S.PinnedPool.MIN + 1)  # the next size class: a new block
    assert other[0] == 2 * S.PinnedPool.MIN and pool.allocated == 3 * S.PinnedPool.MIN
    pool.give_back(other)
    _, small = pool.take(10)  # its own class is empty: the next class's free block serves it
    assert small[0] == 2 * S.PinnedPool.MIN and pool.allocated == 3 * S.PinnedPool.MIN
    pool.give_back(small)
    pool.reserve(S.PinnedPool.MIN * 64, 2)  # reserve allocates blocks of its own class
    assert len(pool.free[S.PinnedPool.MIN * 64]) == 2
    _, tiny = pool.take(10)  # 64 classes up is beyond the span: the 2*MIN block, not a reserved one
    assert tiny[0] == 2 * S.PinnedPool.MIN and len(pool.free[S.PinnedPool.MIN * 64]) == 2


def test_mesh_window_rule():
    """field_b200.mesh.window: floor/ceil of the vertex range in pitches from `lo`, widened by the
    margin (and one more voxel above), clamped to a global grid when one is given, never negative
    in extent (faltkarna_v1_mesh_to_sdf.py:153-166)."""
    import field_b200.mesh as M
    V = np.array([[0.25, 1.0, -0.5], [2.0, 1.75, 0.5]])
    gmin, shape = M.window(V, 0.5, np.zeros(3), margin_vox_pad=2)
    # x: floor(0.5) - 2 = -2 .. ceil(4) + 3 = 7; y: 2 - 2 = 0 .. 4 + 3 = 7; z: -1 - 2 = -3 .. 1 + 3 = 4
    assert list(gmin) == [-2, 0, -3] and shape == (9, 7, 7)
    gmin, shape = M.window(V, 0.5, np.zeros(3), global_shape=(5, 100, 2), margin_vox_pad=2)
    assert list(gmin) == [0, 0, 0] and shape == (5, 7, 2)
    far = V + 100.0  # entirely above a small global grid: empty extent, not negative
    gmin, shape = M.window(far, 0.5, np.zeros(3), global_shape=(4, 4, 4))
    assert shape == (0, 0, 0)
