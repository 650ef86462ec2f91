"""Continuous-batching server: results alone equal results in the concurrent mix, admission by
budget with LRU eviction, failures fail only their own request (GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _recipe(seed, n_parts=40):
    import field_b200.recipes as R
    import field_b200.expr as X
    rng = np.random.default_rng(seed)
    q = n_parts // 4
    return X.subtract_all(X.union_all(R.parts(rng, q, q, q, n_parts - 3 * q, scale=0.6)), R.tools(rng, 4))


def _requests(fields, rng):
    import field_b200.recipes as R
    reqs = []
    for k in range(24):
        f = fields[k % len(fields)]
        kind = ("query", "edt", "query", "edit")[k % 4]
        if kind == "query":
            reqs.append(("query", dict(field=f, points=rng.uniform(0, 1, size=(20000, 3)).astype(np.float32))))
        elif kind == "edt":
            reqs.append(("edt", dict(field=f)))
        else:
            reqs.append(("edit", dict(field=f, tools=R.tools(rng, 3), op="subtract")))
    return reqs


def _same(a, b):
    if isinstance(a, tuple):
        return all(np.array_equal(x, y) for x, y in zip(a, b))
    return a == b


@pytest.mark.parametrize("arena", [0, 2e9])  # the caching allocator, or resident buffers from an arena
def test_results_alone_equal_results_in_the_mix(arena):
    import field_b200.serve as S
    import field_b200.batch as BT
    metas = [BT.cube_meta(n, b) for n, b in ((64, 8), (128, 8), (96, 4), (128, 16))]
    # run 1: one request at a time
    with S.FieldServer(slots=4) as srv:
        fields = [srv.submit("build", recipe=_recipe(i), meta=m).result(timeout=60)["field"] for i, m in enumerate(metas)]
        reqs = _requests(fields, np.random.default_rng(0))
        alone = [srv.submit(k, **a).result(timeout=60) for k, a in reqs]
    # run 2: the same builds and requests submitted all at once
    with S.FieldServer(slots=4, arena_bytes=arena) as srv:
        futs = [srv.submit("build", recipe=_recipe(i), meta=m) for i, m in enumerate(metas)]
        fields2 = [f.result(timeout=60)["field"] for f in futs]
        assert fields2 == fields
        reqs = _requests(fields2, np.random.default_rng(0))
        futs = [srv.submit(k, **a) for k, a in reqs]
        mixed = [f.result(timeout=60) for f in futs]
    # per field, requests take effect in submission order: every result equals its result alone
    for i, ((k, a), x, y) in enumerate(zip(reqs, alone, mixed)):
        assert _same(x, y), (i, k)


def test_edit_appends_tools_like_a_recompiled_recipe():
    import field_b200.serve as S
    import field_b200.batch as BT
    import field_b200.expr as X
    import field_b200.recipes as R
    meta = BT.cube_meta(96, 8)
    rng = np.random.default_rng(5)
    tools = R.tools(rng, 6)
    pts = rng.uniform(0, 1, size=(5000, 3)).astype(np.float32)
    with S.FieldServer(slots=2) as srv:
        a = srv.submit("build", recipe=_recipe(7), meta=meta).result(timeout=60)["field"]
        srv.submit("edit", field=a, tools=tools, op="subtract").result(timeout=60)
        edited = srv.submit("query", field=a, points=pts).result(timeout=60)
        b = srv.submit("build", recipe=X.subtract_all(_recipe(7), tools), meta=meta).result(timeout=60)["field"]
        direct = srv.submit("query", field=b, points=pts).result(timeout=60)
        assert srv.fields[a].n_active == srv.fields[b].n_active
    assert _same(edited, direct)


def test_budget_admission_evicts_least_recently_used():
    import field_b200.serve as S
    import field_b200.batch as BT
    meta = BT.cube_meta(128, 8)
    with S.FieldServer(slots=2) as srv:
        first = srv.submit("build", recipe=_recipe(0), meta=meta).result(timeout=60)["field"]
        # room for about two resident fields next to one build's admission estimate
        probe = S._Request("build", dict(recipe=None, meta=meta))
        budget = srv._estimate(probe) + 2.5 * srv.fields[first].nbytes
        srv.budget = budget
        ids = [first] + [srv.submit("build", recipe=_recipe(i), meta=meta).result(timeout=60)["field"]
                         for i in range(1, 6)]
        assert srv.resident_bytes() <= budget
        assert ids[0] not in srv.fields  # the oldest field was evicted to admit later builds
        with pytest.raises(KeyError):
            srv.submit("query", field=ids[0], points=np.zeros((4, 3), np.float32)).result(timeout=60)
        v, g = srv.submit("query", field=ids[-1], points=np.full((8, 3), 0.5, np.float32)).result(timeout=60)
        assert v.shape == (8,) and g.shape == (8, 3)


def test_a_failing_request_leaves_the_server_usable():
    import field_b200.serve as S
    import field_b200.batch as BT
    with S.FieldServer(slots=2) as srv:
        fid = srv.submit("build", recipe=_recipe(3), meta=BT.cube_meta(64, 8)).result(timeout=60)["field"]
        with pytest.raises(ValueError):
            srv.submit("edit", field=fid, tools=[], op="intersect").result(timeout=60)
        with pytest.raises(Exception):
            srv.submit("build", recipe={"op": "nonsense"}, meta=BT.cube_meta(64, 8)).result(timeout=60)
        out = srv.submit("edt", field=fid).result(timeout=60)
        assert out["voxels"] == 64 ** 3


def test_arena_ranges_return_when_fields_go():
    import gc
    import field_b200.serve as S
    import field_b200.batch as BT
    with S.FieldServer(slots=2, arena_bytes=1e9) as srv:
        ids = [srv.submit("build", recipe=_recipe(i), meta=BT.cube_meta(96, 8)).result(timeout=60)["field"]
               for i in range(3)]
        srv.submit("edt", field=ids[0]).result(timeout=60)
        srv.submit("edit", field=ids[1], tools=[], op="subtract").result(timeout=60)
        assert srv.arena.used > 0
        srv.fields.clear()
    gc.collect()
    assert srv.arena.used == 0 and srv.arena.free == [(0, srv.arena.nbytes)]


def test_a_full_arena_evicts_idle_fields_instead_of_leaving_it():
    """With the arena full, a build evicts least-recently-used idle fields until its buffers fit;
    every resident buffer stays inside the arena (no device allocation on the request path), and
    the newest field still answers."""
    import gc
    import field_b200.serve as S
    import field_b200.batch as BT
    meta = BT.cube_meta(96, 8)
    with S.FieldServer(slots=2, arena_bytes=2e9) as probe:
        probe.submit("build", recipe=_recipe(0), meta=meta).result(timeout=60)
        per_field = probe.arena.used
    gc.collect()
    with S.FieldServer(slots=2, arena_bytes=int(2.5 * per_field)) as srv:
        base, end = srv.arena.base.data_ptr(), srv.arena.base.data_ptr() + srv.arena.nbytes
        ids = [srv.submit("build", recipe=_recipe(i), meta=meta).result(timeout=60)["field"] for i in range(6)]
        assert ids[0] not in srv.fields and ids[-1] in srv.fields
        assert len(srv.fields) <= 2
        for f in srv.fields.values():
            for t in [f.fb.slab, f.tiles]:
                assert base <= t.data_ptr() and t.data_ptr() + t.numel() * t.element_size() <= end
        v, g = srv.submit("query", field=ids[-1], points=np.full((8, 3), 0.5, np.float32)).result(timeout=60)
        assert v.shape == (8,) and np.isfinite(v).all()


@pytest.mark.parametrize("n", [0, 1, 4097, 1_000_003])
def test_int32_sum_kernel_equals_numpy(n):
    """fb_sum_i32_device, the served EDT request's summary: the exact int64 sum of int32 values
    (negative ones included), its output word zeroed by the call itself."""
    import torch
    import field_b200._lib as L
    rng = np.random.default_rng(n)
    a = rng.integers(-(2 ** 31), 2 ** 31 - 1, size=n, dtype=np.int64).astype(np.int32)
    d = torch.from_numpy(a).cuda() if n else torch.empty(0, dtype=torch.int32, device="cuda")
    out = torch.full((1,), 12345, dtype=torch.int64, device="cuda")  # stale content: the call clears it
    L.check(L.lib().fb_sum_i32_device(d.data_ptr() if n else None, n, out.data_ptr(), L.stream_handle()), "sum")
    assert int(out.item()) == int(a.astype(np.int64).sum())
