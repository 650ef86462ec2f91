"""Field builds at the benchmark configurations' full sizes, checked against the float64 oracle (GPU).

* The plain single build (256^3, 64 primitives, 8^3 leaves): every block's kind and the ascending
  active ids bit-equal to the oracle's classification of all 32 768 blocks, and every leaf voxel
  within 1e-5 pitch of the float64 value with no sign disagreement.
* The plain method at scale (1024^3, 3584 parts minus 512 milling capsules): the kinds of a two
  block thick slab across the whole grid (32 768 blocks) bit-equal, and 2000 seeded active blocks
  (1 024 000 voxels) within 1e-5 pitch with no sign disagreement.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-5  # of the voxel pitch, against float64


def _leaf_error(comp, meta, field, pick):
    ids = field.active[:field.n_active].cpu().numpy()[pick].astype(np.int32)
    got = field.tiles[pick].cpu().numpy().astype(np.float64).reshape(len(pick), -1)
    want = oracle.tiles_program(comp.prims, comp.program, meta, ids).reshape(len(pick), -1)
    err = np.abs(got - want) / meta.pitch
    sign = int(np.count_nonzero((got >= 0) != (want >= 0)))
    return float(err.max()), sign


def test_plain_single_build_256_full_grid():
    import field_b200.build as B
    import field_b200.expr as X
    import field_b200.recipes as R
    recipe, meta = R.plain_union(seed=0, n=256, block=8)
    comp = X.compile_recipe(recipe)
    fb = B.FieldBuilder(comp, meta)
    field = fb.build()
    kind, _ = oracle.classify_program(comp.prims, comp.program, meta)
    got = field.kind.cpu().numpy()
    assert meta.n_blocks == 32768
    assert (got == kind).all(), f"{int((got != kind).sum())} of {meta.n_blocks} block decisions differ"
    active = np.where(kind == 0)[0]
    assert field.n_active == len(active)
    assert (field.active[:field.n_active].cpu().numpy() == active).all()
    err, sign = _leaf_error(comp, meta, field, np.arange(field.n_active))
    assert sign == 0
    assert err <= TOL, err


def test_plain_method_at_scale_1024():
    import field_b200.build as B
    import field_b200.expr as X
    import field_b200.recipes as R
    recipe, meta = R.milled_part(seed=1, n=1024, block=8)
    comp = X.compile_recipe(recipe)
    fb = B.FieldBuilder(comp, meta)
    field = fb.build()
    kind = field.kind.cpu().numpy()
    # a slab two blocks thick in x through the middle of the part, every block of it
    nbx, nby, nbz = meta.n_bx, meta.n_by, meta.n_bz
    slab = (np.arange(63 * nby * nbz, 65 * nby * nbz)).astype(np.int64)
    want, _ = oracle.classify_blocks(comp.prims, comp.program, meta, slab)
    assert (kind[slab] == want).all(), f"{int((kind[slab] != want).sum())} slab block decisions differ"
    assert (want == 0).sum() > 1000  # the slab crosses the part's surface
    rng = np.random.default_rng(12)
    pick = np.sort(rng.choice(field.n_active, size=2000, replace=False))
    err, sign = _leaf_error(comp, meta, field, pick)
    assert sign == 0
    assert err <= TOL, err
