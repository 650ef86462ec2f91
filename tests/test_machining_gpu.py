"""The reference's machining part (src/field_engine/tillverkningsfalt_v1_kernel.py:190-300) built as a
recipe -- round bar, revolved turned-profile table, arched pocket and cross bore -- on the GPU:
block kinds bit-equal to the float64 oracle over the whole grid, leaf values within 1e-5 pitch of
it (plus float32's resolution at the part's 50 mm coordinates), the oracle's recipe evaluation
equal to a float64 restatement of the reference's kernel, and
the reference's negative control (a short drill leaves a plug) (GPU)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _scene(pitch, short=False):
    import field_b200.expr as X
    import field_b200.recipes as R
    recipe, meta, table, c = R.machining_scene(pitch3d=pitch, short_drill=short)
    return X.compile_recipe(recipe), meta, table, c


def _restated(table, c, pts):
    # the table's origin and pitch as the sampler receives them: float32, like the reference kernel's
    f32 = lambda v: float(np.float32(v))
    return oracle.cnc_subtract(table, f32(c["r0_2d"]), f32(c["z0_2d"]), f32(c["pitch2d"]), pts, c["r_blank"], c["z_blank_lo"],
                               c["z_blank_hi"], c["half_x"], c["half_y"], c["arch_r"], c["arch_cz"], c["rho_mill"],
                               c["drill_r"], c["drill_z"], c["drill_x_half"])


@pytest.mark.parametrize("pitch", [0.35, 0.2])  # a small grid; a large one (> 2^17 blocks)
def test_machining_part_matches_oracle_and_reference_kernel(pitch):
    import field_b200.build as B
    comp, meta, table, c = _scene(pitch)
    field = B.FieldBuilder(comp, meta).build()
    hp = comp.host_prims()
    kind, _ = oracle.classify_program(hp, comp.program, meta)
    got = field.kind.cpu().numpy()
    assert (got == kind).all(), f"{int((got != kind).sum())} block decisions differ"
    rng = np.random.default_rng(int(pitch * 100))
    pick = np.sort(rng.choice(field.n_active, size=min(400, field.n_active), replace=False))
    ids = field.active[:field.n_active].cpu().numpy()[pick].astype(np.int32)
    tiles = field.tiles[pick].cpu().numpy().astype(np.float64).reshape(len(pick), -1)
    want = oracle.tiles_program(hp, comp.program, meta, ids).reshape(len(pick), -1)
    assert int(np.count_nonzero((tiles >= 0) != (want >= 0))) == 0
    # the part's coordinates reach 50 mm, where one float32 ulp is 3.8e-6 mm (1.9e-5 of a 0.2 mm pitch),
    # and the arched roof has vertical tangents: values are held to 1e-5 pitch plus 8 such ulps
    tol = TOL * meta.pitch + 8 * float(np.spacing(np.float32(50.0)))
    assert np.abs(tiles - want).max() <= tol
    # the recipe is the reference's kernel: its float64 value equals the literal restatement
    b = meta.block
    bi, rem = np.divmod(ids.astype(np.int64), meta.n_by * meta.n_bz)
    bj, bk = np.divmod(rem, meta.n_bz)
    li, lj, lk = np.indices((b, b, b)).reshape(3, -1)
    ix = (bi[:, None] * b + li[None]).ravel()
    iy = (bj[:, None] * b + lj[None]).ravel()
    iz = (bk[:, None] * b + lk[None]).ravel()
    pts = np.stack([meta.x0 + ix * meta.pitch, meta.y0 + iy * meta.pitch, meta.z0 + iz * meta.pitch], 1)
    assert np.abs(_restated(table, c, pts) - want.ravel()).max() <= 1e-9


def test_short_drill_leaves_a_plug():
    """Negative control of the reference (tillverkningsfalt_v1_kernel.py:238-239): the bore through
    the whole bar removes the material on its axis near the bar's surface; a 30 mm drill does not."""
    import field_b200.build as B
    import field_b200.query as Q
    out = {}
    for short in (False, True):
        comp, meta, table, c = _scene(0.35, short)
        B.FieldBuilder(comp, meta).build()
        pts = np.array([[x, 0.0, c["drill_z"]] for x in (-44.0, -40.0, 40.0, 44.0)])
        out[short] = Q.eval_batch(comp, pts)
        assert np.abs(out[short] - _restated(table, c, pts)).max() <= 1e-4
    assert (out[False] > 0).all()  # bored out
    assert (out[True] < 0).all()   # the plug
