"""Mesh -> signed distance field on the GPU (libfield_b200's meshsdf_field_cpu through field_b200.mesh)
against the reference's own meshsdf_field_cpu compiled from mesh_sdf_native_v1/field.cpp (oracle/_ref):
solid, surface layer, statistics and sd bits equal on seeded closed meshes (non-dyadic pitches, a
1e6 mm offset for the local-z path, both surface-correction settings), the window and status
contract of field_stage, and a window without a solid voxel."""
import numpy as np
import pytest

import oracle
import field_b200.recipes as R

pytestmark = pytest.mark.gpu

CASES = [(0, 0.3137, 0.0, True), (1, 0.17, 0.0, False), (2, 0.25, 1.0e6, True), (3, 0.1234, 0.0, True),
         (4, 0.41, -2.5e5, False)]


def _grid(V, pitch):
    import field_b200.mesh as M
    lo = V.min(0) - 2 * pitch
    gmin, shape = M.window(V, pitch, lo)
    return lo + gmin * pitch, shape, (pitch * M.JITTER_FRAC * M.GOLDEN[0], pitch * M.JITTER_FRAC * M.GOLDEN[1])


@pytest.mark.parametrize("seed,pitch,offset,corr", CASES)
def test_mesh_field_equals_the_reference(seed, pitch, offset, corr):
    import field_b200.mesh as M
    V, T = R.mesh_scene(seed, offset)
    origin, shape, jit = _grid(V, pitch)
    rc, solid, sd, yta, stats = oracle.ref_mesh_field(V, T, origin, pitch, jit, shape, corr)
    assert rc == 0
    g_solid, g_sd, g_yta, g_stats, ts = M.field_grid(V, T, origin, pitch, shape, jitter=jit, surface_correction=corr)
    assert np.array_equal(g_solid, solid)
    assert np.array_equal(g_yta, yta)
    assert np.array_equal(g_stats, stats)
    assert 0 < stats[3] < solid.size and stats[1] > 0
    assert g_sd.tobytes() == sd.tobytes()
    assert len(ts) == 5 and (ts >= 0).all()


def test_field_stage_window_and_contract():
    import field_b200.mesh as M
    V, T = R.mesh_scene(5)
    pitch, lo = 0.27, np.array([-3.0, -1.0, 0.5])
    gmin, shape, yta, solid, sd, diag = M.field_stage(V, T, pitch, lo)
    origin = lo + gmin * pitch
    rc, r_solid, r_sd, r_yta, stats = oracle.ref_mesh_field(
        V, T, origin, pitch, (pitch * M.JITTER_FRAC * M.GOLDEN[0], pitch * M.JITTER_FRAC * M.GOLDEN[1]), shape)
    assert rc == 0 and np.array_equal(solid, r_solid) and np.array_equal(yta, r_yta)
    assert sd.tobytes() == r_sd.tobytes()
    assert diag["n_traffar"] == stats[1] and diag["n_par"] == stats[0] and not diag["one_class"]
    # clamped to a global window: the local window shrinks, the field is that of the clamped grid
    g2, shape2, *_ = M.field_stage(V, T, pitch, lo, global_shape=(40, 60, 50))
    assert (g2 >= 0).all() and all(a <= b for a, b in zip(np.add(g2, shape2), (40, 60, 50)))
    with pytest.raises(ValueError):
        M.field_stage(V, T + len(V), pitch, lo)  # face index outside [0, nv): status 2
    with pytest.raises(ValueError):
        M.field_grid(V, T, (0, 0, 0), -1.0, (8, 8, 8))  # status 1
    bad = V.copy()
    bad[0, 0] = np.nan
    with pytest.raises(ValueError):
        M.field_stage(bad, T, pitch, lo)


def test_window_without_solid_voxel():
    """A sphere smaller than a voxel between samples: no solid voxel; the kernel's convention
    (-1 to the missing class, 0 to the other) equals the reference's."""
    import field_b200.mesh as M
    V, T = R.mesh_sphere((0.05, 0.05, 0.05), 0.02, 8, 16)
    pitch = 0.1
    origin, shape, jit = _grid(V, pitch)
    rc, solid, sd, yta, stats = oracle.ref_mesh_field(V, T, origin, pitch, jit, shape, True)
    g_solid, g_sd, g_yta, g_stats, _ = M.field_grid(V, T, origin, pitch, shape, jitter=jit)
    assert rc == 0 and stats[3] == 0
    assert np.array_equal(g_solid, solid) and np.array_equal(g_stats, stats)
    assert g_sd.tobytes() == sd.tobytes()


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_windows_over_512_voxels_equal_the_reference(axis):
    """A long bar with spheres along it: a window of 700+ voxels on one axis (the banded EDT serves
    512; these take the long-axis passes).  Solid, surface, statistics and sd bytes equal the
    reference's, which accepts any grid below 2^31 cells."""
    import field_b200.mesh as M
    lo, hi = np.array([0.0, 0.0, 0.0]), np.array([3.0, 2.5, 2.0])
    hi[axis] = 70.0
    parts = [R.mesh_box(lo, hi)]
    for t in (0.2, 0.5, 0.8):
        c = (lo + hi) / 2
        c[axis] = t * hi[axis]
        parts.append(R.mesh_sphere(c, 3.1 + t, 16, 32))
    V, T = R.mesh_merge(*parts)
    pitch = 0.097
    origin, shape, jit = _grid(V, pitch)
    assert shape[axis] > 512 and max(shape[a] for a in range(3) if a != axis) <= 512
    rc, solid, sd, yta, stats = oracle.ref_mesh_field(V, T, origin, pitch, jit, shape, True)
    assert rc == 0
    g_solid, g_sd, g_yta, g_stats, _ = M.field_grid(V, T, origin, pitch, shape, jitter=jit)
    assert np.array_equal(g_solid, solid)
    assert np.array_equal(g_yta, yta)
    assert np.array_equal(g_stats, stats)
    assert 0 < stats[3] < solid.size
    # one float32 ulp where sqrt(n) pitch and the reference's offset form round to either side
    a, b = g_sd.view(np.int32).astype(np.int64), sd.view(np.int32).astype(np.int64)
    assert int(np.abs(a - b).max()) <= 1
    assert np.count_nonzero(a != b) <= 1e-4 * a.size
