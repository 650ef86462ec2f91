"""Seeded synthetic workloads with the shapes, sizes and value distributions of the benchmark
configurations (no external dataset is involved).

* ``plain_union``  -- spheres (centres U[0.1,0.9]^3, radii U[0.02,0.1]) and axis-aligned boxes
  (half extents U[0.02,0.08]) in a unit-cube domain, one hard union; 256^3 at pitch 1/256, 8^3
  leaves, seed 0 for the plain single build.
* ``milled_part``  -- the plain method at scale: spheres, boxes, capsules and tori in equal numbers
  with the same distributions scaled by 1/4, unioned, then milling-tool capsules (radius
  U[0.005,0.02], straight sweeps with endpoints U[0.05,0.95]^3) subtracted in order.
* ``obstacle_grid``-- a uint8 occupancy grid of random boxes, scaled to a target fill fraction.
* ``batch_recipes``-- many independent recipes: primitive counts log-uniform in [8, 2048], domains
  from {64, 128, 256, 512}^3, each part followed by tool subtractions.
* ``tangent_pairs``-- adversarial near-tangent sphere pairs (gap U[0, 0.5]*pitch) and thin box walls.
"""
from __future__ import annotations

import math

import numpy as np

from . import expr as X
from .grid import GridMeta


def _unit_vectors(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def parts(rng, n_sphere, n_box, n_capsule=0, n_torus=0, scale=1.0, lo=0.1, hi=0.9):
    """Primitive nodes: spheres, boxes, capsules, tori with the plain-build distributions x scale."""
    out = []
    c = rng.uniform(lo, hi, size=(n_sphere, 3))
    r = rng.uniform(0.02, 0.1, size=n_sphere) * scale
    out += [X.sphere(float(r[i]), c[i]) for i in range(n_sphere)]
    c = rng.uniform(lo, hi, size=(n_box, 3))
    h = rng.uniform(0.02, 0.08, size=(n_box, 3)) * scale
    out += [X.box(h[i], c[i]) for i in range(n_box)]
    if n_capsule:
        c = rng.uniform(lo, hi, size=(n_capsule, 3))
        d = _unit_vectors(rng, n_capsule) * rng.uniform(0.02, 0.08, size=(n_capsule, 1)) * scale
        r = rng.uniform(0.01, 0.04, size=n_capsule) * scale
        out += [X.capsule(c[i] - d[i], c[i] + d[i], float(r[i])) for i in range(n_capsule)]
    if n_torus:
        c = rng.uniform(lo, hi, size=(n_torus, 3))
        R = rng.uniform(0.04, 0.1, size=n_torus) * scale
        rr = R * rng.uniform(0.15, 0.4, size=n_torus)
        axes = rng.integers(0, 3, size=n_torus)
        out += [X.torus(float(R[i]), float(rr[i]), "xyz"[axes[i]], c[i]) for i in range(n_torus)]
    return out


def tools(rng, n, r_lo=0.005, r_hi=0.02, lo=0.05, hi=0.95):
    """Milling-tool passes: capsules along random straight sweeps."""
    a = rng.uniform(lo, hi, size=(n, 3))
    b = rng.uniform(lo, hi, size=(n, 3))
    r = rng.uniform(r_lo, r_hi, size=n)
    return [X.capsule(a[i], b[i], float(r[i])) for i in range(n)]


def plain_union(seed=0, n=256, block=8, n_sphere=32, n_box=32):
    """(recipe, GridMeta) of the plain single build."""
    rng = np.random.default_rng(seed)
    nodes = parts(rng, n_sphere, n_box)
    meta = GridMeta(0.0, 0.0, 0.0, 1.0 / n, n, n, n, block)
    return X.union_all(nodes), meta


def milled_part(seed=1, n=1024, block=8, n_parts=3584, n_tools=512):
    """(recipe, GridMeta) of the plain method at scale: n_parts primitives in equal mix, unioned,
    minus n_tools milling capsules."""
    rng = np.random.default_rng(seed)
    q = n_parts // 4
    nodes = parts(rng, q, q, q, n_parts - 3 * q, scale=0.25)
    order = rng.permutation(len(nodes))
    recipe = X.union_all([nodes[i] for i in order])
    recipe = X.subtract_all(recipe, tools(rng, n_tools))
    meta = GridMeta(0.0, 0.0, 0.0, 1.0 / n, n, n, n, block)
    return recipe, meta


def _raster_boxes(n, centres, half):
    g = np.zeros((n, n, n), np.uint8)
    lo = np.clip(np.floor(centres - half), 0, n).astype(int)
    hi = np.clip(np.ceil(centres + half), 0, n).astype(int)
    for i in range(len(centres)):
        g[lo[i, 0]:hi[i, 0], lo[i, 1]:hi[i, 1], lo[i, 2]:hi[i, 2]] = 1
    return g


def obstacle_grid(seed=2, n=512, n_boxes=2000, fill=0.08):
    """uint8 (n, n, n) occupancy of n_boxes random boxes whose size is scaled (bisection on a coarse
    raster, then on the full one) so that the filled fraction is close to ``fill``."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, 1, size=(n_boxes, 3))
    shape = rng.uniform(0.5, 1.5, size=(n_boxes, 3))

    def frac(res, s):
        return _raster_boxes(res, centres * res, shape * s * res).mean()
    lo, hi = 0.0, 0.5
    coarse = max(32, n // 4)
    for _ in range(24):
        s = 0.5 * (lo + hi)
        lo, hi = (s, hi) if frac(coarse, s) < fill else (lo, s)
    lo, hi = 0.5 * lo, 2.0 * hi
    for _ in range(10 if n <= 256 else 7):
        s = 0.5 * (lo + hi)
        lo, hi = (s, hi) if frac(n, s) < fill else (lo, s)
    return _raster_boxes(n, centres * n, shape * 0.5 * (lo + hi) * n)


def batch_recipes(count=256, seed=3, sizes=(64, 128, 256, 512), tool_fraction=0.125):
    """List of (recipe, n, n_prims): primitive counts log-uniform in [8, 2048], cubic domains
    drawn uniformly from ``sizes``; a fraction of the primitives are milling tools subtracted
    after the union of the parts."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n_prims = int(round(math.exp(rng.uniform(math.log(8), math.log(2048)))))
        n = int(rng.choice(sizes))
        n_tools = int(n_prims * tool_fraction)
        n_parts = max(1, n_prims - n_tools)
        # keep the part count per unit volume bounded: primitive size shrinks with the count
        scale = float(min(1.0, (64.0 / n_parts) ** (1.0 / 3.0)))
        q = n_parts // 4
        nodes = parts(rng, n_parts - 3 * q, q, q, q, scale=scale)
        recipe = X.union_all(nodes)
        if n_tools:
            recipe = X.subtract_all(recipe, tools(rng, n_tools, 0.005 * max(scale, 0.25), 0.02 * max(scale, 0.25)))
        out.append((recipe, n, n_parts + n_tools))
    return out


def tangent_pairs(seed=4, n_pairs=1000, pitch=1.0 / 512, walls=64):
    """Adversarial thin features: sphere pairs whose gap is U[0, 0.5]*pitch and box walls half a
    voxel thick, in the unit cube.  Returns a recipe (union of everything)."""
    rng = np.random.default_rng(seed)
    nodes = []
    for _ in range(n_pairs):
        c = rng.uniform(0.1, 0.9, size=3)
        r1, r2 = rng.uniform(0.004, 0.02, size=2)
        d = _unit_vectors(rng, 1)[0]
        gap = rng.uniform(0.0, 0.5) * pitch
        nodes.append(X.sphere(r1, c))
        nodes.append(X.sphere(r2, c + d * (r1 + r2 + gap)))
    for _ in range(walls):
        c = rng.uniform(0.1, 0.9, size=3)
        h = rng.uniform(0.01, 0.05, size=3)
        h[rng.integers(0, 3)] = 0.25 * pitch
        nodes.append(X.box(h, c))
    return X.union_all(nodes)


# ------------------------------------------------------------------------------------ meshes
# Closed, outward-oriented triangle meshes (float64 vertices, int64 faces) for the mesh -> field stage.

def mesh_sphere(center, radius, n_theta=24, n_phi=48):
    """UV sphere."""
    th = np.linspace(0, np.pi, n_theta + 1)[1:-1]
    ph = np.linspace(0, 2 * np.pi, n_phi, endpoint=False)
    ring = np.stack([np.outer(np.sin(th), np.cos(ph)), np.outer(np.sin(th), np.sin(ph)),
                     np.outer(np.cos(th), np.ones_like(ph))], axis=-1).reshape(-1, 3)
    V = np.vstack([[0, 0, 1], ring, [0, 0, -1]]) * radius + np.asarray(center)
    top, bot = 0, len(V) - 1
    idx = lambda i, j: 1 + i * n_phi + (j % n_phi)
    T = []
    for j in range(n_phi):
        T.append((top, idx(0, j), idx(0, j + 1)))
        T.append((bot, idx(n_theta - 2, j + 1), idx(n_theta - 2, j)))
    for i in range(n_theta - 2):
        for j in range(n_phi):
            a, b, c, d = idx(i, j), idx(i, j + 1), idx(i + 1, j), idx(i + 1, j + 1)
            T.append((a, c, b))
            T.append((b, c, d))
    return V.astype(np.float64), np.asarray(T, np.int64)


def mesh_box(lo, hi):
    """Axis-aligned box, 12 triangles."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    V = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
    T = np.array([(0, 1, 3), (0, 3, 2), (4, 6, 7), (4, 7, 5), (0, 4, 5), (0, 5, 1),
                  (2, 3, 7), (2, 7, 6), (0, 2, 6), (0, 6, 4), (1, 5, 7), (1, 7, 3)], np.int64)
    return V, T


def mesh_torus(center, R, r, n_u=48, n_v=24):
    """Torus around the z axis through `center`."""
    u = np.linspace(0, 2 * np.pi, n_u, endpoint=False)
    v = np.linspace(0, 2 * np.pi, n_v, endpoint=False)
    uu, vv = np.meshgrid(u, v, indexing="ij")
    V = np.stack([(R + r * np.cos(vv)) * np.cos(uu), (R + r * np.cos(vv)) * np.sin(uu), r * np.sin(vv)], -1)
    V = V.reshape(-1, 3) + np.asarray(center)
    idx = lambda i, j: (i % n_u) * n_v + (j % n_v)
    T = []
    for i in range(n_u):
        for j in range(n_v):
            a, b, c, d = idx(i, j), idx(i + 1, j), idx(i, j + 1), idx(i + 1, j + 1)
            T.append((a, b, d))
            T.append((a, d, c))
    return V.astype(np.float64), np.asarray(T, np.int64)


def mesh_merge(*meshes):
    """One mesh of several (face indices offset)."""
    Vs, Ts, off = [], [], 0
    for V, T in meshes:
        Vs.append(V)
        Ts.append(T + off)
        off += len(V)
    return np.vstack(Vs), np.vstack(Ts)


def mesh_scene(seed=0, offset=0.0, fine=1):
    """A sphere, a rotated box and a torus in a ~20 mm region (mm units), moved by `offset`."""
    rng = np.random.default_rng(seed)
    s = mesh_sphere(rng.uniform(4, 6, 3), rng.uniform(2.5, 3.5), 24 * fine, 48 * fine)
    b = mesh_box(rng.uniform(9, 10, 3), rng.uniform(13, 15, 3))
    th = rng.uniform(0.2, 0.8)
    Rz = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    c = b[0].mean(0)
    b = ((b[0] - c) @ Rz.T + c, b[1])
    t = mesh_torus(rng.uniform(5, 7, 3) + np.array([0, 8, 0]), rng.uniform(3, 4), rng.uniform(0.8, 1.4), 48 * fine, 24 * fine)
    V, T = mesh_merge(s, b, t)
    return V + offset, T


# ------------------------------------------------------------------------------------ machining scene
# The reference's machining test part (src/field_engine/tillverkningsfalt_v1_kernel.py:56-118, :190-236):
# a stepped shaft with three ring grooves, turned from a round bar with a 1 mm nose radius, a pocket
# milled with a 3 mm end mill under an arched roof, and a cross bore.
MACHINING = dict(rho_turn=1.0, rho_mill=3.0, drill_r=11.15, radial_allowance=1.5, axial_allowance=1.0,
                 pitch2d=0.04, r_land=47.7, r_groove=45.5, groove_w=3.0, z_lo=-21.0, z_hi=32.0,
                 groove_centers=(14.0, 19.0, 24.0), half_x=10.4, half_y=23.0, arch_r=10.4, roof_z=17.6,
                 drill_z=11.15, drill_x_short=30.0)


def turned_profile_table(c=MACHINING):
    """(sdf2d float32 (nr, nz), r0, z0) of the turned profile: the sharp-cornered (r, z) profile
    rasterised at pitch2d, closed with a disk of the nose radius (what a nose-radius tool reaches:
    convex corners sharp, concave ones rounded), then signed by exact Euclidean distance transforms
    (negative inside) -- the construction of tillverkningsfalt_v1_kernel.py:91-131.  The closing is
    dilation then erosion by thresholding exact distances (outside-the-raster pixels ignored)."""
    from scipy import ndimage
    poly = [(c["z_lo"], c["r_land"])]
    for zc in c["groove_centers"]:
        h = c["groove_w"] / 2.0
        poly += [(zc - h, c["r_land"]), (zc - h, c["r_groove"]), (zc + h, c["r_groove"]), (zc + h, c["r_land"])]
    poly += [(c["z_hi"], c["r_land"])]
    poly = sorted(poly, key=lambda t: t[0])
    p2 = c["pitch2d"]
    z0, z1 = c["z_lo"] - 2.0, c["z_hi"] + 2.0
    r0, r1 = 0.0, c["r_land"] + 2.0
    nz = int(round((z1 - z0) / p2)) + 1
    nr = int(round((r1 - r0) / p2)) + 1
    zz = np.linspace(z0, z1, nz)
    rr = np.linspace(r0, r1, nr)
    r_of_z = np.interp(zz, [q[0] for q in poly], [q[1] for q in poly])
    mask0 = rr[:, None] <= r_of_z[None, :]
    rho = max(1, int(round(c["rho_turn"] / p2)))
    dilated = ndimage.distance_transform_edt(~mask0) <= rho
    closed = ~(ndimage.distance_transform_edt(dilated) <= rho)
    d_out = ndimage.distance_transform_edt(~closed) * p2
    d_in = ndimage.distance_transform_edt(closed) * p2
    return np.where(closed, -d_in, d_out).astype(np.float32), float(rr[0]), float(zz[0])


def machining_scene(pitch3d=0.35, block=8, short_drill=False, c=MACHINING):
    """(recipe, GridMeta, table, constants) of the machining part: the round bar intersected with the
    revolved turned profile, minus the arched pocket, minus the cross bore (through the whole bar, or
    the short negative-control drill) -- the operations and grid of tillverkningsfalt_v1_kernel.py:
    193-236, 248-300."""
    from . import expr as X
    table, r0, z0 = turned_profile_table(c)
    r_blank = c["r_land"] + c["radial_allowance"]
    zb_lo, zb_hi = c["z_lo"] - c["axial_allowance"], c["z_hi"] + c["axial_allowance"]
    arch_cz = c["roof_z"] - c["arch_r"]
    half = c["drill_x_short"] if short_drill else r_blank + 1
    recipe = X.intersect(X.round_bar(r_blank, zb_lo, zb_hi), X.revolve_table(table, r0, z0, c["pitch2d"]))
    recipe = X.subtract(recipe, X.arched_pocket(c["half_x"], c["half_y"], c["rho_mill"], c["arch_r"], arch_cz))
    recipe = X.subtract(recipe, X.cross_bore(c["drill_r"], c["drill_z"], half))
    x0 = -r_blank - 1
    n_xy = int(round((2 * r_blank + 2) / pitch3d)) + 1
    nz = int(round((zb_hi - zb_lo) / pitch3d)) + 1
    meta = GridMeta(x0, x0, zb_lo, pitch3d, n_xy, n_xy, nz, block)
    consts = dict(r_blank=r_blank, z_blank_lo=zb_lo, z_blank_hi=zb_hi, arch_cz=arch_cz, drill_x_half=half,
                  r0_2d=r0, z0_2d=z0, **c)
    return recipe, meta, table, consts
