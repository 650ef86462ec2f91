"""SDF recipes: the reference's expression-node format, compiled to a flat primitive table plus a
CSG program for the GPU.

Node constructors keep the reference's names, arguments and plain-dict JSON format
(src/field_engine/ikarus_v1/expr.py:93-210): halfspace, sphere, box, cylinder, cone, rect_frustum,
transform, translate, rotate, axis_project, offset, scale, union, intersect, subtract.  Added
without a reference counterpart: capsule (milling / drilling tool sweeps), torus and
cylinder_z_infinite (the test field of src/field_engine/faltkarna_v1.py:102-104).

``compile_recipe(node)`` folds every transform / scale / axis_project / leaf offset into the
leaf's own record, so the device evaluates ``value = s * f(A x + t) - off`` per primitive with
``f`` the canonical primitive centred on its own origin, and emits a postfix program over those
primitives.  Hard (k == 0) unions, intersections and subtractions of unions are re-associated
into a left-deep chain ``acc = op_i(acc, prim_i)`` -- exact for min/max -- which is what the
GPU's Lipschitz culling works on; smooth operators are never re-associated.  Trees that do not
reduce to a chain run as a general postfix program (every primitive at every voxel).
"""
from __future__ import annotations

import json
import math

import numpy as np

PRIM = np.dtype([("type", "<i4"), ("flags", "<i4"), ("p", "<f8", (12,)), ("A", "<f8", (12,)),
                 ("s", "<f8"), ("off", "<f8")])
INSN = np.dtype([("op", "<i4"), ("arg", "<i4"), ("k", "<f8")])

# primitive types (canonical frames)
(P_SPHERE, P_BOX, P_CYLINDER, P_CONE, P_HALFSPACE, P_FRUSTUM, P_CAPSULE, P_TORUS, P_CYL_INF,
 P_GRID, P_REVOLVE, P_BAR, P_POCKET, P_XBORE) = range(14)
TABLE_KINDS = (P_GRID, P_REVOLVE)  # records whose p[9] names a table and p[10] holds its address
# postfix program ops
OP_PUSH, OP_UNION, OP_INTERSECT, OP_SUBTRACT, OP_OFFSET = range(5)
# chain ops (device culling form)
CH_SET, CH_SETNEG, CH_UNION, CH_INTERSECT, CH_SUBTRACT, CH_OFFSET = range(6)

LEAF_OPS = ("halfspace", "sphere", "box", "cylinder", "cone", "rect_frustum", "capsule", "torus",
            "cylinder_z_infinite", "gridfield", "revolve_table", "round_bar", "arched_pocket", "cross_bore")


# --------------------------------------------------------------------------------------------- transforms
def mat4_identity():
    return [[1.0, 0.0, 0.0, 0.0], [0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0], [0.0, 0.0, 0.0, 1.0]]


def mat4_translate(tx, ty, tz):
    m = mat4_identity()
    m[0][3], m[1][3], m[2][3] = float(tx), float(ty), float(tz)
    return m


def mat4_rot_axis(axis, deg):
    """Rotation about a coordinate axis by ``deg`` degrees (src/field_engine/ikarus_v1/expr.py:37-52)."""
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    m = mat4_identity()
    if axis == "x":
        m[1][1], m[1][2], m[2][1], m[2][2] = c, -s, s, c
    elif axis == "y":
        m[0][0], m[0][2], m[2][0], m[2][2] = c, s, -s, c
    elif axis == "z":
        m[0][0], m[0][1], m[1][0], m[1][1] = c, -s, s, c
    else:
        raise ValueError(f"axis must be x/y/z, got {axis!r}")
    return m


def mat4_mul(a, b):
    return (np.asarray(a, float) @ np.asarray(b, float)).tolist()


def mat4_inverse_affine(m):
    """World -> local inverse of an affine 4x4 (rotation/scale + translation)."""
    M = np.asarray(m, dtype=np.float64)
    R = M[:3, :3]
    if abs(np.linalg.det(R)) < 1e-15:
        raise ValueError("singular transform, cannot invert")
    inv = np.linalg.inv(R)
    out = np.eye(4)
    out[:3, :3] = inv
    out[:3, 3] = -inv @ M[:3, 3]
    return out.tolist()


# --------------------------------------------------------------------------------------------- nodes
def halfspace(normal, offset):
    nx, ny, nz = normal
    nrm = math.sqrt(nx * nx + ny * ny + nz * nz)
    if not nrm > 1e-12:
        raise ValueError("halfspace normal must be non-zero")
    return {"op": "halfspace", "normal": [nx / nrm, ny / nrm, nz / nrm], "offset": float(offset)}


def sphere(radius, center=(0.0, 0.0, 0.0)):
    return {"op": "sphere", "radius": float(radius), "center": list(map(float, center))}


def box(half_extents, center=(0.0, 0.0, 0.0)):
    return {"op": "box", "half_extents": list(map(float, half_extents)), "center": list(map(float, center))}


def cylinder(radius, height, axis="z", center=(0.0, 0.0, 0.0)):
    return {"op": "cylinder", "radius": float(radius), "height": float(height), "axis": axis,
            "center": list(map(float, center))}


def cone(radius1, radius2, height, axis="z", center=(0.0, 0.0, 0.0)):
    return {"op": "cone", "radius1": float(radius1), "radius2": float(radius2), "height": float(height),
            "axis": axis, "center": list(map(float, center))}


def rect_frustum(z0, z1, hx0, hy0, hx1, hy1, cx0=0.0, cy0=0.0, cx1=0.0, cy1=0.0):
    if not z1 > z0:
        raise ValueError("rect_frustum requires z1 > z0")
    return {"op": "rect_frustum", "z0": float(z0), "z1": float(z1), "hx0": float(hx0), "hy0": float(hy0),
            "hx1": float(hx1), "hy1": float(hy1), "cx0": float(cx0), "cy0": float(cy0), "cx1": float(cx1),
            "cy1": float(cy1)}


def capsule(a, b, radius):
    """Segment a-b swept by a ball of ``radius`` (a milling-tool pass or a drill)."""
    return {"op": "capsule", "a": list(map(float, a)), "b": list(map(float, b)), "radius": float(radius)}


def torus(major, minor, axis="z", center=(0.0, 0.0, 0.0)):
    return {"op": "torus", "major": float(major), "minor": float(minor), "axis": axis,
            "center": list(map(float, center))}


def cylinder_z_infinite(radius, center=(0.0, 0.0)):
    """Unbounded cylinder along z (src/field_engine/faltkarna_v1.py:102-104)."""
    return {"op": "cylinder_z_infinite", "radius": float(radius), "center": list(map(float, center))}


def gridfield(npz_path, key="occupancy", mode="occupancy", iso=0.5, pitch_override=None):
    """Leaf sampling an existing voxel grid trilinearly (src/field_engine/ikarus_v1/expr.py:143-152):
    the npz holds the (nx, ny, nz) array under `key` and, optionally, ``global_origin_mm`` and
    ``pitch_mm``.  mode "sdf": values are signed distances; "occupancy": (iso - value) * pitch."""
    return {"op": "gridfield", "npz_path": npz_path, "key": key, "mode": mode, "iso": float(iso),
            "pitch_override": pitch_override}


def revolve_table(table, r0, z0, pitch):
    """A 2-D signed-distance table over (r, z) -- r the distance from the z axis, rows r0 + i*pitch,
    columns z0 + j*pitch -- revolved about z and sampled bilinearly: the turned-profile term of the
    reference's machining kernel (src/field_engine/tillverkningsfalt_v1_kernel.py:265-277)."""
    return {"op": "revolve_table", "table": np.ascontiguousarray(table, dtype=np.float32), "r0": float(r0),
            "z0": float(z0), "pitch": float(pitch)}


def round_bar(radius, z_lo, z_hi):
    """max(r - radius, max(z_lo - z, z - z_hi)): the round bar (blank) of the reference's machining
    kernel (tillverkningsfalt_v1_kernel.py:262-263)."""
    return {"op": "round_bar", "radius": float(radius), "z_lo": float(z_lo), "z_hi": float(z_hi)}


def arched_pocket(half_x, half_y, edge_radius, arch_radius, arch_center_z):
    """A rounded rectangle in x/y (side-edge radius edge_radius) under an arched roof
    z <= arch_center_z + sqrt(arch_radius^2 - x^2), open below: the milled pocket of the reference's
    machining kernel (tillverkningsfalt_v1_kernel.py:281-291); subtract it from the part."""
    return {"op": "arched_pocket", "half_x": float(half_x), "half_y": float(half_y),
            "edge_radius": float(edge_radius), "arch_radius": float(arch_radius),
            "arch_center_z": float(arch_center_z)}


def cross_bore(radius, axis_z, half_length):
    """A bore along x at height axis_z clipped to |x| <= half_length, in the max form of the
    reference's machining kernel (tillverkningsfalt_v1_kernel.py:294-297); subtract it."""
    return {"op": "cross_bore", "radius": float(radius), "axis_z": float(axis_z), "half_length": float(half_length)}


def transform(child, mat4):
    return {"op": "transform", "child": child, "mat4": mat4}


def translate(child, tx, ty, tz):
    return transform(child, mat4_translate(tx, ty, tz))


def rotate(child, axis, deg, about=(0.0, 0.0, 0.0)):
    ax, ay, az = about
    m = mat4_mul(mat4_translate(ax, ay, az), mat4_mul(mat4_rot_axis(axis, deg), mat4_translate(-ax, -ay, -az)))
    return transform(child, m)


def axis_project(child, axis, ref):
    if axis not in (0, 1, 2):
        raise ValueError(f"axis_project: axis must be 0/1/2, got {axis!r}")
    return {"op": "axis_project", "child": child, "axis": int(axis), "ref": float(ref)}


def offset(child, delta):
    return {"op": "offset", "child": child, "delta": float(delta)}


def scale(child, s):
    return {"op": "scale", "child": child, "s": float(s)}


def union(a, b, k=0.0):
    return {"op": "union", "a": a, "b": b, "k": float(k)}


def intersect(a, b, k=0.0):
    return {"op": "intersect", "a": a, "b": b, "k": float(k)}


def subtract(a, b, k=0.0):
    return {"op": "subtract", "a": a, "b": b, "k": float(k)}


def union_all(nodes):
    """Left-deep hard union of a sequence of nodes."""
    nodes = list(nodes)
    if not nodes:
        raise ValueError("union_all needs at least one node")
    acc = nodes[0]
    for n in nodes[1:]:
        acc = union(acc, n)
    return acc


def subtract_all(base, tools):
    """``base`` minus every tool in order (left-deep hard subtractions)."""
    acc = base
    for t in tools:
        acc = subtract(acc, t)
    return acc


def save(node, path):
    with open(path, "w") as f:
        json.dump({"ikarus_version": "1.0", "tree": node}, f, indent=1)
    return path


def load(path):
    with open(path) as f:
        data = json.load(f)
    if isinstance(data, dict) and "tree" in data and "ikarus_version" in data:
        return data["tree"]
    return data


def node_count(node):
    if not isinstance(node, dict):
        return 0
    return 1 + sum(node_count(node[k]) for k in ("child", "a", "b") if k in node)


# --------------------------------------------------------------------------------------------- compiler
_AXIS_PERM = {"z": (0, 1, 2), "y": (0, 2, 1), "x": (1, 2, 0)}  # local rows (radial, radial, axial)


def _affine(rows3x4):
    m = np.eye(4)
    m[:3, :] = rows3x4
    return m


class Compiled:
    """A compiled recipe: ``prims`` (PRIM records), ``program`` (postfix INSN), ``chain``
    (left-deep CH_* INSN records, or None when the tree does not reduce to a chain) and ``tables``
    (float32 arrays of the table-backed leaves, named by their records' p[9])."""

    def __init__(self, prims, program, chain, tables=()):
        self.prims = prims
        self.program = program
        self.chain = chain
        self.tables = [np.ascontiguousarray(t, dtype=np.float32) for t in tables]

    def with_table_addresses(self, addresses):
        """A copy of the primitive records with each table-backed record's p[10] set to the raw bits
        of addresses[p[9]] (the address of its table where the evaluator will read it)."""
        prims = self.prims.copy()
        for i in np.where(np.isin(prims["type"], TABLE_KINDS))[0]:
            prims["p"][i, 10] = np.array([int(addresses[int(prims["p"][i, 9])])], np.uint64).view(np.float64)[0]
        return prims

    def sampling_guard(self):
        """A bound on the float32 error of the table-backed leaves' samples (0 without them), for the
        guard band of the float64 recheck: the sample coordinate carries a few float32 ulps of the
        table's coordinate range, which moves the sample by that many cells times the table's steepest
        step, and the interpolation rounds about a dozen times at the table's magnitude; doubled."""
        bound = 0.0
        for rec in self.prims:
            if int(rec["type"]) not in TABLE_KINDS:
                continue
            t = self.tables[int(rec["p"][9])]
            p = rec["p"]
            if int(rec["type"]) == P_GRID:
                pitch, shape, origin, axes = p[3], t.shape, np.abs(p[:3]), 3
                scale = 1.0 if p[5] else pitch  # occupancy samples are (iso - v) * pitch
            else:
                pitch, shape, origin, axes = p[2], t.shape, np.abs(p[:2]), 2
                scale = 1.0
            reach = float(np.max(origin + (np.asarray(shape, np.float64) - 1) * pitch))
            steep = max(float(np.abs(np.diff(t.astype(np.float64), axis=a)).max()) if t.shape[a] > 1 else 0.0
                        for a in range(t.ndim))
            coord = 4.0 * float(np.spacing(np.float32(reach))) / pitch
            mag = float(np.abs(t).max()) + (abs(p[4]) if int(rec["type"]) == P_GRID else 0.0)
            err = (axes * coord * steep + 12.0 * float(np.spacing(np.float32(mag)))) * scale
            bound = max(bound, 2.0 * err * abs(float(rec["s"])))
        return bound

    def host_prims(self):
        """The primitive records with the host tables' addresses (for CPU evaluators of them)."""
        return self.with_table_addresses([t.ctypes.data for t in self.tables])

    @property
    def n_prims(self):
        return len(self.prims)

    def lipschitz(self):
        """Per-primitive Lipschitz bound of the world-space value (for culling, reporting)."""
        out = np.empty(len(self.prims))
        for i, p in enumerate(self.prims):
            A = p["A"].reshape(3, 4)[:, :3]
            out[i] = abs(p["s"]) * np.linalg.norm(A, 2) * _canon_lipschitz(p)
        return out


def _canon_lipschitz(p):
    if p["type"] == P_CONE:
        r1, r2, h = p["p"][0], p["p"][1], p["p"][2]
        return 2.0 + abs(r2 - r1) / h
    return 1.0


def _load_gridfield(node):
    """(float32 array, origin, pitch) of a gridfield leaf, read as the reference reads it
    (src/field_engine/ikarus_v1/eval_warp.py:448-452, including its precedence: the override applies
    only when the npz carries ``pitch_mm``)."""
    with np.load(node["npz_path"]) as d:
        arr = np.asarray(d[node["key"]], dtype=np.float32)
        origin = np.asarray(d["global_origin_mm"], dtype=np.float64) if "global_origin_mm" in d else np.zeros(3)
        pitch = (node["pitch_override"] or float(d["pitch_mm"])) if "pitch_mm" in d else 1.0
    if arr.ndim != 3 or min(arr.shape) < 1:
        raise ValueError("gridfield array must be 3-D and nonempty")
    if not np.isfinite(arr).all() or not (pitch > 0 and np.isfinite(pitch)):
        raise ValueError("gridfield values and pitch must be finite (pitch > 0)")
    return arr, origin, float(pitch)


class _Compiler:
    def __init__(self):
        self.prims = []
        self.tables = []

    def leaf(self, node, M, sigma):
        """PRIM record for a leaf under world->frame map M (4x4) and output scale sigma."""
        op = node["op"]
        p = np.zeros(12)
        canon = np.eye(4)
        perm = (0, 1, 2)

        def shift(c):
            t = np.eye(4)
            t[:3, 3] = -np.asarray(c, float)
            return t
        if op == "sphere":
            canon = shift(node["center"])
            p[0] = node["radius"]
            typ = P_SPHERE
        elif op == "box":
            canon = shift(node["center"])
            p[:3] = node["half_extents"]
            typ = P_BOX
        elif op == "cylinder":
            canon = shift(node["center"])
            perm = _AXIS_PERM[node["axis"]]
            p[0], p[1] = node["radius"], node["height"] / 2.0
            typ = P_CYLINDER
        elif op == "cone":
            canon = shift(node["center"])
            perm = _AXIS_PERM[node["axis"]]
            p[0], p[1], p[2] = node["radius1"], node["radius2"], node["height"]
            if not p[2] > 0:
                raise ValueError("cone height must be positive")
            typ = P_CONE
        elif op == "halfspace":
            n = np.asarray(node["normal"], float)
            canon = shift(n * node["offset"])
            p[:3] = n
            typ = P_HALFSPACE
        elif op == "rect_frustum":
            canon = shift((node["cx0"], node["cy0"], node["z0"]))
            p[:7] = (node["z1"] - node["z0"], node["hx0"], node["hy0"], node["hx1"], node["hy1"],
                     node["cx1"] - node["cx0"], node["cy1"] - node["cy0"])
            typ = P_FRUSTUM
        elif op == "capsule":
            a = np.asarray(node["a"], float)
            canon = shift(a)
            p[:3] = np.asarray(node["b"], float) - a
            p[3] = node["radius"]
            typ = P_CAPSULE
        elif op == "torus":
            canon = shift(node["center"])
            perm = _AXIS_PERM[node["axis"]]
            p[0], p[1] = node["major"], node["minor"]
            typ = P_TORUS
        elif op == "cylinder_z_infinite":
            cx, cy = node["center"]
            canon = shift((cx, cy, 0.0))
            p[0] = node["radius"]
            typ = P_CYL_INF
        elif op == "gridfield":
            arr, origin, pitch = _load_gridfield(node)
            f32 = lambda v: float(np.float32(v))  # the sampler's float32 parameters
            p[:9] = (f32(origin[0]), f32(origin[1]), f32(origin[2]), f32(pitch), f32(node["iso"]),
                     1.0 if node["mode"] == "sdf" else 0.0, *arr.shape)
            p[9] = len(self.tables)
            self.tables.append(arr)
            typ = P_GRID
        elif op == "revolve_table":
            t = np.ascontiguousarray(node["table"], dtype=np.float32)
            if t.ndim != 2 or min(t.shape) < 2 or not np.isfinite(t).all() or not node["pitch"] > 0:
                raise ValueError("revolve_table needs a finite 2-D table of at least 2 x 2 and pitch > 0")
            f32 = lambda v: float(np.float32(v))
            p[:5] = (f32(node["r0"]), f32(node["z0"]), f32(node["pitch"]), *t.shape)
            p[9] = len(self.tables)
            self.tables.append(t)
            typ = P_REVOLVE
        elif op == "round_bar":
            p[:3] = (node["radius"], node["z_lo"], node["z_hi"])
            typ = P_BAR
        elif op == "arched_pocket":
            p[:5] = (node["half_x"], node["half_y"], node["edge_radius"], node["arch_radius"], node["arch_center_z"])
            typ = P_POCKET
        elif op == "cross_bore":
            p[:3] = (node["radius"], node["axis_z"], node["half_length"])
            typ = P_XBORE
        else:
            raise ValueError(f"unknown leaf op {op!r}")
        P = np.eye(4)[list(perm) + [3]]
        total = P @ canon @ M
        rec = np.zeros(1, PRIM)[0]
        rec["type"] = typ
        rec["p"] = p
        rec["A"] = total[:3, :].reshape(-1)
        rec["s"] = sigma
        rec["off"] = 0.0
        self.prims.append(rec)
        return len(self.prims) - 1

    # ---- general postfix emission (no re-association)
    # The deeper operand of each boolean is evaluated first (Sethi-Ullman order), so a tree of N
    # leaves needs at most log2(N) + 1 stack slots whatever its shape.  Union and intersection are
    # symmetric in their operands (the same value bits: min / max and |a - b| do not depend on the
    # order); subtract(a, b) with the deeper b is evaluated as intersect(-b, a), the same float64
    # operations as max(a, -b) + h^2 k / 4 with h from |a + b|.  A negated subtree is emitted with a
    # negative output scale: leaves get s < 0 and off < 0 (value = s f - off, negation is exact in
    # round-to-nearest), offsets flip with it, union and intersection swap, and -subtract(a, b) is
    # union(-a, b).
    def _stack_need(self, node, memo):
        """Stack slots the postfix program of ``node`` needs in the deeper-operand-first order."""
        key = id(node)
        if key in memo:
            return memo[key]
        op = node["op"]
        if op in LEAF_OPS:
            r = 1
        elif op in ("transform", "scale", "axis_project", "offset"):
            r = self._stack_need(node["child"], memo)
        elif op in ("union", "intersect", "subtract"):
            spine = []
            cur = node
            while cur["op"] in ("union", "intersect", "subtract") and id(cur) not in memo:
                spine.append(cur)
                cur = cur["a"]
            r = self._stack_need(cur, memo)
            for nd in reversed(spine):
                nb = self._stack_need(nd["b"], memo)
                r = max(r, nb) if r != nb else r + 1
                memo[id(nd)] = r
        else:
            raise ValueError(f"unknown op {op!r}")
        memo[key] = r
        return r

    def emit(self, node, M, sigma, out, memo=None):
        if memo is None:
            memo = {}
        op = node["op"]
        if op in LEAF_OPS:
            out.append((OP_PUSH, self.leaf(node, M, sigma), 0.0))
        elif op == "transform":
            self.emit(node["child"], np.asarray(mat4_inverse_affine(node["mat4"])) @ M, sigma, out, memo)
        elif op == "scale":
            s = float(node["s"])
            if not s > 0:
                raise ValueError("scale factor must be positive")
            self.emit(node["child"], np.diag([1 / s, 1 / s, 1 / s, 1.0]) @ M, sigma * s, out, memo)
        elif op == "axis_project":
            Pm = np.eye(4)
            Pm[node["axis"], :] = 0.0
            Pm[node["axis"], 3] = node["ref"]
            self.emit(node["child"], Pm @ M, sigma, out, memo)
        elif op == "offset":
            n0 = len(out)
            self.emit(node["child"], M, sigma, out, memo)
            if len(out) == n0 + 1 and out[-1][0] == OP_PUSH:
                self.prims[out[-1][1]]["off"] += sigma * node["delta"]
            else:
                out.append((OP_OFFSET, -1, sigma * node["delta"]))
        elif op in ("union", "intersect", "subtract"):
            # the run of the left spine evaluated left operand first, iteratively (recipes are
            # left-deep chains thousands of operations long); it ends at a leaf-side operand or at a
            # node whose right operand is the deeper one, which recurses
            run = []
            cur = node
            while cur["op"] in ("union", "intersect", "subtract") and (
                    self._stack_need(cur["b"], memo) <= self._stack_need(cur["a"], memo)):
                run.append(cur)
                cur = cur["a"]
            if cur["op"] in ("union", "intersect", "subtract"):
                code, sb = self._bool_code(cur["op"], sigma, b_first=True)
                self.emit(cur["b"], M, sb, out, memo)
                self.emit(cur["a"], M, sigma, out, memo)
                out.append((code, -1, abs(sigma) * cur["k"]))
            else:
                self.emit(cur, M, sigma, out, memo)
            for nd in reversed(run):
                code, sb = self._bool_code(nd["op"], sigma, b_first=False)
                self.emit(nd["b"], M, sb, out, memo)
                out.append((code, -1, abs(sigma) * nd["k"]))
        else:
            raise ValueError(f"unknown op {op!r}")

    @staticmethod
    def _bool_code(op, sigma, b_first):
        """Opcode and the right operand's output scale of boolean `op` under output scale `sigma`
        (the left operand always keeps `sigma`)."""
        if sigma > 0:
            if op == "subtract":
                return (OP_INTERSECT, -sigma) if b_first else (OP_SUBTRACT, sigma)
            return (OP_UNION if op == "union" else OP_INTERSECT), sigma
        if op == "subtract":  # -(a - b) = union(-a, b)
            return OP_UNION, -sigma
        return (OP_INTERSECT if op == "union" else OP_UNION), sigma

    # ---- chain emission: returns list of (CH_op, prim, k) or None
    def chain(self, node, M, sigma):
        # Walk the left spine of booleans iteratively (recipes are left-deep chains thousands of
        # operations long), then append each right operand bottom-up.
        spine = []
        cur = node
        while cur["op"] in ("union", "intersect", "subtract"):
            spine.append(cur)
            cur = cur["a"]
        acc = self._chain_root(cur, M, sigma)
        if acc is None:
            return None
        for nd in reversed(spine):
            op = nd["op"]
            k = sigma * nd["k"]
            code = {"union": CH_UNION, "intersect": CH_INTERSECT, "subtract": CH_SUBTRACT}[op]
            # the right operand: a single primitive, or (hard only) a same-kind run of primitives
            leaves = self._leaf_run(nd["b"], M, sigma, "intersect" if op == "intersect" else "union",
                                    allow_run=(k == 0.0))
            if leaves is None:
                return None
            acc = acc + [(code, i, k) for i in leaves]
        return acc

    def _chain_root(self, node, M, sigma):
        op = node["op"]
        if op in LEAF_OPS:
            return [(CH_SET, self.leaf(node, M, sigma), 0.0)]
        if op in ("transform", "scale", "axis_project"):
            return self._wrap_leafish(node, M, sigma)
        if op == "offset":
            inner = self.chain(node["child"], M, sigma)
            if inner is None:
                return None
            if len(inner) == 1 and inner[0][0] == CH_SET:
                self.prims[inner[0][1]]["off"] += sigma * node["delta"]
                return inner
            return inner + [(CH_OFFSET, -1, sigma * node["delta"])]
        return None

    def _wrap_leafish(self, node, M, sigma):
        """transform/scale/axis_project around a subtree: fold into M and recurse."""
        op = node["op"]
        if op == "transform":
            return self.chain(node["child"], np.asarray(mat4_inverse_affine(node["mat4"])) @ M, sigma)
        if op == "scale":
            s = float(node["s"])
            if not s > 0:
                raise ValueError("scale factor must be positive")
            return self.chain(node["child"], np.diag([1 / s, 1 / s, 1 / s, 1.0]) @ M, sigma * s)
        Pm = np.eye(4)
        Pm[node["axis"], :] = 0.0
        Pm[node["axis"], 3] = node["ref"]
        return self.chain(node["child"], Pm @ M, sigma)

    def _leaf_run(self, node, M, sigma, kind, allow_run):
        """Primitive indices of ``node`` if it is one leaf, or (allow_run) a hard ``kind`` run of
        leaves; None otherwise.  Offsets on a single leaf fold into it."""
        op = node["op"]
        if op in LEAF_OPS:
            return [self.leaf(node, M, sigma)]
        if op == "transform":
            return self._leaf_run(node["child"], np.asarray(mat4_inverse_affine(node["mat4"])) @ M, sigma, kind,
                                  allow_run)
        if op == "scale":
            s = float(node["s"])
            if not s > 0:
                raise ValueError("scale factor must be positive")
            return self._leaf_run(node["child"], np.diag([1 / s, 1 / s, 1 / s, 1.0]) @ M, sigma * s, kind, allow_run)
        if op == "axis_project":
            Pm = np.eye(4)
            Pm[node["axis"], :] = 0.0
            Pm[node["axis"], 3] = node["ref"]
            return self._leaf_run(node["child"], Pm @ M, sigma, kind, allow_run)
        if op == "offset":
            r = self._leaf_run(node["child"], M, sigma, kind, False)
            if r is None:
                return None
            self.prims[r[0]]["off"] += sigma * node["delta"]
            return r
        if allow_run and op == kind and node["k"] == 0.0:
            a = self._leaf_run(node["a"], M, sigma, kind, True)
            if a is None:
                return None
            b = self._leaf_run(node["b"], M, sigma, kind, True)
            if b is None:
                return None
            return a + b
        return None


def _chain_to_program(chain):
    """The postfix program that evaluates a chain in the same association order."""
    prog = []
    for op, prim, k in chain:
        if op == CH_SET:
            prog.append((OP_PUSH, prim, 0.0))
        elif op == CH_OFFSET:
            prog.append((OP_OFFSET, -1, k))
        else:
            prog.append((OP_PUSH, prim, 0.0))
            prog.append(({CH_UNION: OP_UNION, CH_INTERSECT: OP_INTERSECT, CH_SUBTRACT: OP_SUBTRACT}[op], -1, k))
    return prog


def _records(rows):
    arr = np.zeros(len(rows), INSN)
    for i, (op, arg, k) in enumerate(rows):
        arr[i] = (op, arg, k)
    return arr


def compile_recipe(node) -> Compiled:
    """Compile an expression tree (plain dict nodes) for the GPU evaluators."""
    c = _Compiler()
    ch = c.chain(node, np.eye(4), 1.0)
    if ch is not None:
        prims = np.array(c.prims, dtype=PRIM) if c.prims else np.zeros(0, PRIM)
        return Compiled(prims, _records(_chain_to_program(ch)), _records(ch), c.tables)
    c = _Compiler()
    prog = []
    c.emit(node, np.eye(4), 1.0, prog)
    depth = max_depth = 0
    for op, _, _ in prog:
        depth += 1 if op == OP_PUSH else (0 if op == OP_OFFSET else -1)
        max_depth = max(max_depth, depth)
    if max_depth > 32:  # reachable only with more than 2^31 leaves (deeper operand first)
        raise ValueError("expression tree too deep for the GPU stack evaluator (depth > 32)")
    prims = np.array(c.prims, dtype=PRIM) if c.prims else np.zeros(0, PRIM)
    return Compiled(prims, _records(prog), None, c.tables)


def compile_tools(tools):
    """PRIM records of edit tools, one primitive each (a leaf under transforms / scale / offset)."""
    recs = []
    for tool in tools:
        c = _Compiler()
        ch = c.chain(tool, np.eye(4), 1.0)
        if ch is None or len(ch) != 1 or ch[0][0] != CH_SET:
            raise ValueError("an edit tool must be a single primitive")
        if c.tables:
            raise ValueError("an edit tool cannot be a table-backed leaf")
        recs.append(c.prims[ch[0][1]])
    return np.array(recs, dtype=PRIM) if recs else np.zeros(0, PRIM)


def extend(comp: Compiled, tool_prims, op="subtract") -> Compiled:
    """``comp`` with each tool primitive subtracted from (op "subtract") or unioned to (op "union")
    the result in order -- the compiled form of subtract(...subtract(recipe, t1)..., tn) -- without
    recompiling the recipe: the tools' records are appended to the table, one chain entry each
    (or push + operator in the postfix program of a recipe that has no chain)."""
    if op not in ("union", "subtract"):
        raise ValueError("edit op must be union or subtract")
    tool_prims = np.asarray(tool_prims, dtype=PRIM)
    base = len(comp.prims)
    prims = np.concatenate([comp.prims, tool_prims])
    idx = range(base, base + len(tool_prims))
    # the program of a chain ends with push + operator per hard chain entry, so the tools' part is
    # appended to the existing program in both forms
    code = OP_SUBTRACT if op == "subtract" else OP_UNION
    rows = []
    for i in idx:
        rows += [(OP_PUSH, i, 0.0), (code, -1, 0.0)]
    program = np.concatenate([comp.program, _records(rows)])
    if comp.chain is not None:
        ch = CH_SUBTRACT if op == "subtract" else CH_UNION
        return Compiled(prims, program, np.concatenate([comp.chain, _records([(ch, i, 0.0) for i in idx])]),
                        comp.tables)
    return Compiled(prims, program, None, comp.tables)


def eval_sdf_py(node, p):
    """Pure-Python float64 evaluation of a tree (the reference's ground truth, for small checks;
    src/field_engine/ikarus_v1/expr.py:263-385).  Uses the compiled form on one point."""
    comp = compile_recipe(node)
    pts = np.asarray(p, dtype=np.float64).reshape(1, 3)
    return float(_eval_compiled_numpy(comp, pts)[0])


def _eval_compiled_numpy(comp, pts):
    """Vectorised float64 NumPy evaluation of a compiled program (host-side helper)."""
    vals = []
    for op, arg, k in comp.program:
        if op == OP_PUSH:
            vals.append(_prim_numpy(comp.prims[arg], pts))
        elif op == OP_OFFSET:
            vals[-1] = vals[-1] - k
        else:
            b = vals.pop()
            a = vals.pop()
            if op == OP_SUBTRACT:
                b2 = -b
                if k <= 0:
                    r = np.maximum(a, b2)
                else:
                    h = np.maximum(k - np.abs(a + b), 0.0) / k
                    r = np.maximum(a, b2) + h * h * k * 0.25
            elif op == OP_UNION:
                if k <= 0:
                    r = np.minimum(a, b)
                else:
                    h = np.maximum(k - np.abs(a - b), 0.0) / k
                    r = np.minimum(a, b) - h * h * k * 0.25
            else:
                if k <= 0:
                    r = np.maximum(a, b)
                else:
                    h = np.maximum(k - np.abs(a - b), 0.0) / k
                    r = np.maximum(a, b) + h * h * k * 0.25
            vals.append(r)
    return vals[0]


def _prim_numpy(rec, pts):
    A = rec["A"].reshape(3, 4)
    q = pts @ A[:, :3].T + A[:, 3]
    x, y, z = q[:, 0], q[:, 1], q[:, 2]
    p = rec["p"]
    t = rec["type"]
    if t == P_SPHERE:
        f = np.sqrt(x * x + y * y + z * z) - p[0]
    elif t == P_BOX:
        qq = np.abs(q) - p[:3]
        f = np.linalg.norm(np.maximum(qq, 0), axis=1) + np.minimum(qq.max(axis=1), 0)
    elif t == P_CYLINDER:
        qx, qy = np.sqrt(x * x + y * y) - p[0], np.abs(z) - p[1]
        f = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2) + np.minimum(np.maximum(qx, qy), 0)
    elif t == P_CONE:
        h = p[2]
        tt = np.clip((z + h / 2.0) / h, 0.0, 1.0)
        qx = np.sqrt(x * x + y * y) - (p[0] + (p[1] - p[0]) * tt)
        qy = np.abs(z) - h / 2.0
        f = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2) + np.minimum(np.maximum(qx, qy), 0)
    elif t == P_HALFSPACE:
        f = x * p[0] + y * p[1] + z * p[2]
    elif t == P_FRUSTUM:
        z1, hx0, hy0, hx1, hy1, cx1, cy1 = p[:7]
        kx, ky, kcx, kcy = (hx1 - hx0) / z1, (hy1 - hy0) / z1, cx1 / z1, cy1 / z1
        a1, a2, a3, a4 = -(kx + kcx), -(kx - kcx), -(ky + kcy), -(ky - kcy)
        f = np.max(np.stack([-z, z - z1, (x + a1 * z - hx0) / np.sqrt(1 + a1 * a1),
                             (-x + a2 * z - hx0) / np.sqrt(1 + a2 * a2), (y + a3 * z - hy0) / np.sqrt(1 + a3 * a3),
                             (-y + a4 * z - hy0) / np.sqrt(1 + a4 * a4)]), axis=0)
    elif t == P_CAPSULE:
        b = p[:3]
        bb = float(b @ b)
        hh = np.clip((q @ b) / bb, 0.0, 1.0) if bb > 0 else np.zeros(len(q))
        f = np.linalg.norm(q - hh[:, None] * b, axis=1) - p[3]
    elif t == P_TORUS:
        qx = np.sqrt(x * x + y * y) - p[0]
        f = np.sqrt(qx * qx + z * z) - p[1]
    elif t == P_CYL_INF:
        f = np.sqrt(x * x + y * y) - p[0]
    elif t == P_BAR:
        f = np.maximum(np.sqrt(x * x + y * y) - p[0], np.maximum(p[1] - z, z - p[2]))
    elif t == P_POCKET:
        qx, qy = np.abs(x) - (p[0] - p[2]), np.abs(y) - (p[1] - p[2])
        dxy = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2) + np.minimum(np.maximum(qx, qy), 0) - p[2]
        f = np.maximum(dxy, z - (p[4] + np.sqrt(np.maximum(p[3] * p[3] - x * x, 0.0))))
    elif t == P_XBORE:
        f = np.maximum(np.sqrt(y * y + (z - p[1]) ** 2) - p[0], np.abs(x) - p[2])
    else:
        raise ValueError(f"primitive type {t} has no host evaluator (table-backed kinds run on the device)")
    return rec["s"] * f - rec["off"]
