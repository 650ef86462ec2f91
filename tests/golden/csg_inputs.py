"""Input fields of the reference's CSG probes, restated.

The bracket / plate / holes boxes and the sphere / plate / hole primitives, sampled on the
probes' grid (origin (-2, -2, -4), shape round((24, 16, 22) / pitch) + 1):
probes/field_engine/field_csg_probe.py:18-27 (BOXES, box_distance) and
probes/field_engine/field_csg_curved_probe.py:27-37 (distances), with the programs of
probes/field_engine/field_csg_batch_probe.py:44.  make_golden.py checks that the oracle's CSG of
these inputs reproduces the reference's captured outputs bit for bit, which pins this restatement.
"""
import numpy as np

BOXES = [((0, 0, 0), (20, 6, 4)), ((0, 0, 0), (4, 6, 16)),
         ((0, 0, 0), (20, 12, 2)), ((5, 3, -2), (8, 5, 6)), ((12, 3, -2), (15, 5, 6))]


def box_distance(points, bounds):
    lo, hi = np.asarray(bounds[0]), np.asarray(bounds[1])
    q = np.abs(points - (lo + hi) / 2) - (hi - lo) / 2
    return np.linalg.norm(np.maximum(q, 0), axis=-1) + np.minimum(q.max(axis=-1), 0)


def distances(points, curved):
    if not curved:
        return [box_distance(points, b) for b in BOXES]
    sphere = np.linalg.norm(points - np.array([10, 6, 6]), axis=-1) - 6
    plate = box_distance(points, ((0, 0, 0), (20, 12, 2)))
    q = np.stack((np.linalg.norm(points[:, :2] - [10, 6], axis=-1) - 1.5, np.abs(points[:, 2] - 6) - 10), axis=-1)
    cylinder = np.linalg.norm(np.maximum(q, 0), axis=-1) + np.minimum(q.max(axis=-1), 0)
    return [sphere, plate, cylinder]


def program(curved):
    return [("union", 0, 1), ("difference", 3, 2)] if curved else \
        [("union", 0, 1), ("union", 5, 2), ("union", 3, 4), ("difference", 6, 7)]


def case(curved, pitch):
    """(input fields float32, origin, shape, program)."""
    origin = np.array([-2., -2., -4.])
    shape = tuple(np.rint(np.array([24, 16, 22]) / pitch).astype(int) + 1)
    indices = np.indices(shape).reshape(3, -1).T
    fields = [a.reshape(shape).astype(np.float32) for a in distances(origin + indices * pitch, curved)]
    return fields, origin, shape, program(curved)
