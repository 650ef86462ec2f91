"""csg_execute against the reference's own compiled csg_execute (oracle/_ref/libref_csg_batch.so,
src/field_engine/csg_batch_native_v1/execute.cpp + csg_tile_native_v1/gather.cpp) through the same
ctypes call: equal status and equal output bytes, for valid programs up to the reference's bounds
(256 fields, 1024 instructions) and for every failure class -- arguments (1), program (2), operand
gathers (3: bounds, malformed leaves, gaps, overlaps, fields without leaves), non-finite results
(4) -- including failures in a later tile, where the reference has already written the earlier
tiles (GPU)."""
import ctypes as ct

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SHAPE = (40, 70, 35)  # 3 x 3 x 3 of the reference's 16 x 32 x 16 tiles
POISON = np.uint32(0x7FC0DEAD)  # NaN pattern the caller's output starts from


def _libs():
    import field_b200._lib as L
    ref = oracle.ref_library("csg_batch")
    if ref is None:
        pytest.skip("oracle/_ref/libref_csg_batch.so is not built")
    return L.lib(), ref


def _call(lib, fields, program, shape=SHAPE, nodes_override=None, count_override=None, length_override=None):
    """(status, output bytes) of csg_execute on packed operands `fields` = [(nodes, payload)]."""
    fn = lib.csg_execute
    fn.argtypes = [ct.c_void_p] * 4 + [ct.c_int32, ct.c_void_p, ct.c_void_p, ct.c_int32, ct.c_void_p]
    fn.restype = ct.c_int
    nodes = [f[0] for f in fields]
    payloads = [f[1] for f in fields]
    nptr = (ct.c_void_p * len(fields))(*(n.ctypes.data if n is not None else None for n in nodes))
    if nodes_override:
        for i, v in nodes_override.items():
            nptr[i] = v
    pptr = (ct.c_void_p * len(fields))(*(p.ctypes.data for p in payloads))
    counts = np.array([len(n) if n is not None else 1 for n in nodes], np.int64)
    lengths = np.array([len(p) for p in payloads], np.int64)
    if count_override:
        for i, v in count_override.items():
            counts[i] = v
    if length_override:
        for i, v in length_override.items():
            lengths[i] = v
    sh = np.array(shape, np.int32)
    enc = oracle.encode_program(program, len(fields))
    out = np.full(int(np.prod(shape)), POISON, np.uint32)
    rc = fn(nptr, counts.ctypes.data, pptr, lengths.ctypes.data, len(fields), sh.ctypes.data, enc.ctypes.data,
            len(enc), out.ctypes.data)
    return rc, out.tobytes()


def _same(fields, program, **kw):
    ours, ref = _libs()
    a = _call(ours, fields, program, **kw)
    b = _call(ref, fields, program, **kw)
    assert a[0] == b[0], (a[0], b[0])
    assert a[1] == b[1], "output bytes differ"
    return a[0]


def _packed(dense, threshold=64):
    nodes, payload = oracle.pack(np.ascontiguousarray(dense, np.float32), threshold)
    return nodes, payload


def _smooth(rng, shape=SHAPE):
    x, y, z = np.indices(shape, dtype=np.float64)
    c = rng.uniform(0, 1, 3) * np.array(shape)
    return (np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - rng.uniform(5, 20)).astype(np.float32)


def test_valid_programs_equal_the_reference():
    rng = np.random.default_rng(0)
    base = [_packed(_smooth(rng)) for _ in range(6)]
    fields = [base[i % 6] for i in range(256)]
    # a left-deep chain over every field
    chain = [("union", 0, 1)] + [("difference" if i % 3 == 0 else "union", 256 + i - 2, i) for i in range(2, 256)]
    assert _same(fields, chain) == 0
    # a random DAG of 1024 instructions, many values live at once (slots beyond the per-thread array)
    prog = []
    for n in range(1024):
        op = ["union", "difference", "offset"][int(rng.integers(3))]
        left = int(rng.integers(0, 256 + n))
        if op == "offset":
            prog.append((op, left, float(rng.normal() * 3)))
        else:
            prog.append((op, left, int(rng.integers(0, 256 + n))))
    assert _same(fields, prog) == 0
    # a wide tree: 128 pairwise unions of inputs, then a balanced reduction (128 values live)
    tree = [("union", 2 * i, 2 * i + 1) for i in range(128)]
    level, nxt = list(range(256, 384)), 384
    while len(level) > 1:
        new = []
        for i in range(0, len(level), 2):
            tree.append(("difference" if i % 4 else "union", level[i], level[i + 1]))
            new.append(nxt)
            nxt += 1
        level = new
    assert _same(fields, tree) == 0


def test_argument_and_program_failures_equal_the_reference():
    rng = np.random.default_rng(1)
    f = [_packed(_smooth(rng))]
    assert _same(f, [("union", 0, 1)]) == 2  # reference to a later value
    assert _same(f, [("offset", 0, float("inf"))]) == 2
    assert _same(f, [("union", 0, 0)], shape=(4097, 1, 1)) == 1
    assert _same(f, [("union", 0, 0)], shape=(4096, 4096, 2)) == 1


def test_gather_failures_equal_the_reference():
    rng = np.random.default_rng(2)
    good = _packed(_smooth(rng))
    program = [("union", 0, 1)]

    def broken(mutate):
        nodes = good[0].copy()
        mutate(nodes)
        return nodes, good[1]
    leaf = int(np.where(good[0]["children"][:, 0] < 0)[0][0])

    def bad_offset(n):
        n["offset"][leaf] = len(good[1])

    def bad_stored(n):
        n["stored_shape"][leaf] = n["shape"][leaf] + 1

    def no_leaves(n):
        n["children"][:, 0] = 0
    for mutate in (bad_offset, bad_stored, no_leaves):
        assert _same([good, broken(mutate)], program) == 3, mutate.__name__
    # overlap: every leaf twice
    assert _same([good, (np.concatenate([good[0], good[0][good[0]["children"][:, 0] < 0]]), good[1])], program) == 3
    # argument bounds of the gather: count and sample bounds, a null node pointer
    assert _same([good, good], program, count_override={1: 0}) == 3
    assert _same([good, good], program, length_override={1: 0}) == 3
    assert _same([good, good], program, nodes_override={1: None}) == 3
    # a broken operand that the program never reads is not gathered
    assert _same([good, broken(bad_offset)], [("offset", 0, 1.0)]) == 0


def test_failures_in_a_later_tile_keep_the_earlier_tiles():
    rng = np.random.default_rng(3)
    dense = _smooth(rng)
    dense[:, :, :] = np.where(np.indices(SHAPE)[0] >= 20, np.float32(1.0), dense)  # constant far half
    good = _packed(dense)
    # a gap: shrink one constant (fully collapsed) leaf in the far half
    nodes = good[0].copy()
    cand = np.where((nodes["children"][:, 0] < 0) & (nodes["stored_shape"] == 1).all(axis=1)
                    & (nodes["lo"][:, 0] >= 20) & (nodes["shape"][:, 2] > 1))[0]
    assert len(cand)

    def tile(x, y, z):
        return ((x // 16) * 3 + y // 32) * 3 + z // 16
    # the leaf whose far z face (the voxels the gap uncovers) lies in the earliest tile
    gap_tile = lambda i: tile(*(nodes["lo"][i] + np.array([0, 0, nodes["shape"][i, 2] - 1])))
    first = min(cand, key=gap_tile)
    assert gap_tile(first) < 13
    nodes["shape"][first, 2] -= 1
    assert _same([good, (nodes, good[1])], [("union", 0, 1)]) == 3
    # a non-finite result in tile 13 of 27
    big = _smooth(rng)
    big[30, 60, 30] = np.float32(3.0e38)
    assert tile(30, 60, 30) == 13
    assert _same([_packed(big)], [("offset", 0, -1.0e38)]) == 4
    # the earlier tile's gather failure is where the reference stops
    assert _same([_packed(big), (nodes, good[1])], [("offset", 0, -1.0e38), ("union", 2, 1)]) == 3
