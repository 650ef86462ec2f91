"""General (non-chain) programs of any shape compile into a bounded stack: the deeper operand of each
boolean is evaluated first, a deep subtracted subtree through exact negation.  Checked on the CPU
against an independent float64 evaluation of the tree with the reference's operator semantics
(src/field_engine/ikarus_v1/expr.py:364-384), through the oracle's postfix evaluator."""
import numpy as np
import pytest

import oracle
import field_b200.expr as X


def ref_value(node, p):
    """Reference semantics, evaluated directly on the tree (spheres, booleans, offset, scale)."""
    op = node["op"]
    if op == "sphere":
        return np.linalg.norm(p - np.asarray(node["center"], float), axis=1) - node["radius"]
    if op == "box":
        q = np.abs(p - np.asarray(node["center"], float)) - np.asarray(node["half_extents"], float)
        return np.linalg.norm(np.maximum(q, 0.0), axis=1) + np.minimum(q.max(axis=1), 0.0)
    if op == "offset":
        return ref_value(node["child"], p) - node["delta"]
    if op == "scale":
        return node["s"] * ref_value(node["child"], p / node["s"])
    a, b, k = ref_value(node["a"], p), ref_value(node["b"], p), node["k"]
    if op == "union":
        m = np.minimum(a, b)
        return m if k <= 0 else m - (np.maximum(k - np.abs(a - b), 0) / k) ** 2 * k * 0.25
    if op == "intersect":
        m = np.maximum(a, b)
        return m if k <= 0 else m + (np.maximum(k - np.abs(a - b), 0) / k) ** 2 * k * 0.25
    m = np.maximum(a, -b)
    return m if k <= 0 else m + (np.maximum(k - np.abs(a + b), 0) / k) ** 2 * k * 0.25


def right_deep(nodes, op, ks):
    out = nodes[-1]
    for nd, k in zip(reversed(nodes[:-1]), reversed(ks)):
        out = {"union": X.union, "intersect": X.intersect, "subtract": X.subtract}[op](nd, out, k=k)
    return out


def spheres(rng, n):
    return [X.sphere(float(rng.uniform(0.03, 0.12)), tuple(rng.uniform(0.1, 0.9, 3))) for _ in range(n)]


def deep_cases():
    rng = np.random.default_rng(11)
    ks = lambda n: [float(k) for k in rng.choice([0.0, 0.02, 0.05], n)]
    s = spheres(rng, 300)
    chain = right_deep(s[:120], "union", ks(119))
    yield "right-deep smooth union", chain
    yield "box minus right-deep union", X.subtract(X.box((0.4, 0.4, 0.4), (0.5, 0.5, 0.5)), chain, k=0.03)
    inner = X.subtract(X.offset(s[120], -0.05), right_deep(s[121:200], "intersect", ks(78)), k=0.01)
    yield "nested negated subtract", X.subtract(X.scale(X.sphere(0.3, (1.0, 1.0, 1.0)), 0.5), inner, k=0.02)
    mixed = s[200]
    for i, nd in enumerate(s[201:300]):
        kind = ("union", "intersect", "subtract")[i % 3]
        mixed = {"union": X.union, "intersect": X.intersect, "subtract": X.subtract}[kind](
            X.offset(nd, 0.01 * (i % 4)), mixed, k=0.01 * (i % 3))
    yield "right-deep mixed operators", mixed


@pytest.mark.parametrize("name,tree", list(deep_cases()), ids=[c[0] for c in deep_cases()])
def test_deep_tree_compiles_to_bounded_stack_and_keeps_its_values(name, tree):
    comp = X.compile_recipe(tree)
    depth = max_depth = 0
    for op in comp.program["op"]:
        depth += 1 if op == X.OP_PUSH else (0 if op == X.OP_OFFSET else -1)
        max_depth = max(max_depth, depth)
    assert depth == 1 and max_depth <= 8, max_depth
    pts = np.random.default_rng(3).uniform(0.0, 1.0, (4000, 3))
    got = oracle.eval_points(comp.prims, comp.program, pts)
    want = ref_value(tree, pts)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


def test_shallow_trees_keep_their_natural_order():
    """Where the left operand is at least as deep, the program is the left-first one."""
    a, b, c = X.sphere(0.1, (0.2, 0.2, 0.2)), X.sphere(0.1, (0.5, 0.5, 0.5)), X.sphere(0.1, (0.7, 0.7, 0.7))
    comp = X.compile_recipe(X.subtract(X.union(a, b, k=0.05), c, k=0.05))
    assert list(comp.program["op"]) == [X.OP_PUSH, X.OP_PUSH, X.OP_UNION, X.OP_PUSH, X.OP_SUBTRACT]
    assert (comp.prims["s"] > 0).all()
