"""EDT consumers on the CPU: the oracle's restatements (clearance in millimetres, the route-validity
mask, the lattice Laplacian of src/field_engine/opt/laplaceflode_v1.py:69-97) against the golden
arrays the reference module itself produced (tests/golden/make_clearance_golden.py), and the host
argument checks of field_b200.clearance (which run before any device call)."""
import numpy as np
import pytest

import oracle
from conftest import GOLDEN

CASES = 8


def golden_case(z, k):
    return {name.split("/", 1)[1]: z[name] for name in z.files if name.startswith(f"{k}/")}


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN / "clearance_golden.npz") as z:
        return [golden_case(z, k) for k in range(CASES)]


def test_oracle_clearance_equals_reference(golden):
    for g in golden:
        pitch = float(g["params"][0])
        assert np.array_equal(oracle.clearance_mm(g["occ"], pitch), g["edt_mm"])


def test_oracle_lattice_laplacian_equals_reference(golden):
    for g in golden:
        pitch, p_kond = float(g["params"][0]), float(g["params"][1])
        n, node, u, v, kond, indptr, indices, data = oracle.lattice_laplacian(g["occ"], g["edt_mm"], pitch, p_kond)
        assert n == int(g["params"][4])
        for got, want in ((node, "nodkarta"), (u, "u"), (v, "v"), (kond, "kond"), (indptr, "indptr"),
                          (indices, "indices"), (data, "data")):
            assert np.array_equal(got, g[want]), want


def test_route_validity_mask_rule(golden):
    for g in golden:
        min_r, margin = float(g["params"][2]), float(g["params"][3])
        assert np.array_equal((~g["occ"]) & (g["edt_mm"] >= min_r + margin), g["valid"])


def test_laplacian_rows_sum_to_zero_and_are_symmetric(golden):
    from scipy import sparse
    for g in golden:
        n = int(g["params"][4])
        L = sparse.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
        assert abs(L - L.T).max() == 0 if n else True
        if n:
            scale = np.abs(L).sum(axis=1).A.ravel() + 1e-300
            assert np.all(np.abs(L.sum(axis=1).A.ravel()) <= 1e-14 * scale)


def test_host_checks_reject_bad_input():
    import field_b200.clearance as C
    with pytest.raises(ValueError):
        C.bygg_gitterlaplacian(np.zeros((2, 2, 2), np.uint8), np.zeros((2, 2, 2)), 1.0)
    with pytest.raises(ValueError):
        C.bygg_gitterlaplacian(np.zeros((2, 2, 2, 2), bool), np.zeros((2, 2, 2, 2)), 1.0)
    with pytest.raises(ValueError):
        C.giltig_frirum(np.zeros((0, 2, 2), bool), np.zeros((0, 2, 2)), 1.0, 0.5)
    with pytest.raises(ValueError):
        C.edt_mm([[0, 1]], 1.0)
