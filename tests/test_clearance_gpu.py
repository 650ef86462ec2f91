"""EDT consumers on the GPU (field_b200.clearance through libfield_b200.so) against the reference's
golden arrays and the oracle: node map, edges and CSR structure bit for bit, the clearance and the
validity mask bit for bit; conductances and Laplacian values within 2 ulp (CUDA's float64 pow against
the host libm's: rtol 5e-16).  Full size: the 512^3 obstacle grid of the default EDT through
size-independent properties (counts, row sums, symmetry)."""
import numpy as np
import pytest

import oracle
from conftest import GOLDEN

pytestmark = pytest.mark.gpu
RTOL = 5e-16  # 2 ulp of float64 (conductances: m * sqrt(m) on the device, libm pow on the host)
RTOL_L = 1e-15  # Laplacian values: diagonals sum up to six conductances


def check_network(got, want_n, want):
    n, node, u, v, kond, L = got
    assert n == want_n
    assert np.array_equal(node, want["nodkarta"])
    assert np.array_equal(u, want["u"]) and np.array_equal(v, want["v"])
    np.testing.assert_allclose(kond, want["kond"], rtol=RTOL, atol=0)
    assert np.array_equal(L.indptr, want["indptr"]) and np.array_equal(L.indices, want["indices"])
    np.testing.assert_allclose(L.data, want["data"], rtol=RTOL_L, atol=0)


def oracle_dict(occ, E, pitch, p_kond):
    n, node, u, v, kond, indptr, indices, data = oracle.lattice_laplacian(occ, E, pitch, p_kond)
    return n, dict(nodkarta=node, u=u, v=v, kond=kond, indptr=indptr, indices=indices, data=data)


def test_golden_cases_equal_the_reference():
    import field_b200.clearance as C
    with np.load(GOLDEN / "clearance_golden.npz") as z:
        for k in range(8):
            g = {name.split("/", 1)[1]: z[name] for name in z.files if name.startswith(f"{k}/")}
            pitch, p_kond, min_r, margin, n = (float(x) for x in g["params"])
            E = C.edt_mm(g["occ"], pitch)
            assert E.dtype == np.float64 and np.array_equal(E, g["edt_mm"])
            assert np.array_equal(C.giltig_frirum(g["occ"], E, min_r, margin), g["valid"])
            check_network(C.bygg_gitterlaplacian(g["occ"], g["edt_mm"], pitch, p_kond), int(n), g)


@pytest.mark.parametrize("shape,frac,pitch,p_kond", [((64, 64, 64), 0.08, 0.25, 1.5),
                                                       ((100, 37, 129), 0.3, 1.7, 1.5),
                                                       ((33, 1, 70), 0.5, 0.9, 2.0),
                                                       ((48, 48, 48), 0.02, 1.0, 0.0)])
def test_seeded_grids_equal_the_oracle(shape, frac, pitch, p_kond):
    import field_b200.clearance as C
    rng = np.random.default_rng(hash(shape) % 2 ** 32)
    occ = rng.random(shape) < frac
    occ.flat[0] = True
    E = C.edt_mm(occ, pitch)
    assert np.array_equal(E, oracle.clearance_mm(occ, pitch))
    n, want = oracle_dict(occ, E, pitch, p_kond)
    check_network(C.bygg_gitterlaplacian(occ, E, pitch, p_kond), n, want)


def test_edge_cases():
    import field_b200.clearance as C
    # every cell occupied: no node, empty rows
    occ = np.ones((4, 5, 6), bool)
    n, node, u, v, kond, L = C.bygg_gitterlaplacian(occ, np.zeros(occ.shape), 1.0)
    assert n == 0 and (node == -1).all() and u.size == 0 and L.shape == (0, 0) and list(L.indptr) == [0]
    # one free cell without free neighbours: a node with an empty row
    occ[2, 2, 2] = False
    n, node, u, v, kond, L = C.bygg_gitterlaplacian(occ, np.ones(occ.shape), 1.0)
    assert n == 1 and node[2, 2, 2] == 0 and u.size == 0 and list(L.indptr) == [0, 0]
    # 1-D and 2-D grids run as 3-D ones with leading unit axes
    rng = np.random.default_rng(4)
    for shape in ((57,), (23, 31)):
        occ = rng.random(shape) < 0.3
        E = rng.uniform(0.0, 5.0, shape)
        n, want = oracle_dict(occ, E, 0.7, 1.5)
        check_network(C.bygg_gitterlaplacian(occ, E, 0.7, 1.5), n, want)
    # NaN clearance propagates through the floor as np.maximum does
    occ = np.zeros((3, 3, 3), bool)
    E = np.ones(occ.shape)
    E[1, 1, 1] = np.nan
    n, node, u, v, kond, L = C.bygg_gitterlaplacian(occ, E, 1.0)
    n2, want = oracle_dict(occ, E, 1.0, 1.5)
    assert np.array_equal(np.isnan(kond), np.isnan(want["kond"])) and np.isnan(kond).sum() == 6
    # an obstacle-free grid has no clearance
    with pytest.raises(ValueError):
        C.edt_mm(np.zeros((4, 4, 4), bool), 1.0)


def test_device_tensors_stay_on_the_device():
    import torch
    import field_b200.clearance as C
    rng = np.random.default_rng(9)
    occ = rng.random((40, 50, 60)) < 0.1
    occ_d = torch.from_numpy(occ).cuda()
    E, n, node, u, v, kond, L = C.fritt_natverk(occ_d, 0.5)
    assert E.is_cuda and node.is_cuda and L.is_sparse_csr and L.values().is_cuda
    n2, want = oracle_dict(occ, E.cpu().numpy(), 0.5, 1.5)
    assert n == n2 and np.array_equal(node.cpu().numpy(), want["nodkarta"])
    assert np.array_equal(L.crow_indices().cpu().numpy(), want["indptr"])
    assert np.array_equal(L.col_indices().cpu().numpy(), want["indices"])
    np.testing.assert_allclose(L.values().cpu().numpy(), want["data"], rtol=RTOL_L, atol=0)
    valid = C.giltig_frirum(occ_d, E, 1.0, 0.5)
    assert valid.is_cuda and np.array_equal(valid.cpu().numpy(), (~occ) & (E.cpu().numpy() >= 1.5))


def test_full_size_properties():
    """512^3 obstacle grid (2000 boxes, 8 % fill): node count, edge counts per axis, CSR entries,
    zero row sums, symmetry of the edge list, and the clearance against the squared EDT."""
    import torch
    import field_b200.clearance as C
    import field_b200.recipes as R
    occ = torch.from_numpy(R.obstacle_grid(seed=2, n=512, n_boxes=2000, fill=0.08)).cuda().bool()
    E, n, node, u, v, kond, L = C.fritt_natverk(occ, 0.01)
    free = ~occ
    assert n == int(free.sum())
    pairs = [free[:-1] & free[1:], free[:, :-1] & free[:, 1:], free[:, :, :-1] & free[:, :, 1:]]
    assert u.numel() == sum(int(p.sum()) for p in pairs)
    deg = torch.zeros(free.shape, dtype=torch.int32, device=occ.device)
    deg[:-1] += pairs[0]; deg[1:] += pairs[0]
    deg[:, :-1] += pairs[1]; deg[:, 1:] += pairs[1]
    deg[:, :, :-1] += pairs[2]; deg[:, :, 1:] += pairs[2]
    assert L.values().numel() == int(deg[free].sum()) + int((deg[free] > 0).sum())
    assert bool((node[free] == torch.arange(n, device=occ.device, dtype=torch.int32)).all())
    assert bool((node[occ] == -1).all())
    assert bool((u < v).all())
    rows = torch.repeat_interleave(torch.arange(n, device=occ.device),
                                   L.crow_indices()[1:].long() - L.crow_indices()[:-1].long())
    rsum = torch.zeros(n, dtype=torch.float64, device=occ.device).index_add_(0, rows, L.values())
    rabs = torch.zeros(n, dtype=torch.float64, device=occ.device).index_add_(0, rows, L.values().abs())
    assert bool((rsum.abs() <= 1e-14 * rabs).all())
    # each edge appears twice off the diagonal with -kond
    off = L.col_indices().long() != rows
    assert int(off.sum()) == 2 * u.numel()
    assert torch.equal(torch.sort(-L.values()[off]).values, torch.sort(torch.cat([kond, kond])).values)
    # clearance equals the float64 root of the squared EDT times the pitch
    import field_b200.edt as ED
    sq = ED.squared_distance_device(occ.view(torch.uint8), sites_nonzero=True)
    assert torch.equal(E, sq.double().sqrt() * 0.01)


def test_host_results_reuse_the_page_locked_pool():
    """Host results are views of pooled page-locked blocks: once a call's arrays are dropped, the
    next call of the same size allocates no new page-locked memory, and its arrays are correct."""
    import gc
    import field_b200.clearance as C
    rng = np.random.default_rng(21)
    occ = rng.random((30, 40, 50)) < 0.15
    E = C.edt_mm(occ, 0.3)
    first = C.bygg_gitterlaplacian(occ, E, 0.3)
    want_n, want = oracle_dict(occ, E, 0.3, 1.5)
    check_network(first, want_n, want)
    del first
    gc.collect()
    before = C._POOL.allocated
    second = C.bygg_gitterlaplacian(occ, E, 0.3)
    assert C._POOL.allocated == before
    check_network(second, want_n, want)
